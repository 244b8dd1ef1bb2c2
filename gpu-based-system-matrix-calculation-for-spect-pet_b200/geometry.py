"""Parameter-file layout and seeded synthetic geometries.

The four parameter files are flat float32 arrays with fixed read sizes
(reference: PEGen_RayTracing_CircularHole/PEGen_CircularHole.cpp:33-56 reads
80000/80000/100/100 floats).  The index layout follows the reference kernels,
not the README, where the two disagree:

* Collimator (PESysMatGen.cu:961-990, :1151-1181, :1240-1262):
    [0]                 number of layers L
    [(m+1)*10 + k]      layer m header, k = 0 nHoles, 1 width (x), 2 thickness (y),
                        3 height (z), 4 y offset from layer 0, 5 mu_tot, 6 mu_pe, 7 mu_C
    [100 + 9*h + k]     hole h (global numbering, layer 0 first), k = 0 x, 1 y1, 2 y2,
                        3 z, 4 radius, 5 mu_tot, 6 mu_pe, 7 mu_C, 8 flag
* Detector (PESysMatGen.cu:1058-1064):
    [0]                 number of crystals D
    [12*d + k]          crystal d, k = 1 x, 2 y, 3 z, 4 width (x), 5 thickness (y),
                        6 height (z), 7 mu_tot, 8 mu_pe, 9 mu_C, 10 energy resolution,
                        11 rotation about y, 12 flag
* Image (PESysMatGen.cu:995-1009): [0..2] voxel counts, [3..5] voxel sizes,
    [6] rotations, [7] angle per rotation, [8..10] FOV shift, [11] FOV-to-collimator
    distance, [20] rotation index of the current call (set by the caller).
* Physics (ReadMe.md:183-196; scatter.cu:1144-1150): [0] use Compton, [1..3] save
    flags, [4] same energy window, [5] lower, [6] upper, [7] photopeak energy (keV),
    [8] compute crystal relationship bitmap, [9] compute collimator bitmap.

Geometries here are synthetic stand-ins: the reference ships no parameter files.
Values are chosen as stated in the docstring of each builder.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

N_COLLIMATOR = 80000
N_DETECTOR = 80000
N_IMAGE = 100
N_PHYSICS = 100

MAX_LAYERS = 9              # the 10th layer header would overlap the hole table at index 100
MAX_HOLES = (N_COLLIMATOR - 100) // 9
MAX_CRYSTALS = (N_DETECTOR - 1) // 12

# 140.5 keV in tungsten and NaI (per mm); the photoelectric share of tungsten is a
# stated generator choice because only the total coefficient is specified.
MU_W_TOTAL = 3.4
MU_W_PE_FRACTION = 0.87


@dataclass
class Geometry:
    """One system: the four float32 parameter arrays plus a short name."""
    name: str
    collimator: np.ndarray
    detector: np.ndarray
    image: np.ndarray
    physics: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n_det(self) -> int:
        return int(math.floor(float(self.detector[0]) + 0.0001))

    @property
    def n_vox(self) -> int:
        nx, ny, nz = (int(math.floor(float(self.image[i]) + 0.001)) for i in range(3))
        return nx * ny * nz

    @property
    def n_rot(self) -> int:
        return int(math.floor(float(self.image[6]) + 0.001))

    @property
    def n_layers(self) -> int:
        return int(math.floor(float(self.collimator[0]) + 0.000001))

    @property
    def n_holes(self) -> int:
        return sum(int(self.collimator[(m + 1) * 10]) for m in range(self.n_layers))

    @property
    def n_holes_layer0(self) -> int:
        return int(math.floor(float(self.collimator[10]) + 0.000001))

    def with_rotation(self, idx: int) -> "Geometry":
        img = self.image.copy()
        img[20] = float(idx)
        return Geometry(self.name, self.collimator, self.detector, img, self.physics, dict(self.meta))

    def write(self, directory: str) -> None:
        """Write Params_{Collimator,Detector,Image,Physics}.dat as the reference CLI reads them."""
        os.makedirs(directory, exist_ok=True)
        for fname, arr in (("Params_Collimator.dat", self.collimator),
                           ("Params_Detector.dat", self.detector),
                           ("Params_Image.dat", self.image),
                           ("Params_Physics.dat", self.physics)):
            np.asarray(arr, dtype=np.float32).tofile(os.path.join(directory, fname))


def read_params(directory: str, name: str = "files") -> Geometry:
    """Read the four parameter files; short files are zero-padded like the reference's
    zero-initialised `new float[n]()` buffers followed by a short fread."""
    out = []
    for fname, n in (("Params_Collimator.dat", N_COLLIMATOR), ("Params_Detector.dat", N_DETECTOR),
                     ("Params_Image.dat", N_IMAGE), ("Params_Physics.dat", N_PHYSICS)):
        raw = np.fromfile(os.path.join(directory, fname), dtype=np.float32)
        arr = np.zeros(n, dtype=np.float32)
        arr[:min(n, raw.size)] = raw[:n]
        out.append(arr)
    return Geometry(name, *out)


def _physics(same_window=True, lo=126.45, hi=154.55, energy=140.5, compton=1.0):
    p = np.zeros(N_PHYSICS, dtype=np.float32)
    p[:10] = [compton, 1, 1, 1, 1.0 if same_window else 0.0, lo, hi, energy, 1, 1]
    return p


def _image(n, width, fov2coll, n_rot=1, dtheta=0.0, shift=(0.0, 0.0, 0.0)):
    im = np.zeros(N_IMAGE, dtype=np.float32)
    im[0:3] = n
    im[3:6] = width
    im[6] = n_rot
    im[7] = dtheta
    im[8:11] = shift
    im[11] = fov2coll
    return im


class _CollimatorBuilder:
    def __init__(self):
        self.layers = []

    def add_layer(self, width, thickness, height, y_offset, mu_tot, mu_pe, mu_c, holes):
        """holes: iterable of (x, z, radius); y extent is the layer's own thickness."""
        self.layers.append((width, thickness, height, y_offset, mu_tot, mu_pe, mu_c, list(holes)))

    def build(self) -> np.ndarray:
        c = np.zeros(N_COLLIMATOR, dtype=np.float32)
        if len(self.layers) > MAX_LAYERS:
            raise ValueError("too many collimator layers")
        c[0] = len(self.layers)
        h = 0
        for m, (w, t, ht, yo, mt, mp, mc, holes) in enumerate(self.layers):
            base = (m + 1) * 10
            c[base:base + 8] = [len(holes), w, t, ht, yo, mt, mp, mc]
            for (x, z, r) in holes:
                if h >= MAX_HOLES:
                    raise ValueError("too many holes")
                o = 100 + 9 * h
                c[o:o + 9] = [x, yo - t / 2.0, yo + t / 2.0, z, r, 0.0, 0.0, 0.0, 1.0]
                h += 1
        return c


def _detector(centres, size, mu=(0.23, 0.18), eres=0.10, rotations=None):
    """centres: (D,3) raw coordinates (y measured from collimator layer 0 centre)."""
    centres = np.asarray(centres, dtype=np.float64)
    n = centres.shape[0]
    if n > MAX_CRYSTALS:
        raise ValueError("too many crystals")
    d = np.zeros(N_DETECTOR, dtype=np.float32)
    d[0] = n
    mt, mp = mu
    for i in range(n):
        o = 12 * i
        rot = 0.0 if rotations is None else float(rotations[i])
        d[o + 1:o + 13] = [centres[i, 0], centres[i, 1], centres[i, 2], size[0], size[1], size[2],
                           mt, mp, mt - mp, eres, rot, 1.0]
    return d


def _square_holes(n_side, pitch, radius):
    off = (n_side - 1) / 2.0
    return [((i - off) * pitch, (j - off) * pitch, radius) for j in range(n_side) for i in range(n_side)]


def _hex_holes(n_cols, n_rows, pitch, radius):
    dz = pitch * math.sqrt(3.0) / 2.0
    out = []
    for j in range(n_rows):
        shift = 0.5 * pitch if (j % 2) else 0.0
        for i in range(n_cols):
            x = (i - (n_cols - 1) / 2.0) * pitch + shift - 0.25 * pitch
            z = (j - (n_rows - 1) / 2.0) * dz
            out.append((x, z, radius))
    return out


def _crystal_grid(nx, nz, pitch, y):
    xs = (np.arange(nx) - (nx - 1) / 2.0) * pitch
    zs = (np.arange(nz) - (nz - 1) / 2.0) * pitch
    return [(x, y, z) for z in zs for x in xs]


def _w_layer(cb, width, thickness, height, holes, y_offset=0.0, mu=MU_W_TOTAL):
    cb.add_layer(width, thickness, height, y_offset, mu, mu * MU_W_PE_FRACTION,
                 mu * (1.0 - MU_W_PE_FRACTION), holes)


def config1() -> Geometry:
    """Plain PE system: 32x32x1 voxels of 1 mm, tungsten plate T=10 mm (32x32 mm, a
    generator choice covering the detector) with 7x7 holes of 1.0 mm diameter at 2.0 mm
    pitch, front face 50 mm from the FOV centre; NaI 16x16 crystals 2x5x2 mm at 2 mm pitch,
    2 mm behind the plate."""
    t = 10.0
    cb = _CollimatorBuilder()
    _w_layer(cb, 32.0, t, 32.0, _square_holes(7, 2.0, 0.5))
    det = _detector(_crystal_grid(16, 16, 2.0, t / 2 + 2.0 + 2.5), (2.0, 5.0, 2.0))
    return Geometry("config1", cb.build(), det, _image((32, 32, 1), (1, 1, 1), 50.0 + t / 2),
                    _physics())


def config2(nz: int = 32) -> Geometry:
    """Production PE system: 96x96xnz voxels of 1 mm; hexagonal 48x48 holes, 1.5 mm
    diameter, 2.0 mm pitch, tungsten 20 mm thick (plate 104x104 mm, generator choice);
    FOV-to-collimator 58 + T/2 mm (clears the 48 mm FOV half-depth); NaI 64x64 crystals
    1.6x6x1.6 mm at 1.6 mm pitch, 2 mm behind the plate."""
    t = 20.0
    cb = _CollimatorBuilder()
    _w_layer(cb, 104.0, t, 104.0, _hex_holes(48, 48, 2.0, 0.75))
    det = _detector(_crystal_grid(64, 64, 1.6, t / 2 + 2.0 + 3.0), (1.6, 6.0, 1.6))
    return Geometry("config2", cb.build(), det, _image((96, 96, nz), (1, 1, 1), 58.0 + t / 2),
                    _physics())


def config3() -> Geometry:
    """PE + primary Compton: 48x48x16 voxels of 2 mm; collimator of config 1 with 32x32
    holes (plate 64x64 mm); NaI 32x32 crystals 2x6x2 mm at 2 mm pitch, 2 mm behind."""
    t = 10.0
    cb = _CollimatorBuilder()
    _w_layer(cb, 64.0, t, 64.0, _square_holes(32, 2.0, 0.5))
    det = _detector(_crystal_grid(32, 32, 2.0, t / 2 + 2.0 + 3.0), (2.0, 6.0, 2.0))
    return Geometry("config3", cb.build(), det, _image((48, 48, 16), (2, 2, 2), 50.0 + t / 2),
                    _physics())


def mini(seed: int = 0, rotated: bool = False, layers: int = 1, n_rot: int = 1,
         nvox=(8, 8, 2), ncry=(6, 6), nholes=5) -> Geometry:
    """Small seeded system for CPU-oracle tests (seconds of oracle time).

    `rotated` gives every crystal a seeded rotation about y and shifts the FOV;
    `layers` > 1 stacks tungsten layers at increasing y offset."""
    rng = np.random.default_rng(seed)
    t = 6.0
    cb = _CollimatorBuilder()
    holes = _square_holes(nholes, 2.0, 0.5 + 0.1 * rng.random())
    for m in range(layers):
        _w_layer(cb, 2.0 * nholes + 4.0, t, 2.0 * nholes + 4.0, holes, y_offset=m * (t + 1.0))
    y_det = (layers - 1) * (t + 1.0) + t / 2 + 2.0 + 2.5
    centres = _crystal_grid(ncry[0], ncry[1], 2.0, y_det)
    rots = rng.uniform(0, 2 * math.pi, size=len(centres)) if rotated else None
    det = _detector(centres, (2.0, 5.0, 2.0), rotations=rots)
    shift = tuple(rng.uniform(-1.0, 1.0, size=3)) if rotated else (0.0, 0.0, 0.0)
    img = _image(nvox, (2.0, 2.0, 2.0), 30.0 + t / 2, n_rot=n_rot,
                 dtheta=(2 * math.pi / n_rot if n_rot > 1 else 0.0), shift=shift)
    return Geometry(f"mini{seed}{'r' if rotated else ''}{layers}", cb.build(), det, img, _physics())


def config4(n_instances: int = 64, seed: int = 4) -> list:
    """Batched design sweep: `n_instances` systems with seeded hole diameter U[0.8, 2.0] mm and
    tungsten plate thickness U[5, 25] mm (32x32 holes at 2.5 mm pitch, plate 84x84 mm, so
    every diameter fits the pitch), each with its own number of rotations U{12..60} and
    step 2*pi/n; 32x32x16 voxels of 2 mm, front face 50 mm from the FOV centre; NaI 32x32
    crystals 2x5x2 mm at 2 mm pitch, 2 mm behind the plate.  Returns Geometry objects whose
    image parameters carry n_rot and the step."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_instances):
        dia = float(rng.uniform(0.8, 2.0))
        t = float(rng.uniform(5.0, 25.0))
        n_rot = int(rng.integers(12, 61))
        cb = _CollimatorBuilder()
        _w_layer(cb, 84.0, t, 84.0, _square_holes(32, 2.5, dia / 2.0))
        det = _detector(_crystal_grid(32, 32, 2.0, t / 2 + 2.0 + 2.5), (2.0, 5.0, 2.0))
        img = _image((32, 32, 16), (2, 2, 2), 50.0 + t / 2, n_rot=n_rot, dtheta=2 * math.pi / n_rot)
        out.append(Geometry(f"config4_{k}", cb.build(), det, img, _physics(),
                            dict(hole_diameter=dia, thickness=t, n_rot=n_rot)))
    return out


def apply_theta(geo: Geometry, theta) -> Geometry:
    """The system at parameters theta = (mu_W, mu_crystal, hole radius, dx, dy, dz, tilt):
    every layer's mu_total and every crystal's mu_total (mu_pe kept, mu_C = mu_total - mu_pe)
    and every hole's radius are set; hole centres are rotated by `tilt` (radians) about the
    y axis and shifted by (dx, dz); hole caps and layer planes are shifted by dy.  Coordinates
    are computed in double and rounded to the float parameter format once."""
    mu_w, mu_c, radius, dx, dy, dz, tilt = (float(t) for t in theta)
    col = geo.collimator.astype(np.float64)
    det = geo.detector.astype(np.float64)
    n_layers = int(round(col[0]))
    for m in range(n_layers):
        base = (m + 1) * 10
        col[base + 4] += dy
        col[base + 5] = mu_w
    n_holes = geo.n_holes
    h = col[100:100 + 9 * n_holes].reshape(n_holes, 9)
    x, z = h[:, 0].copy(), h[:, 3].copy()
    c, s_ = math.cos(tilt), math.sin(tilt)
    h[:, 0] = x * c - z * s_ + dx
    h[:, 3] = x * s_ + z * c + dz
    h[:, 1] += dy
    h[:, 2] += dy
    h[:, 4] = radius
    col[100:100 + 9 * n_holes] = h.reshape(-1)
    n_det = geo.n_det
    d = det[1:1 + 12 * n_det].reshape(n_det, 12)
    changed = d[:, 6] != np.float64(np.float32(mu_c))
    d[changed, 8] = mu_c - d[changed, 7]
    d[:, 6] = mu_c
    det[1:1 + 12 * n_det] = d.reshape(-1)
    return Geometry(geo.name, col.astype(np.float32), det.astype(np.float32), geo.image, geo.physics,
                    dict(geo.meta, theta=tuple(float(t) for t in theta)))


def apply_theta_shapes(shapes, theta) -> np.ndarray:
    """Elliptical hole shapes (n_holes, 3) rows (rho_x, rho_z, theta_h) at parameters theta:
    the tilt turns every elliptical hole's frame with the hole pattern (theta_h + tilt,
    computed in double and rounded to float once); circular rows (rho_x <= 0) are kept."""
    out = np.array(shapes, dtype=np.float32).reshape(-1, 3).copy()
    tilt = float(theta[6])
    ell = out[:, 0] > 0
    out[ell, 2] = (out[ell, 2].astype(np.float64) + tilt).astype(np.float32)
    return out


def theta_of(geo: Geometry) -> np.ndarray:
    """Nominal theta of a system built here (layer 0 mu, crystal 0 mu, hole 0 radius, no
    shift or tilt)."""
    return np.array([float(geo.collimator[15]), float(geo.detector[7]), float(geo.collimator[104]),
                     0.0, 0.0, 0.0, 0.0])


def ellipsoid_phantom(n, width, n_ellipsoids=5, seed=5) -> np.ndarray:
    """Seeded phantom of uniform ellipsoids (activity U[0.5, 4]) on an n = (nx, ny, nz) grid of
    voxel size `width`, flattened as ix + nx*(iy + ny*iz)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    xs = (np.arange(nx) - nx / 2 + 0.5) * width[0]
    ys = (np.arange(ny) - ny / 2 + 0.5) * width[1]
    zs = (np.arange(nz) - nz / 2 + 0.5) * width[2]
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    img = np.zeros((nz, ny, nx))
    half = np.array([nx * width[0], ny * width[1], nz * width[2]]) / 2
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.5, 0.5, 3) * half
        r = rng.uniform(0.15, 0.4, 3) * half
        a = rng.uniform(0.5, 4.0)
        inside = ((X - c[0]) / r[0]) ** 2 + ((Y - c[1]) / r[1]) ** 2 + ((Z - c[2]) / r[2]) ** 2 <= 1.0
        img[inside] += a
    return img.reshape(-1).astype(np.float32)


def config5(seed: int = 5):
    """Calibration problem: 64x64x16 voxels of 1 mm holding a seeded phantom of 5 uniform
    ellipsoids; tungsten plate T = 10 mm (100x100 mm, a generator choice covering the
    detector) with 32x32 holes of radius 0.75 mm at 2.0 mm pitch, front face 40 mm from the
    FOV centre (clears the 32 mm half-depth); NaI 48x48 crystals 2x5x2 mm at 2 mm pitch, 2 mm
    behind the plate.  Returns (geometry at nominal theta, phantom x, nominal theta, true
    theta*) with theta* = nominal + offsets N(0, 0.1 mm) and tilt N(0, 0.2 deg)."""
    t = 10.0
    cb = _CollimatorBuilder()
    _w_layer(cb, 100.0, t, 100.0, _square_holes(32, 2.0, 0.75))
    det = _detector(_crystal_grid(48, 48, 2.0, t / 2 + 2.0 + 2.5), (2.0, 5.0, 2.0))
    geo = Geometry("config5", cb.build(), det, _image((64, 64, 16), (1, 1, 1), 40.0 + t / 2), _physics())
    x = ellipsoid_phantom((64, 64, 16), (1.0, 1.0, 1.0), 5, seed)
    rng = np.random.default_rng(seed + 1)
    theta0 = theta_of(geo)
    theta_star = theta0.copy()
    theta_star[3:6] += rng.normal(0.0, 0.1, 3)
    theta_star[6] += math.radians(rng.normal(0.0, 0.2))
    return geo, x, theta0, theta_star


CONFIGS = {"config1": config1, "config2": config2, "config3": config3}


def by_name(name: str) -> Geometry:
    if name in CONFIGS:
        return CONFIGS[name]()
    if name.startswith("mini"):
        return mini()
    raise KeyError(name)


def voxel_slab(geo: Geometry, iz: int, iy0: int = 0, ny: int | None = None) -> Geometry:
    """The same system restricted to voxel rows iy0..iy0+ny-1 of z-plane iz.

    Voxel centres are (i - N/2 + 0.5) * w + shift (PESysMatGen.cu:1041-1047).  With the
    restricted grid the FOV shift absorbs the offset, and for integer or half-integer
    offsets times the voxel size the sub-grid reproduces the full grid's voxel centres
    bit for bit, so every matrix element of the slab equals the full matrix element."""
    nx = int(round(float(geo.image[0])))
    ny_full = int(round(float(geo.image[1])))
    nz_full = int(round(float(geo.image[2])))
    ny = ny_full if ny is None else ny
    img = geo.image.copy()
    wy, wz = float(geo.image[4]), float(geo.image[5])
    img[1] = ny
    img[2] = 1
    # centre of row block: offset of the sub-grid origin in units of voxels
    off_y = (iy0 - ny_full / 2.0) - (0 - ny / 2.0)
    off_z = (iz - nz_full / 2.0 + 0.5) - (0 - 0.5 + 0.5)
    img[9] = np.float32(float(geo.image[9]) + off_y * wy)
    img[10] = np.float32(float(geo.image[10]) + off_z * wz)
    meta = dict(geo.meta)
    meta.update(slab=(iz, iy0, ny), parent=geo.name)
    return Geometry(f"{geo.name}_z{iz}_y{iy0}+{ny}", geo.collimator, geo.detector, img, geo.physics, meta)
