"""GPU tests of the local-coordinate FP32 mode (SYSMAT_MODE_LOCAL), through the C ABI.

The mode evaluates the reference's element program in float arithmetic arranged so that only
small, local quantities are rounded (oracle/oracle_local.h states the scheme; its CPU twin is
oracle.pe_local).  Its bar: within 1e-5 of the FP64 restatement on every element of systems
in generic position; on an exactly regular grid (configuration 1 as generated) some rays cross a
threshold of the program exactly, where the last bit of any evaluation decides the branch, and
those rare elements are bounded separately."""
import numpy as np
import pytest

from conftest import TOL, geometry, golden, oracle, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _local(torch, ctx, rotation=0.0, **blk):
    nd = blk.get("det_count", ctx.n_det)
    nv = blk.get("vox_count", ctx.n_vox)
    out = torch.empty((nd, nv), dtype=torch.float32, device="cuda")
    ctx.pe(out, rotation=rotation, mode=sysmat.MODE_LOCAL, **blk)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["mini0", "mini1r2", "mini2w"])
def test_local_mode_within_1e5_of_fp64(gpu, name):
    geo, z = golden(name)
    ctx = sysmat.Context(geo)
    a = _local(gpu, ctx, rotation=float(geo.image[20]))
    o64 = oracle.pe(geo, prec=64)
    r = rel_err(a, o64)
    assert a.max() > 0
    assert r.max() <= TOL and np.median(r) < 1e-6, (r.max(), np.median(r))
    # the reference's float program is further from FP64 on the same elements
    r_ref = rel_err(z["pe"], o64[z["rows"]])
    assert r[z["rows"]].max() < r_ref.max()
    # the device and its CPU twin evaluate the same float scheme (other fused multiply-adds
    # and summation order only)
    twin = oracle.pe_local(geo)
    assert np.median(rel_err(a, twin)) < 1e-6


def _config1_shifted():
    """Configuration 1 moved by a generic sub-micron offset: its voxel centres, hole rims and
    crystal faces sit on exact rationals, so many rays cross a threshold of the program exactly
    (an exit point on a hole's rim), where the last bit of any evaluation decides the branch;
    the shifted system has no such ties."""
    geo, _ = golden("config1")
    img = geo.image.copy()
    img[8] = np.float32(img[8] + 1.234e-4)
    img[10] = np.float32(img[10] - 0.567e-4)
    return geometry.Geometry("config1_shifted", geo.collimator, geo.detector, img, geo.physics)


def test_local_mode_config1_within_1e5_of_fp64(gpu):
    geo = _config1_shifted()
    ctx = sysmat.Context(geo)
    a = _local(gpu, ctx)
    o64 = oracle.pe(geo, prec=64)
    r = rel_err(a, o64)
    assert r.max() <= TOL and np.median(r) < 1e-6, (r.max(), np.median(r))
    assert r.max() < rel_err(oracle.pe(geo, prec=32), o64).max()


def test_local_mode_exact_config1_ties_are_rare(gpu):
    """On the exact grid the outliers are the exact ties described above: few, and each one a
    ray on a hole's rim (the element moves by the whole chord's attenuation)."""
    geo, _ = golden("config1")
    ctx = sysmat.Context(geo)
    a = _local(gpu, ctx)
    r = rel_err(a, oracle.pe(geo, prec=64))
    assert np.median(r) < 1e-7 and np.mean(r > TOL) < 0.005, (np.median(r), np.mean(r > TOL))


@pytest.mark.parametrize("seed", [14, 15])
def test_local_mode_on_fresh_seeded_systems(gpu, seed):
    g = geometry.mini(seed=seed, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4)).with_rotation(seed % 8)
    ctx = sysmat.Context(g)
    a = _local(gpu, ctx, rotation=float(seed % 8))
    r = rel_err(a, oracle.pe(g, prec=64))
    assert np.median(r) < 1e-6 and r.max() <= TOL, (np.median(r), r.max())


def test_local_mode_config2_full_size_sample(gpu):
    """Configuration 2 at full size: 8 crystals x 2 voxel rows of z-plane 16 against FP64."""
    torch = gpu
    geo = geometry.config2()
    ctx = sysmat.Context(geo)
    rows = np.sort(np.random.default_rng(6).choice(geo.n_det, 8, replace=False))
    v0, nv = 96 * 96 * 16 + 96 * 40, 96 * 2
    out = torch.empty((len(rows), nv), dtype=torch.float32, device="cuda")
    for i, d in enumerate(rows):
        ctx.pe(out[i:i + 1], det_begin=int(d), det_count=1, vox_begin=v0, vox_count=nv, mode=sysmat.MODE_LOCAL)
    a = out.cpu().numpy()
    o64 = oracle.pe(geo, prec=64, dets=rows, v0=v0, nv=nv)
    o32 = oracle.pe(geo, prec=32, dets=rows, v0=v0, nv=nv)
    r, r32 = rel_err(a, o64), rel_err(o32, o64)
    assert a.max() > 0
    assert r.max() <= TOL and np.median(r) < 1e-6, (np.median(r), r.max())
    assert r.max() < r32.max()                          # the float program's own error is larger


def test_local_blocks_equal_the_full_matrix(gpu):
    torch = gpu
    geo, _ = golden("mini1r2")
    ctx = sysmat.Context(geo)
    rot = float(geo.image[20])
    full = _local(torch, ctx, rotation=rot)
    for (d0, nd, v0, nv) in ((0, 3, 0, 17), (7, 5, 31, 40), (ctx.n_det - 1, 1, ctx.n_vox - 1, 1)):
        out = torch.full((nd, nv + 5), -1.0, dtype=torch.float32, device="cuda")
        ctx.pe(out[:, :nv], rotation=rot, det_begin=d0, det_count=nd, vox_begin=v0, vox_count=nv,
               mode=sysmat.MODE_LOCAL)
        blk = out.cpu().numpy()
        assert np.array_equal(blk[:, :nv], full[d0:d0 + nd, v0:v0 + nv])
        assert np.all(blk[:, nv:] == -1.0)


def test_local_mode_rejects_elliptical_holes(gpu):
    torch = gpu
    geo, _ = golden("mini0")
    ctx = sysmat.Context(geo)
    shapes = np.zeros((geo.n_holes, 3), dtype=np.float32)
    shapes[0] = (0.4, 0.3, 0.5)
    ctx.set_hole_shapes(shapes)
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    with pytest.raises(sysmat.SysmatError):
        ctx.pe(out, mode=sysmat.MODE_LOCAL)
