"""Generate the golden fixtures by running the reference's own programs on a GPU.

The reference ships no tests and no fixtures, so these vectors are produced by its
unmodified CUDA sources compiled for sm_100a (oracle/Makefile, target `ref`) and called
through the reference host entry points (PESysMatGen, the three `scatter` programs).
Run on a machine with a GPU:

    python tests/golden/make_golden.py --out golden_out

and copy the resulting .npz files into tests/golden/.  Each fixture stores the four
parameter arrays it was made from, so it does not depend on the generator staying
unchanged.  Large matrices are stored as a fixed row sample (`rows`); bitmaps that are
too large are stored as a checksum and a word sample.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_lib  # noqa: E402

_spec = importlib.util.spec_from_file_location(
    "sysmat_geometry",
    os.path.join(ROOT, "gpu-based-system-matrix-calculation-for-spect-pet_b200", "geometry.py"))
geometry = importlib.util.module_from_spec(_spec)
sys.modules["sysmat_geometry"] = geometry
_spec.loader.exec_module(geometry)

MAX_FULL = 300_000        # store whole matrices up to this many elements
MAX_BITMAP_WORDS = 65536


def _geo_arrays(geo):
    return dict(collimator=geo.collimator, detector=geo.detector, image=geo.image,
                physics=geo.physics)


def _rows(n_det, n_vox):
    if n_det * n_vox <= MAX_FULL:
        return np.arange(n_det)
    step = max(1, (n_det * n_vox) // MAX_FULL + 1)
    return np.arange(0, n_det, step)


def _bitmap_fields(prefix, words):
    out = {f"{prefix}_sha256": np.frombuffer(hashlib.sha256(words.tobytes()).digest(), np.uint8),
           f"{prefix}_nwords": np.array(words.size, np.int64)}
    if words.size <= MAX_BITMAP_WORDS:
        out[f"{prefix}_words"] = words
    else:
        idx = np.linspace(0, words.size - 1, MAX_BITMAP_WORDS).astype(np.int64)
        out[f"{prefix}_sample_idx"] = idx
        out[f"{prefix}_sample_words"] = words[idx]
    return out


def run_case(name, geo, scatter_variants, outdir, timings):
    rec = _geo_arrays(geo)
    t0 = time.perf_counter()
    pe = ref_lib.pe(geo)
    timings[f"{name}/pe_s"] = time.perf_counter() - t0
    rows = _rows(geo.n_det, geo.n_vox)
    rec["rows"] = rows
    rec["pe"] = pe[rows]
    for variant in scatter_variants:
        sgeo = geo
        t0 = time.perf_counter()
        dst, bitmaps = ref_lib.scatter(sgeo, pe, variant=variant)
        timings[f"{name}/scatter_{variant}_s"] = time.perf_counter() - t0
        rec[f"scatter_{variant}"] = dst[rows]
        for key, words in bitmaps.items():
            if f"bitmap_{key}_sha256" not in rec:
                rec.update(_bitmap_fields(f"bitmap_{key}", words))
    np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **rec)
    print(f"{name}: D={geo.n_det} V={geo.n_vox} rows={rows.size} "
          f"pe_max={float(pe.max()):.4e}", flush=True)


def cases():
    out = []
    g = geometry.mini(seed=0)
    out.append(("mini0", g, ("combined", "collimator", "crystal")))
    g = geometry.mini(seed=1, rotated=True, layers=2, n_rot=1)
    img = g.image.copy()
    img[7] = 0.3            # angle per rotation, rotation index 1 below
    g = geometry.Geometry("mini1r2", g.collimator, g.detector, img, g.physics).with_rotation(1)
    out.append(("mini1r2", g, ("combined", "collimator", "crystal")))
    g = geometry.mini(seed=2, nvox=(10, 6, 3), ncry=(5, 7), nholes=6)
    phys = g.physics.copy()
    phys[4] = 0.0           # per-crystal energy window from the crystal's resolution
    g = geometry.Geometry("mini2w", g.collimator, g.detector, g.image, phys)
    out.append(("mini2w", g, ("combined",)))
    out.append(("config1", geometry.config1(), ()))
    out.append(("config2_strip", geometry.voxel_slab(geometry.config2(), 16, 47, 2), ()))
    out.append(("config3_z8", geometry.voxel_slab(geometry.config3(), 8),
                ("combined", "collimator")))
    # configuration 4 (design sweep): two instances at one of their rotations, voxel row 16 of
    # z-plane 8 x all crystals; configuration 5 (calibration system at nominal theta): voxel
    # row 32 of z-plane 8 x all crystals
    g4 = geometry.config4()
    for k, r in ((7, 5), (40, 11)):
        out.append((f"config4_i{k}r{r}", geometry.voxel_slab(g4[k].with_rotation(r), 8, 16, 1), ()))
    out.append(("config5_z8", geometry.voxel_slab(geometry.config5()[0], 8, 32, 1), ()))
    return out


def ellipse_args(n=4000, seed=17):
    """Seeded arguments for the elliptical-cylinder chord: rays from a voxel region to a
    detector region crossing a plate at y in [40, 50], ellipses near the crossing (semi-axes
    0.3-1.5 mm, any orientation), with a tenth of them circles."""
    rng = np.random.default_rng(seed)
    a = np.zeros((n, 13), dtype=np.float32)
    xi, yi, zi = rng.uniform(-20, 20, n), rng.uniform(-30, 0, n), rng.uniform(-20, 20, n)
    xo, yo, zo = rng.uniform(-30, 30, n), np.full(n, 60.0), rng.uniform(-30, 30, n)
    yy = rng.uniform(40, 50, n)
    s = (yy - yi) / (yo - yi)
    rx, rz = rng.uniform(0.3, 1.5, n), rng.uniform(0.3, 1.5, n)
    circ = rng.random(n) < 0.1
    rz[circ] = rx[circ]
    xc = xi + s * (xo - xi) + rng.normal(0, 1.0, n)
    zc = zi + s * (zo - zi) + rng.normal(0, 1.0, n)
    a[:] = np.stack([xi, yi, zi, xo, yo, zo, xc, np.full(n, 40.0), np.full(n, 50.0), zc, rx, rz,
                     rng.uniform(0, np.pi, n)], 1)
    return a


def ellipse_case(outdir):
    args = ellipse_args()
    np.savez_compressed(os.path.join(outdir, "ellipse_chords.npz"), args=args, ref=ref_lib.ell_chords(args))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="golden_out")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    if not ref_lib.available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    os.makedirs(args.out, exist_ok=True)
    timings = {}
    for name, geo, variants in cases():
        if args.only and name not in args.only.split(","):
            continue
        run_case(name, geo, variants, args.out, timings)
    if not args.only or "ellipse" in args.only.split(","):
        ellipse_case(args.out)
    with open(os.path.join(args.out, "timings.json"), "w") as f:
        json.dump(timings, f, indent=1)
    print(json.dumps(timings))


if __name__ == "__main__":
    main()
