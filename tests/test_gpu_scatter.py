"""GPU parity tests of the relationship bitmaps and the primary-Compton scatter kernels,
through the C ABI, against the reference's own outputs and the CPU oracle."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from conftest import TOL, geometry, golden, oracle, rel_err, sysmat
from test_oracle import flip_explained

pytestmark = pytest.mark.gpu


def _pe(torch, ctx, geo):
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(out, rotation=float(geo.image[20]))
    return out


def _setup(torch, name):
    geo, z = golden(name)
    ctx = sysmat.Context(geo)
    bc, bh = ctx.bitmap_crystal(), ctx.bitmap_collimator()
    if z["pe"].shape[0] == geo.n_det:
        pe = torch.from_numpy(np.ascontiguousarray(z["pe"])).cuda()
    else:
        pe = _pe(torch, ctx, geo)
    ctx.scatter_prepare(bc, bh)
    return geo, z, ctx, bc, bh, pe


@pytest.mark.parametrize("name", ["mini0", "mini1r2", "mini2w", "config3_z8"])
def test_bitmaps_match_reference(gpu, name):
    geo, z = golden(name)
    ctx = sysmat.Context(geo)
    for key, t in (("crystal", ctx.bitmap_crystal()), ("collimator", ctx.bitmap_collimator())):
        h = t.cpu().numpy().view(np.uint32)
        assert h.size == int(z[f"bitmap_{key}_nwords"])
        assert hashlib.sha256(h.tobytes()).digest() == bytes(z[f"bitmap_{key}_sha256"])


CASES = [("mini0", "scatter_combined"), ("mini0", "scatter_collimator"), ("mini0", "scatter_crystal"),
         ("mini1r2", "scatter_combined"), ("mini1r2", "scatter_collimator"),
         ("mini2w", "scatter_combined"), ("config3_z8", "scatter_combined"),
         ("config3_z8", "scatter_collimator")]
PARTS = {"scatter_combined": (3, sysmat.HOLE_MODEL_COMBINED),
         "scatter_collimator": (2, sysmat.HOLE_MODEL_VARIANT),
         "scatter_crystal": (1, sysmat.HOLE_MODEL_COMBINED)}


@pytest.mark.parametrize("name,key", CASES)
def test_scatter_matches_reference(gpu, name, key):
    geo, z, ctx, bc, bh, pe = _setup(gpu, name)
    parts, model = PARTS[key]
    out = gpu.empty_like(pe)
    ctx.scatter(out, pe, parts=parts, hole_model=model, rotation=float(geo.image[20]))
    a = out.cpu().numpy()[z["rows"]]
    r = rel_err(a, z[key])
    assert np.mean(r > TOL) <= 0.01, (name, key, np.mean(r > TOL))
    bad = np.argwhere(r > 1e-4)
    if bad.size:
        part = {"scatter_collimator": "collimator_variant", "scatter_crystal": "crystal"}.get(key, "collimator")
        bm = (bc if part == "crystal" else bh).cpu().numpy().view(np.uint32)
        pe_h = pe.cpu().numpy()
        for i, v in bad:
            d = int(z["rows"][i])
            ok = flip_explained(geo, pe_h, part, bm, d, int(v))
            if not ok and key == "scatter_combined":
                ok = flip_explained(geo, pe_h, "crystal", bc.cpu().numpy().view(np.uint32), d, int(v))
            assert ok, (name, key, d, v, r[i, v])


def test_scatter_vs_fp64_oracle_fresh_system(gpu):
    geo = geometry.mini(seed=21, rotated=True, nvox=(6, 6, 2), ncry=(5, 5))
    ctx = sysmat.Context(geo)
    pe = _pe(gpu, ctx, geo)
    bc, bh = ctx.bitmap_crystal(), ctx.bitmap_collimator()
    ctx.scatter_prepare(bc, bh)
    out = gpu.empty_like(pe)
    pe_h = pe.cpu().numpy()
    bch = bc.cpu().numpy().view(np.uint32)
    bhh = bh.cpu().numpy().view(np.uint32)
    for parts, part, bm in ((1, "crystal", bch), (2, "collimator", bhh)):
        ctx.scatter(out, pe, parts=parts)
        a = out.cpu().numpy()
        o64 = oracle.scatter(geo, pe_h, part, bm, prec=64)
        r = rel_err(a, o64)
        assert np.mean(r > TOL) <= 0.01
        for d, v in np.argwhere(r > 1e-4):
            assert flip_explained(geo, pe_h, part, bm, int(d), int(v))


def test_native_scatter_vs_fp64_oracle(gpu):
    """Native model (holes of every layer, their layer's mu, tungsten attenuation of the
    scattered photon) against the oracle's restatement, on a two-layer system."""
    geo = geometry.mini(seed=22, rotated=True, layers=2, nvox=(6, 6, 2), ncry=(5, 5))
    ctx = sysmat.Context(geo)
    pe = _pe(gpu, ctx, geo)
    bc = ctx.bitmap_crystal()
    out = gpu.empty_like(pe)
    ctx.scatter_prepare(bc, ctx.bitmap_collimator())
    ctx.scatter(out, pe, parts=1)
    crystal_ref = out.cpu().numpy()
    ctx.scatter_prepare_native(bc)
    with pytest.raises(sysmat.SysmatError):               # tables prepared for another model
        ctx.scatter(out, pe, parts=2)
    ctx.scatter(out, pe, parts=1, hole_model=sysmat.HOLE_MODEL_NATIVE)
    assert np.array_equal(out.cpu().numpy(), crystal_ref)  # the crystal part is the reference's
    ctx.scatter(out, pe, parts=2, hole_model=sysmat.HOLE_MODEL_NATIVE)
    a = out.cpu().numpy()
    pe_h = pe.cpu().numpy()
    bch = bc.cpu().numpy().view(np.uint32)
    o32 = oracle.scatter(geo, pe_h, "collimator_native", bch, prec=32)
    o64 = oracle.scatter(geo, pe_h, "collimator_native", bch, prec=64)
    assert a.max() > 0
    r = rel_err(a, o32)
    assert np.mean(r > TOL) <= 0.01
    for d, v in np.argwhere(r > 1e-4):
        assert flip_explained(geo, pe_h, "collimator_native", bch, int(d), int(v))
    # against FP64: the tungsten length is a plate chord minus nearly equal hole chords, so
    # float cancellation puts FP32 about 1e-5 (relative) from FP64
    r64 = rel_err(a, o64)
    assert np.median(r64) < 1e-5 and np.mean(r64 > 1e-4) <= 0.01


def test_scatter_block_decomposition_is_exact(gpu):
    geo, z, ctx, bc, bh, pe = _setup(gpu, "config3_z8")
    full = gpu.empty_like(pe)
    ctx.scatter(full, pe)
    full = full.cpu().numpy()
    for (d0, nd, v0, nv) in ((0, 3, 0, 300), (700, 20, 1111, 900)):
        out = gpu.empty((nd, nv), dtype=gpu.float32, device="cuda")
        ctx.scatter(out, pe, det_begin=d0, det_count=nd, vox_begin=v0, vox_count=nv)
        assert np.array_equal(out.cpu().numpy(), full[d0:d0 + nd, v0:v0 + nv])


def test_legacy_scatter_programs_and_bitmap_files(gpu):
    geo, z = golden("mini0")
    pe = np.ascontiguousarray(z["pe"]).reshape(-1)
    n = geo.n_det * geo.n_vox
    with tempfile.TemporaryDirectory() as tmp:
        fc, fh = os.path.join(tmp, "GeoCrystal"), os.path.join(tmp, "GeoCollimator")
        dst = np.zeros(n, np.float32)
        assert sysmat.scatter(geo.collimator, geo.detector, geo.image, geo.physics, pe, fc, fh, dst) == geo.n_vox
        assert np.array_equal(np.fromfile(fc, np.uint32), z["bitmap_crystal_words"])
        assert np.array_equal(np.fromfile(fh, np.uint32), z["bitmap_collimator_words"])
        phys = geo.physics.copy()
        phys[8] = phys[9] = 0                         # load the files instead of computing
        dst2 = np.zeros(n, np.float32)
        sysmat.scatter(geo.collimator, geo.detector, geo.image, phys, pe, fc, fh, dst2)
        assert np.array_equal(dst, dst2)
        assert rel_err(dst.reshape(geo.n_det, -1), z["scatter_combined"]).max() <= TOL
        dcol = np.zeros(n, np.float32)
        sysmat.scatter_collimator(geo.collimator, geo.detector, geo.image, phys, pe, fh, dcol)
        assert rel_err(dcol.reshape(geo.n_det, -1), z["scatter_collimator"]).max() <= TOL
        dcry = np.zeros(n, np.float32)
        sysmat.scatter_crystal(geo.detector, geo.image, phys, pe, fc, dcry)
        assert rel_err(dcry.reshape(geo.n_det, -1), z["scatter_crystal"]).max() <= TOL
        with pytest.raises(sysmat.SysmatError) as ei:
            sysmat.scatter(geo.collimator, geo.detector, geo.image, phys, pe,
                           os.path.join(tmp, "missing"), fh, dst2)
        assert ei.value.code == -4                        # SYSMAT_ERR_IO, not exit(0)


def test_legacy_scatter_reads_large_and_short_bitmap_files(gpu):
    """The file reader streams a bitmap through several reader threads and pinned pieces; a
    file of 200 MB of bitmaps must reproduce the computing call bit for bit, and a short file
    (cut inside a word) reads its missing words as 0, as the reference's zero-filled buffer
    does (scatter.cu:2156-2159)."""
    torch = gpu
    geo, z = golden("config3_z8")
    ctx = sysmat.Context(geo)
    pe_t = _pe(torch, ctx, geo)
    pe = pe_t.cpu().numpy().reshape(-1)
    n = geo.n_det * geo.n_vox
    with tempfile.TemporaryDirectory() as tmp:
        fc, fh = os.path.join(tmp, "GeoCrystal"), os.path.join(tmp, "GeoCollimator")
        dst = np.zeros(n, np.float32)
        sysmat.scatter(geo.collimator, geo.detector, geo.image, geo.physics, pe, fc, fh, dst)
        for f, key in ((fc, "crystal"), (fh, "collimator")):
            assert hashlib.sha256(np.fromfile(f, np.uint8).tobytes()).digest() == bytes(z[f"bitmap_{key}_sha256"])
        phys = geo.physics.copy()
        phys[8] = phys[9] = 0
        dst2 = np.zeros(n, np.float32)
        sysmat.scatter(geo.collimator, geo.detector, geo.image, phys, pe, fc, fh, dst2)
        assert np.array_equal(dst, dst2)
        words = np.fromfile(fh, np.uint32)
        keep = int(words.size * 0.6)
        with open(fh, "r+b") as f:
            f.truncate(4 * keep + 3)                      # a partial last word reads as 0 too
        short = np.zeros(n, np.float32)
        sysmat.scatter(geo.collimator, geo.detector, geo.image, phys, pe, fc, fh, short)
    cut = words.copy()
    cut[keep:] = 0
    ctx.scatter_prepare(ctx.bitmap_crystal(), torch.from_numpy(cut.view(np.int32)).cuda())
    exp = torch.empty((geo.n_det, geo.n_vox), dtype=torch.float32, device="cuda")
    ctx.scatter(exp, pe_t, rotation=float(geo.image[20]))
    assert np.array_equal(short, exp.cpu().numpy().reshape(-1))
    assert not np.array_equal(short, dst)


def test_scatter_argument_errors(gpu):
    geo, z = golden("mini0")
    ctx = sysmat.Context(geo)
    out = gpu.empty((geo.n_det, geo.n_vox), dtype=gpu.float32, device="cuda")
    pe = gpu.zeros_like(out)
    with pytest.raises(sysmat.SysmatError):
        ctx.scatter(out, pe)                              # not prepared
    with pytest.raises(sysmat.SysmatError):
        ctx.scatter_prepare(None, ctx.bitmap_collimator())  # crystal bitmap missing
    ctx.scatter_prepare(None, ctx.bitmap_collimator(), parts=sysmat.SCATTER_COLLIMATOR)
    with pytest.raises(sysmat.SysmatError):
        ctx.scatter(out, pe, parts=3)                     # crystal part not prepared
    ctx.scatter(out, None, parts=sysmat.SCATTER_COLLIMATOR)


def test_compton_flag_off_gives_zero(gpu):
    geo, z = golden("mini0")
    phys = geo.physics.copy()
    phys[0] = 0
    g = geometry.Geometry("nocompton", geo.collimator, geo.detector, geo.image, phys)
    ctx = sysmat.Context(g)
    pe = gpu.from_numpy(np.ascontiguousarray(z["pe"])).cuda()
    ctx.scatter_prepare(ctx.bitmap_crystal(), ctx.bitmap_collimator())
    out = gpu.full_like(pe, 7.0)
    ctx.scatter(out, pe)
    assert np.all(out.cpu().numpy() == 0.0)
