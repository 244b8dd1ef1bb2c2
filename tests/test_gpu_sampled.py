"""GPU tests of the sampled photoelectric form (sysmat_pe_sampled), through the C ABI.

The reference fixes 8 x 16 x 8 crystal sub-elements and one source point, the voxel centre.
The sampled form takes both as parameters: the crystal divisions of the configurations
(4 x 4 x 4; 2 x 2 x 8 in depth), the 2 x 2 x 2 voxel sub-samples, and ragged sizes whose
sub-element count is not a multiple of the warp.  There is no reference output for it, so
it is checked against the oracle's restatement with the same parameters: the FP32 twin (the
same float program per sub-element; the device sums in FP64, the twin in float) and FP64,
against which the device must be as close as the twin is."""
import numpy as np
import pytest

from conftest import TOL, geometry, oracle, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _sampled(torch, ctx, div, sub, rotation=0.0, **blk):
    nd = blk.get("det_count", ctx.n_det)
    nv = blk.get("vox_count", ctx.n_vox)
    out = torch.empty((nd, nv), dtype=torch.float32, device="cuda")
    ctx.pe_sampled(out, div, sub, rotation=rotation, **blk)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _mini_rot():
    return geometry.mini(seed=61, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))


@pytest.mark.parametrize("case", ["config1", "mini_rot"])
def test_reference_sampling_equals_precise_mode(gpu, case):
    """8 x 16 x 8 with one source point: the float program of SYSMAT_MODE_PRECISE, summed in
    FP64 in another order.  The two kernel instances are compiled separately, so the compiler
    may contract a sub-element's position expressions differently (a last-bit change of a
    ray end point); measured: a few ulps on heavily attenuated elements."""
    torch = gpu
    geo = geometry.config1() if case == "config1" else _mini_rot()
    rot = 0.0 if case == "config1" else 3.0
    ctx = sysmat.Context(geo)
    ref = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(ref, rotation=rot, mode=sysmat.MODE_PRECISE)
    b = ref.cpu().numpy()
    a = _sampled(torch, ctx, (8, 16, 8), (1, 1, 1), rotation=rot)
    r = rel_err(a, b)
    assert np.median(r) < 1e-7 and r.max() < 1e-4, (np.median(r), r.max())   # measured max 1.5e-5


CASES = {
    # name: (geometry, rotation, crystal division, voxel sub-samples)
    "config1_4x4x4": (geometry.config1, 0.0, (4, 4, 4), (1, 1, 1)),
    "config2_sampling": (_mini_rot, 5.0, (2, 8, 2), (2, 2, 2)),
    "ragged_30x6": (_mini_rot, 1.0, (3, 5, 2), (3, 1, 2)),
    "ragged_35x2": (_mini_rot, 6.0, (5, 7, 1), (1, 2, 1)),
    "single_ray": (_mini_rot, 2.0, (1, 1, 1), (1, 1, 1)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_sampled_matches_oracle(gpu, name):
    make, rot, div, sub = CASES[name]
    geo = make().with_rotation(int(rot))
    ctx = sysmat.Context(geo)
    a = _sampled(gpu, ctx, div, sub, rotation=rot)
    o32 = oracle.pe_sampled(geo, div, sub, prec=32)
    o64 = oracle.pe_sampled(geo, div, sub, prec=64)
    assert a.max() > 0
    r = rel_err(a, o32)
    assert np.median(r) < 1e-6, np.median(r)
    assert np.mean(r > 3e-5) <= 0.005, np.mean(r > 3e-5)
    assert r.max() < 1e-3, r.max()
    # against FP64 the device is as close as the reference's float arithmetic allows: its
    # own error (the FP32 twin's) is 1.5-4 % of elements above 1e-5 on these coarse samplings,
    # which average fewer sub-elements than 8 x 16 x 8
    r64, rt = rel_err(a, o64), rel_err(o32, o64)
    assert np.median(r64) < 1e-6, np.median(r64)
    assert np.mean(r64 > TOL) <= np.mean(rt > TOL) + 0.02, (np.mean(r64 > TOL), np.mean(rt > TOL))
    assert r64.max() < 10 * max(rt.max(), TOL), (r64.max(), rt.max())


def test_config2_stated_sampling_full_size_sample(gpu):
    """Configuration 2 as stated (2 x 2 x 2 voxel sub-samples, crystals 2 x 8 x 2 with 8 in
    depth) on a sample: 4 crystals x 2 voxel rows of z-plane 16."""
    torch = gpu
    geo = geometry.config2()
    ctx = sysmat.Context(geo)
    rows = np.sort(np.random.default_rng(9).choice(geo.n_det, 4, replace=False))
    v0, nv = 96 * 96 * 16 + 96 * 47, 96 * 2
    out = torch.empty((len(rows), nv), dtype=torch.float32, device="cuda")
    for i, d in enumerate(rows):
        ctx.pe_sampled(out[i:i + 1], (2, 8, 2), (2, 2, 2), det_begin=int(d), det_count=1, vox_begin=v0,
                       vox_count=nv)
    a = out.cpu().numpy()
    o32 = oracle.pe_sampled(geo, (2, 8, 2), (2, 2, 2), prec=32, dets=rows, v0=v0, nv=nv)
    r = rel_err(a, o32)
    assert a.max() > 0
    assert np.median(r) < 1e-6 and r.max() < 1e-4, (np.median(r), r.max())


def test_sampled_blocks_equal_the_full_matrix(gpu):
    torch = gpu
    geo = _mini_rot()
    ctx = sysmat.Context(geo)
    full = _sampled(torch, ctx, (3, 5, 2), (2, 1, 2), rotation=4.0)
    for (d0, nd, v0, nv) in ((0, 3, 0, 17), (7, 5, 31, 40), (19, 1, 89, 1)):
        out = torch.full((nd, nv + 5), -1.0, dtype=torch.float32, device="cuda")
        ctx.pe_sampled(out[:, :nv], (3, 5, 2), (2, 1, 2), rotation=4.0, det_begin=d0, det_count=nd, vox_begin=v0,
                       vox_count=nv)
        blk = out.cpu().numpy()
        assert np.array_equal(blk[:, :nv], full[d0:d0 + nd, v0:v0 + nv])
        assert np.all(blk[:, nv:] == -1.0)


def test_sampled_elliptical_holes(gpu):
    geo = _mini_rot().with_rotation(2)
    H = geo.n_holes
    rng = np.random.default_rng(62)
    r = geo.collimator[100:100 + 9 * H].reshape(H, 9)[:, 4].astype(np.float64)
    shapes = np.stack([r * rng.uniform(0.5, 1.0, H), r * rng.uniform(0.5, 1.0, H),
                       rng.uniform(0.0, np.pi, H)], 1).astype(np.float32)
    ctx = sysmat.Context(geo)
    ctx.set_hole_shapes(shapes)
    a = _sampled(gpu, ctx, (4, 4, 4), (2, 1, 2), rotation=2.0)
    ref = oracle.pe_sampled(geo, (4, 4, 4), (2, 1, 2), prec=32, shapes=shapes)
    r = rel_err(a, ref)
    # the float elliptical chord's conditioning bounds this (test_gpu_ellipse.py)
    assert np.median(r) < 1e-6 and r.max() < 1e-3, (np.median(r), r.max())


def test_invalid_sampling_raises(gpu):
    torch = gpu
    geo = geometry.mini(seed=63)
    ctx = sysmat.Context(geo)
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    for div, sub in (((0, 4, 4), (1, 1, 1)), ((65, 1, 1), (1, 1, 1)), ((32, 32, 8), (1, 1, 1)),
                     ((4, 4, 4), (0, 1, 1)), ((4, 4, 4), (9, 1, 1)), ((4, 4, 4), (4, 4, 8))):
        with pytest.raises(sysmat.SysmatError):
            ctx.pe_sampled(out, div, sub)
    with pytest.raises(sysmat.SysmatError):
        ctx.pe_sampled(out, (4, 4, 4), (1, 1, 1), det_begin=ctx.n_det - 1, det_count=2)
    ctx.pe_sampled(out, (4, 4, 4), (1, 1, 1), det_count=0)          # empty block: no-op
