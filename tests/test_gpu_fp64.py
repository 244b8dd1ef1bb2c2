"""GPU tests of the FP64 mode (SYSMAT_MODE_FP64), through the C ABI.

The FP64 mode evaluates the reference's element program in double from the float parameter
arrays, so its oracle is the FP64 restatement (oracle/oracle_body.h compiled with double):
the same program in the same precision, up to where each compiler fuses multiply-adds.
Elements agree to the float output's rounding, except knife-edge elements: in a regular
system some rays cross a threshold of the program exactly (a cap plane on a hole's rim),
where the last bit of any FP64 evaluation decides the branch; those are identified by
moving the image by 1e-9 mm.  Against the reference's own FP32 outputs (golden fixtures) it
differs by the reference's own rounding error, as the FP64 oracle does."""
import numpy as np
import pytest

from conftest import TOL, geometry, golden, oracle, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _fp64(torch, ctx, rotation=0.0, **blk):
    nd = blk.get("det_count", ctx.n_det)
    nv = blk.get("vox_count", ctx.n_vox)
    out = torch.empty((nd, nv), dtype=torch.float32, device="cuda")
    ctx.pe(out, rotation=rotation, mode=sysmat.MODE_FP64, **blk)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _knife_edge(geo, a, o64, outliers, h=1e-9):
    """Outlier elements whose device value lies within the range the FP64 oracle spans when
    the image moves by +-h mm along x, y or z (widened by 1e-7).  In a system this regular
    (configuration 1) many rays cross a hole's cap plane exactly on its rim or touch a box
    edge, and the reference's program is discontinuous there: which side an FP64 evaluation
    lands on depends on its last bit."""
    tau = 1e-6 * np.abs(o64).max()
    rows = np.unique(outliers[:, 0])
    vals = [o64[rows]]
    for k in (8, 9, 10):
        for sgn in (1.0, -1.0):
            img = geo.image.copy()
            img[k] = np.float32(img[k] + sgn * h)
            g = geometry.Geometry(geo.name, geo.collimator, geo.detector, img, geo.physics)
            vals.append(oracle.pe(g, prec=64, dets=rows))
    V = np.stack(vals)
    lo, hi = V.min(0), V.max(0)
    pos = {d: i for i, d in enumerate(rows)}
    explained = 0
    for d, v in outliers:
        m = 1e-7 * max(abs(o64[d, v]), tau)
        explained += lo[pos[d], v] - m <= a[d, v] <= hi[pos[d], v] + m
    return explained


@pytest.mark.parametrize("name", ["mini0", "mini1r2", "mini2w", "config1"])
def test_fp64_mode_matches_fp64_oracle(gpu, name):
    geo, z = golden(name)
    ctx = sysmat.Context(geo)
    a = _fp64(gpu, ctx, rotation=float(geo.image[20]))
    o64 = oracle.pe(geo, prec=64)
    r = rel_err(a, o64)
    assert a.max() > 0
    assert np.median(r) < 1e-7, np.median(r)
    # float32 output of a double value: at most half an ulp (6e-8) from it when the programs
    # agree; anything further must be a knife-edge element
    outliers = np.argwhere(r > 1e-7)
    assert len(outliers) <= 0.01 * r.size, len(outliers)
    if len(outliers):
        assert _knife_edge(geo, a, o64, outliers) == len(outliers)
    # the reference's FP32 program is further from FP64 than the FP64 mode is
    ref = z["pe"].astype(np.float64)
    assert np.abs(a[z["rows"]] - o64[z["rows"]]).sum() < np.abs(ref - o64[z["rows"]]).sum()


@pytest.mark.parametrize("seed", [14, 15])
def test_fp64_mode_on_fresh_seeded_systems(gpu, seed):
    g = geometry.mini(seed=seed, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4)).with_rotation(seed % 8)
    ctx = sysmat.Context(g)
    a = _fp64(gpu, ctx, rotation=float(seed % 8))
    r = rel_err(a, oracle.pe(g, prec=64))
    assert np.median(r) < 1e-7 and np.mean(r > TOL) < 1e-3, (np.median(r), np.mean(r > TOL), r.max())


def test_fp64_mode_config2_full_size_sample(gpu):
    """Configuration 2 at full size: 6 crystals x 2 voxel rows of z-plane 16 against FP64."""
    torch = gpu
    geo = geometry.config2()
    ctx = sysmat.Context(geo)
    rows = np.sort(np.random.default_rng(5).choice(geo.n_det, 6, replace=False))
    v0, nv = 96 * 96 * 16 + 96 * 40, 96 * 2
    out = torch.empty((len(rows), nv), dtype=torch.float32, device="cuda")
    for i, d in enumerate(rows):
        ctx.pe(out[i:i + 1], det_begin=int(d), det_count=1, vox_begin=v0, vox_count=nv, mode=sysmat.MODE_FP64)
    a = out.cpu().numpy()
    o64 = oracle.pe(geo, prec=64, dets=rows, v0=v0, nv=nv)
    o32 = oracle.pe(geo, prec=32, dets=rows, v0=v0, nv=nv)
    r, r32 = rel_err(a, o64), rel_err(o32, o64)
    assert a.max() > 0
    assert np.median(r) < 1e-7 and r.max() <= TOL, (np.median(r), r.max())
    assert r.max() < r32.max()                          # the float program's own error is larger


def test_fp64_blocks_equal_the_full_matrix(gpu):
    torch = gpu
    geo, _ = golden("mini1r2")
    ctx = sysmat.Context(geo)
    rot = float(geo.image[20])
    full = _fp64(torch, ctx, rotation=rot)
    for (d0, nd, v0, nv) in ((0, 3, 0, 17), (7, 5, 31, 40), (ctx.n_det - 1, 1, ctx.n_vox - 1, 1)):
        out = torch.full((nd, nv + 5), -1.0, dtype=torch.float32, device="cuda")
        ctx.pe(out[:, :nv], rotation=rot, det_begin=d0, det_count=nd, vox_begin=v0, vox_count=nv,
               mode=sysmat.MODE_FP64)
        blk = out.cpu().numpy()
        assert np.array_equal(blk[:, :nv], full[d0:d0 + nd, v0:v0 + nv])
        assert np.all(blk[:, nv:] == -1.0)


def _elliptical(seed):
    geo = geometry.mini(seed=seed, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))
    H = geo.n_holes
    rng = np.random.default_rng(seed)
    r = geo.collimator[100:100 + 9 * H].reshape(H, 9)[:, 4].astype(np.float64)
    shapes = np.stack([r * rng.uniform(0.5, 1.0, H), r * rng.uniform(0.5, 1.0, H),
                       rng.uniform(0.0, np.pi, H)], 1).astype(np.float32)
    shapes[rng.random(H) < 0.2, 0] = 0.0                 # some holes stay circular
    return geo, shapes


def test_fp64_mode_with_elliptical_holes(gpu):
    """The elliptical chord in double against the FP64 restatement of the reference's
    length_ellipticalcylinder_ray: the float chord's ill-conditioning is gone."""
    torch = gpu
    geo, shapes = _elliptical(18)
    geo = geo.with_rotation(2)
    ctx = sysmat.Context(geo)
    ctx.set_hole_shapes(shapes)
    a = _fp64(torch, ctx, rotation=2.0)
    r = rel_err(a, oracle.pe(geo, prec=64, shapes=shapes))
    assert a.max() > 0
    assert np.median(r) < 1e-7 and np.mean(r > 1e-7) < 1e-3 and r.max() < TOL, (np.median(r), r.max())
    ctx.set_hole_shapes(None)                            # back to circles
    b = _fp64(torch, ctx, rotation=2.0)
    assert not np.array_equal(a, b)
    assert rel_err(b, oracle.pe(geo, prec=64)).max() < TOL


def test_fp64_batched_launch_equals_single_calls(gpu):
    """A batch of a circular system, configuration 1 and an elliptical system in FP64."""
    torch = gpu
    geo_e, shapes = _elliptical(19)
    ctxs = [sysmat.Context(geometry.mini(seed=17, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))),
            sysmat.Context(geometry.config1()), sysmat.Context(geo_e)]
    ctxs[2].set_hole_shapes(shapes)
    tasks = [(0, 3.0, 0, ctxs[0].n_det, 0, ctxs[0].n_vox), (1, 0.0, 100, 9, 37, 300), (0, 6.0, 4, 3, 11, 70),
             (2, 5.0, 0, ctxs[2].n_det, 0, ctxs[2].n_vox)]
    exp = []
    for (c, rot, d0, nd, v0, nv) in tasks:
        exp.append(_fp64(torch, ctxs[c], rotation=rot, det_begin=d0, det_count=nd, vox_begin=v0, vox_count=nv))
    outs = [torch.full((t[3], t[5]), -1.0, dtype=torch.float32, device="cuda") for t in tasks]
    plan = sysmat.BatchPlan(ctxs, [t + (o,) for t, o in zip(tasks, outs)])
    for _ in range(2):                                      # graph capture, then replay
        plan.run(mode=sysmat.MODE_FP64)
        torch.cuda.synchronize()
        for o, e in zip(outs, exp):
            assert np.array_equal(o.cpu().numpy(), e)
    plan.close()
