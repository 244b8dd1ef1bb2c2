"""GPU tests of batched photoelectric launches (sysmat_batch_*), through the C ABI.

A batch computes each element exactly as a single-system sysmat_pe call does, so every test
compares bit for bit with per-task sysmat_pe blocks, over mixed systems, rotations, blocks,
brick shapes, graph replays and the autotuner."""
import numpy as np
import pytest

from conftest import check_pe_vs_reference, geometry, golden, sysmat

pytestmark = pytest.mark.gpu


def _systems():
    return [geometry.mini(seed=21, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4)),
            geometry.mini(seed=22, layers=1, n_rot=4, nvox=(7, 4, 2), ncry=(4, 4)),
            geometry.config1()]


def _tasks(ctxs):
    """(ctx, rotation, det_begin, det_count, vox_begin, vox_count) blocks, ragged on purpose."""
    return [(0, 0.0, 0, ctxs[0].n_det, 0, ctxs[0].n_vox),
            (0, 3.0, 2, 7, 11, 61),                 # crosses z-planes, partial rows
            (1, 1.0, 0, ctxs[1].n_det, 5, 40),
            (1, 2.0, 15, 1, 0, ctxs[1].n_vox),      # one detector row
            (2, 0.0, 100, 30, 0, ctxs[2].n_vox),
            (0, 5.0, 19, 1, 89, 1)]                 # one element


def _alloc(torch, tasks, pad=5):
    return [torch.full((nd, nv + pad), -1.0, dtype=torch.float32, device="cuda")
            for (_, _, _, nd, _, nv) in tasks]


def _expected(torch, ctxs, tasks, mode=sysmat.MODE_REFERENCE):
    out = []
    for (c, rot, d0, nd, v0, nv) in tasks:
        t = torch.empty((nd, nv), dtype=torch.float32, device="cuda")
        ctxs[c].pe(t, rotation=rot, det_begin=d0, det_count=nd, vox_begin=v0, vox_count=nv, mode=mode)
        out.append(t.cpu().numpy())
    return out


def _check(outs, exp, tasks):
    for o, e, (_, _, _, nd, _, nv) in zip(outs, exp, tasks):
        a = o.cpu().numpy()
        assert np.array_equal(a[:, :nv], e)
        assert np.all(a[:, nv:] == -1.0)                  # nothing written past the block


@pytest.mark.parametrize("tiles", [(4, 4, 2, 0), (8, 4, 1, 0), (2, 2, 2, 1), (3, 5, 1, 0)])
def test_batch_equals_single_system_calls(gpu, tiles):
    torch = gpu
    ctxs = [sysmat.Context(g) for g in _systems()]
    tasks = _tasks(ctxs)
    exp = _expected(torch, ctxs, tasks)
    outs = _alloc(torch, tasks)
    plan = sysmat.BatchPlan(ctxs, [t + (o[:, :t[5]],) for t, o in zip(tasks, outs)])
    plan.set_tiles(*tiles)
    assert plan.tiles() == tiles
    for _ in range(2):                                    # graph capture, then replay
        plan.run()
        torch.cuda.synchronize()
        _check(outs, exp, tasks)
        for o in outs:
            o.fill_(-1.0)
    plan.close()


def test_batch_precise_mode_and_one_shot(gpu):
    torch = gpu
    ctxs = [sysmat.Context(g) for g in _systems()]
    tasks = _tasks(ctxs)
    exp = _expected(torch, ctxs, tasks, mode=sysmat.MODE_PRECISE)
    outs = _alloc(torch, tasks)
    sysmat.batch(ctxs, [t + (o[:, :t[5]],) for t, o in zip(tasks, outs)], mode=sysmat.MODE_PRECISE)
    _check(outs, exp, tasks)


def test_autotuner_picks_a_candidate_and_keeps_results(gpu):
    torch = gpu
    ctxs = [sysmat.Context(g) for g in _systems()]
    tasks = _tasks(ctxs)
    exp = _expected(torch, ctxs, tasks)
    outs = _alloc(torch, tasks)
    plan = sysmat.BatchPlan(ctxs, [t + (o[:, :t[5]],) for t, o in zip(tasks, outs)])
    tiles = plan.tune()
    assert tiles[:3] in {(4, 4, 2), (4, 4, 1), (8, 4, 1), (4, 2, 2), (2, 2, 2), (8, 8, 1), (4, 4, 4)}
    assert plan.tiles() == tiles
    plan.run()
    torch.cuda.synchronize()
    _check(outs, exp, tasks)


def test_config4_instances_sample(gpu):
    """Several designs of the batched sweep, two rotations each, a crystal row x one z-plane."""
    torch = gpu
    geos = geometry.config4(n_instances=4, seed=4)
    ctxs = [sysmat.Context(g) for g in geos]
    tasks = [(k, float(r), 32 * 13, 32, 1024 * 7, 1024) for k in range(4) for r in (0, geos[k].n_rot // 3)]
    exp = _expected(torch, ctxs, tasks)
    outs = _alloc(torch, tasks)
    plan = sysmat.BatchPlan(ctxs, [t + (o[:, :t[5]],) for t, o in zip(tasks, outs)])
    plan.run()
    torch.cuda.synchronize()
    _check(outs, exp, tasks)
    assert all(e.max() > 0 for e in exp)


@pytest.mark.parametrize("mode", [sysmat.MODE_LOCAL, sysmat.MODE_FP64])
def test_batch_precision_modes_equal_single_calls(gpu, mode):
    """The FP64 and local FP32 forms in a batch, a system with elliptical holes among them:
    every element equals the per-task sysmat_pe element in the same mode bit for bit."""
    torch = gpu
    systems = _systems()
    ell = geometry.mini(seed=57, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))
    H = ell.n_holes
    r = ell.collimator[100:100 + 9 * H].reshape(H, 9)[:, 4]
    shapes = np.stack([0.8 * r, 0.6 * r, np.linspace(0.1, 3.0, H)], 1).astype(np.float32)
    ctxs = [sysmat.Context(g) for g in systems[:2]] + [sysmat.Context(ell)]
    ctxs[2].set_hole_shapes(shapes)
    tasks = [(0, 3.0, 2, 7, 11, 61), (1, 1.0, 0, ctxs[1].n_det, 5, 40), (2, 5.0, 0, ctxs[2].n_det, 0, ctxs[2].n_vox),
             (2, 2.0, 19, 1, 89, 1)]
    exp = _expected(torch, ctxs, tasks, mode=mode)
    outs = _alloc(torch, tasks)
    plan = sysmat.BatchPlan(ctxs, [t + (o[:, :t[5]],) for t, o in zip(tasks, outs)])
    for _ in range(2):                                  # captured run, then a replay
        plan.run(mode=mode)
        torch.cuda.synchronize()
        _check(outs, exp, tasks)
    assert all(e.max() > 0 for e in exp)


def test_batch_matches_reference_on_config4_goldens(gpu):
    """Two configuration-4 designs at one of their rotations (the reference's own PESysMatGen
    output on voxel row 16 of z-plane 8), computed together in one batch."""
    torch = gpu
    pairs = [golden(n) for n in ("config4_i7r5", "config4_i40r11")]
    ctxs = [sysmat.Context(geo) for geo, _ in pairs]
    outs = [torch.empty((c.n_det, c.n_vox), dtype=torch.float32, device="cuda") for c in ctxs]
    items = [(k, float(geo.image[20]), 0, ctxs[k].n_det, 0, ctxs[k].n_vox, outs[k])
             for k, (geo, _) in enumerate(pairs)]
    plan = sysmat.BatchPlan(ctxs, items)
    plan.run()
    torch.cuda.synchronize()
    for o, (geo, z) in zip(outs, pairs):
        check_pe_vs_reference(o.cpu().numpy()[z["rows"]], geo, z)


def test_invalid_batches_raise(gpu):
    torch = gpu
    ctxs = [sysmat.Context(g) for g in _systems()[:2]]
    out = torch.empty((4, 200), dtype=torch.float32, device="cuda")
    with pytest.raises(sysmat.SysmatError):
        sysmat.BatchPlan(ctxs, [(2, 0.0, 0, 4, 0, 10, out)])                 # no context 2
    with pytest.raises(sysmat.SysmatError):
        sysmat.BatchPlan(ctxs, [(0, 0.0, ctxs[0].n_det - 1, 4, 0, 10, out)])  # rows past the end
    with pytest.raises(sysmat.SysmatError):
        sysmat.BatchPlan(ctxs, [(1, 0.0, 0, 1, 0, ctxs[1].n_vox + 1, out)])   # voxels past the end
    plan = sysmat.BatchPlan(ctxs, [(0, 0.0, 0, 0, 0, 10, out)])               # empty batch: no-op
    plan.run()
    with pytest.raises(sysmat.SysmatError):
        plan.set_tiles(0, 4, 4)
    for mode in (4, -1):                                                      # no such mode
        with pytest.raises(sysmat.SysmatError):
            plan.run(mode=mode)
