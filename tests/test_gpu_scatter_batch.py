"""GPU tests of batched scatter launches (sysmat_scatter_batch_*), through the C ABI: every
element of a batch equals the per-task sysmat_scatter element bit for bit, for mixed systems,
parts, hole models, rotations and ragged blocks, on the first (captured) run and on replays."""
import numpy as np
import pytest

from conftest import geometry, golden, sysmat

pytestmark = pytest.mark.gpu


def _prepared(torch, geo, native=False):
    ctx = sysmat.Context(geo)
    pe = {}
    for r in range(int(geo.n_rot)):
        out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
        ctx.pe(out, rotation=float(r))
        pe[r] = out
    if native:
        ctx.scatter_prepare_native(ctx.bitmap_crystal())
    else:
        ctx.scatter_prepare(ctx.bitmap_crystal(), ctx.bitmap_collimator())
    return ctx, pe


def test_scatter_batch_equals_per_task_calls(gpu):
    torch = gpu
    g0, _ = golden("mini0")
    g1 = geometry.mini(seed=31, rotated=True, layers=2, n_rot=4, nvox=(6, 5, 3), ncry=(5, 4))
    g2 = geometry.mini(seed=32, rotated=True, n_rot=2, nvox=(5, 4, 2), ncry=(4, 4))
    (c0, pe0), (c1, pe1), (c2, pe2) = _prepared(torch, g0), _prepared(torch, g1), _prepared(torch, g2, native=True)
    ctxs = [c0, c1, c2]
    pes = [pe0, pe1, pe2]
    H = sysmat.HOLE_MODEL_COMBINED
    tasks = [  # (ctx, parts, model, rotation, det_begin, det_count, vox_begin, vox_count)
        (0, 3, H, 0.0, 0, c0.n_det, 0, c0.n_vox),
        (1, 1, H, 2.0, 3, 7, 5, 61),
        (1, 2, sysmat.HOLE_MODEL_VARIANT, 1.0, 0, c1.n_det, 0, c1.n_vox),
        (1, 3, H, 3.0, c1.n_det - 1, 1, c1.n_vox - 1, 1),
        (2, 3, sysmat.HOLE_MODEL_NATIVE, 1.0, 2, 9, 0, c2.n_vox),
        (0, 2, H, 0.0, 5, 3, 40, 70),
    ]
    expected, outs, items = [], [], []
    for (c, parts, model, rot, d0, nd, v0, nv) in tasks:
        pe = pes[c][int(rot)] if parts & 1 else None
        e = torch.full((nd, nv), -1.0, dtype=torch.float32, device="cuda")
        ctxs[c].scatter(e, pe, parts=parts, hole_model=model, rotation=rot, det_begin=d0, det_count=nd,
                        vox_begin=v0, vox_count=nv)
        expected.append(e.cpu().numpy())
        o = torch.full((nd, nv + 3), -2.0, dtype=torch.float32, device="cuda")
        outs.append(o)
        items.append((c, parts, model, rot, pe, d0, nd, v0, nv, o[:, :nv]))
    torch.cuda.synchronize()
    assert any(np.abs(e).max() > 0 for e in expected)
    plan = sysmat.ScatterBatchPlan(ctxs, items)
    for _ in range(3):                                  # capture, then replays
        for o in outs:
            o[:, : o.shape[1] - 3].fill_(-3.0)
        plan.run()
        torch.cuda.synchronize()
        for o, e in zip(outs, expected):
            h = o.cpu().numpy()
            assert np.array_equal(h[:, :-3], e)
            assert np.all(h[:, -3:] == -2.0)            # nothing written past a block
    plan.close()


def test_scatter_batch_rejects_unprepared_parts(gpu):
    torch = gpu
    g0, _ = golden("mini0")
    ctx = sysmat.Context(g0)
    ctx.scatter_prepare(None, ctx.bitmap_collimator(), parts=sysmat.SCATTER_COLLIMATOR)
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    pe = torch.zeros_like(out)
    with pytest.raises(sysmat.SysmatError):
        sysmat.ScatterBatchPlan([ctx], [(0, 3, sysmat.HOLE_MODEL_COMBINED, 0.0, pe, 0, ctx.n_det, 0, ctx.n_vox, out)])
