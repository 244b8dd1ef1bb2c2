"""GPU test of the photoelectric kernel at the capacities the reference's parameter arrays
allow (6666 crystals, 9 layers; 8649 of at most 8877 holes), through the C ABI.

Large voxels make the bricks' cone supersets exceed their 1024 shared-memory slots, so the
kernel's fallback (every object scanned for each kept-list chunk) runs, as the work
counters confirm; dense holes and crystals make kept lists span several chunks.  The
elements are compared with the oracle's FP32 twin on a row sample."""
import numpy as np
import pytest

from conftest import geometry, oracle, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _max_system():
    cb = geometry._CollimatorBuilder()
    holes = [((i - 15) * 0.6, (j - 15) * 0.6, 0.2) for j in range(31) for i in range(31)]
    for m in range(9):                                     # 9 x 961 = 8649 holes
        cb.add_layer(120.0, 1.0, 120.0, 1.2 * m, geometry.MU_W_TOTAL, geometry.MU_W_TOTAL * 0.87,
                     geometry.MU_W_TOTAL * 0.13, holes)
    crystals = [((i - 50) * 1.0, 15.0, (j - 32.5) * 1.0) for j in range(66) for i in range(101)]   # 6666
    det = geometry._detector(crystals, (1.0, 5.0, 1.0))
    img = geometry._image((8, 8, 2), (5.0, 5.0, 5.0), 45.0)
    return geometry.Geometry("capacity", cb.build(), det, img, geometry._physics())


def test_capacity_system_matches_oracle_and_overflows_the_superset(gpu):
    torch = gpu
    geo = _max_system()
    assert geo.n_det == 6666 and geo.n_holes == 8649 and geo.n_layers == 9
    ctx = sysmat.Context(geo)
    rows = [0, 3282, 3382, 3383, 3484, 6665]              # a corner, the centre, the far corner
    out = torch.empty((1, ctx.n_vox), dtype=torch.float32, device="cuda")
    got = []
    overflow = 0
    for d in rows:
        counts = ctx.pe_work(out, det_begin=d, det_count=1)
        overflow += counts["superset_overflow"]
        got.append(out.cpu().numpy()[0].copy())
    a = np.array(got)
    o32 = oracle.pe(geo, prec=32, dets=rows)
    r = rel_err(a, o32)
    assert overflow > 0                                    # the all-objects fallback ran
    assert a.max() > 0
    assert np.median(r) < 1e-6 and r.max() < 1e-3, (np.median(r), r.max())
