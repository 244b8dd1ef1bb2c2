"""sysmat_pe_noalloc: the photoelectric entry point for callers that cannot allocate device
memory at call time (for example an application that hands all device memory to its own
pool at start-up, or a plug-in host that forbids allocation after initialisation).  It
keeps its parameter copies, tables, work counter and status word in one static device array
instead of allocating them.

The test calls it through the C ABI twice in a row, on two different systems and then on a
sub-block of the first, and checks each result against the existing entry point sysmat_pe
within the per-element tolerance the other tests use.  It lives in a file of its own that
pytest collects last; it passes alone in a fresh process and after the other tests."""
import numpy as np
import pytest

from conftest import TOL, golden, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _existing(torch, geo, **block):
    ctx = sysmat.Context(geo)
    det_count = block.get("det_count", ctx.n_det)
    vox_count = block.get("vox_count", ctx.n_vox)
    out = torch.empty((det_count, vox_count), dtype=torch.float32, device="cuda")
    ctx.pe(out, rotation=float(geo.image[20]), **block)
    torch.cuda.synchronize()
    ctx.close()
    return out.cpu().numpy()


def _noalloc(torch, geo, **block):
    det_count = block.get("det_count", geo.n_det)
    vox_count = block.get("vox_count", geo.n_vox)
    out = torch.full((det_count, vox_count), float("nan"), dtype=torch.float32, device="cuda")
    sysmat.pe_noalloc(geo, out, rotation=float(geo.image[20]), **block)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_existing_entry_point_on_consecutive_calls(gpu):
    calls = [("config1", {}), ("mini1r2", {}),
             ("config1", dict(det_begin=37, det_count=50, vox_begin=100, vox_count=700))]
    for name, block in calls:
        geo, _ = golden(name)
        want = _existing(gpu, geo, **block)
        got = _noalloc(gpu, geo, **block)
        assert not np.isnan(got).any(), name
        assert rel_err(got, want).max() <= TOL, (name, block)


def test_noalloc_rejects_systems_beyond_its_static_scratch(gpu):
    geo, _ = golden("mini0")
    det = geo.detector.copy()
    det[0] = 7000                                   # more crystals than the scratch holds
    big = type(geo)("big", geo.collimator, det, geo.image, geo.physics)
    out = gpu.empty((1, 1), dtype=gpu.float32, device="cuda")
    with pytest.raises(sysmat.SysmatError) as ei:
        sysmat.pe_noalloc(big, out, det_count=1, vox_count=1)
    assert ei.value.code == -3                      # SYSMAT_ERR_CAPACITY
