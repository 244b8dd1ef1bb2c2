"""GPU tests of the dense -> CSR conversion (entries > threshold, column order)."""
import numpy as np
import pytest

from conftest import golden, sysmat

pytestmark = pytest.mark.gpu


def _csr_numpy(a, thr, off=0):
    ptr, col, val = [0], [], []
    for row in a:
        idx = np.nonzero(row > thr)[0]
        col.extend((idx + off).tolist())
        val.extend(row[idx].tolist())
        ptr.append(len(col))
    return np.array(ptr), np.array(col, dtype=np.int64), np.array(val, dtype=np.float32)


@pytest.mark.parametrize("rows,cols", [(1, 1), (7, 33), (300, 1000), (2000, 37)])
def test_csr_matches_numpy(gpu, rows, cols):
    rng = np.random.default_rng(rows * 7 + cols)
    a = rng.random((rows, cols), dtype=np.float32)
    a[a < 0.6] = 0.0
    a[rng.random((rows, cols)) < 0.1] = 5e-10          # below the threshold
    t = gpu.from_numpy(a).cuda()
    ptr, col, val = sysmat.to_csr(t, 1e-9, col_offset=11)
    p2, c2, v2 = _csr_numpy(a, 1e-9, 11)
    assert np.array_equal(ptr.cpu().numpy(), p2)
    assert np.array_equal(col.cpu().numpy(), c2)
    assert np.array_equal(val.cpu().numpy(), v2)


def test_csr_of_a_strided_pe_block_rebuilds_the_dense_block(gpu):
    geo, _ = golden("config1")
    ctx = sysmat.Context(geo)
    out = gpu.zeros((64, 1024 + 5), dtype=gpu.float32, device="cuda")
    ctx.pe(out[:, :1000], det_begin=100, det_count=64, vox_begin=24, vox_count=1000)
    ptr, col, val = sysmat.to_csr(out[:, :1000], 1e-9, col_offset=24)
    dense = np.zeros((64, 1024), np.float32)
    p, c, v = ptr.cpu().numpy(), col.cpu().numpy(), val.cpu().numpy()
    for r in range(64):
        dense[r, c[p[r]:p[r + 1]]] = v[p[r]:p[r + 1]]
    ref = out[:, :1000].cpu().numpy()
    ref = np.where(ref > 1e-9, ref, 0.0)
    assert np.array_equal(dense[:, 24:1024], ref)
    assert p[-1] > 0
