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


@pytest.mark.parametrize("rows_per_block,threshold", [(7, 1e-9), (0, 1e-9), (100, 0.0)])
def test_pe_csr_file_rebuilds_the_thresholded_matrix(gpu, tmp_path, rows_per_block, threshold):
    """The whole matrix of a rotation streamed to a compressed file, block by block, reads back
    as the dense matrix with entries <= threshold dropped."""
    geo, _ = golden("config1")
    ctx = sysmat.Context(geo)
    dense = gpu.empty((ctx.n_det, ctx.n_vox), dtype=gpu.float32, device="cuda")
    ctx.pe(dense)
    a = dense.cpu().numpy()
    path = tmp_path / "pe.smcsr"
    nnz = ctx.pe_csr_file(str(path), threshold=threshold, rows_per_block=rows_per_block)
    rows, cols, thr, mode, ptr, col, val = sysmat.read_csr_file(str(path))
    assert (rows, cols, mode) == (ctx.n_det, ctx.n_vox, sysmat.MODE_REFERENCE)
    assert thr == np.float32(threshold) and nnz == len(val) == ptr[-1] == int((a > threshold).sum())
    back = np.zeros_like(a)
    for r in range(rows):
        back[r, col[ptr[r]:ptr[r + 1]]] = val[ptr[r]:ptr[r + 1]]
    assert np.array_equal(back, np.where(a > threshold, a, 0.0))


def test_pe_csr_file_errors(gpu, tmp_path):
    geo, _ = golden("mini0")
    ctx = sysmat.Context(geo)
    with pytest.raises(sysmat.SysmatError):
        ctx.pe_csr_file(str(tmp_path / "no_such_dir" / "x.smcsr"))
    with pytest.raises(sysmat.SysmatError):
        ctx.pe_csr_file(str(tmp_path / "x.smcsr"), threshold=-1.0)
