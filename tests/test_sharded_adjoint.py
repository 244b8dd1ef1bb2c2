"""CPU tests of the multi-rank projector (adjoint.ShardedProjector) over gloo, world_size 2.

Each rank owns a slab of detector rows; back projections and the theta gradient are summed
across ranks with one all-reduce each.  The rank-local projector here is a dense stand-in
(rows of a seeded matrix A and of seven derivative matrices dA/dtheta_i), so the test covers
the partition, the reductions, MLEM and the autograd path without a GPU: the sharded results
must equal the single-process ones."""
import os
import socket
import types

import numpy as np

from conftest import PKG_DIR, _load

D, V, THETA_N = 7, 11, 7            # 7 rows over 2 ranks: uneven slabs (4 + 3)


class DenseRows:
    """Rows det_begin .. det_begin + det_count of a dense A (float64, CPU tensors)."""

    def __init__(self, A, dA, det_begin, det_count):
        import torch
        self.A = torch.from_numpy(A[det_begin:det_begin + det_count])
        self.dA = torch.from_numpy(dA[:, det_begin:det_begin + det_count])
        self.det_begin, self.det_count = det_begin, det_count
        self.geo = types.SimpleNamespace(n_det=A.shape[0], n_vox=A.shape[1])

    def project(self, x, theta=None):
        return self.A @ x.double()

    def backproject(self, u, theta=None):
        return self.A.T @ u.double()

    def vjp(self, x, u, theta=None):
        import torch
        u, x = u.double(), x.double()
        g = [u @ (self.dA[i] @ x) for i in range(THETA_N)] + [u @ (self.A @ x)]
        return torch.stack(g)


def _system():
    rng = np.random.default_rng(17)
    A = rng.uniform(0.0, 1.0, (D, V))
    A[rng.random((D, V)) < 0.3] = 0.0
    dA = rng.normal(size=(THETA_N, D, V))
    x = rng.uniform(0.5, 2.0, V).astype(np.float32)
    y = rng.poisson(A @ x * 50.0).astype(np.float64) / 50.0
    return A, dA, x, y


def _single_process(adjoint):
    import torch
    A, dA, x, y = _system()
    full = DenseRows(A, dA, 0, D)
    xt = torch.from_numpy(x)
    u = torch.from_numpy(np.linspace(-1.0, 1.0, D).astype(np.float32))
    theta = torch.zeros(THETA_N, dtype=torch.float64, requires_grad=True)
    loss = ((adjoint.project(theta, xt, full) - torch.from_numpy(y)) ** 2).sum()
    loss.backward()
    return dict(vjp=full.vjp(xt, u).numpy(), bp=full.backproject(u).numpy(),
                mlem=adjoint.mlem(full, torch.from_numpy(y), 5).numpy(), grad=theta.grad.numpy())


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    adjoint = _load("sysmat_adjoint", os.path.join(PKG_DIR, "adjoint.py"))
    A, dA, x, y = _system()
    b, c = adjoint.sharding.detector_slab(D, rank, world)
    sp = adjoint.ShardedProjector(types.SimpleNamespace(n_det=D, n_vox=V), local=DenseRows(A, dA, b, c))
    assert (sp.det_begin, sp.det_count) == (b, c)
    xt = torch.from_numpy(x)
    u = torch.from_numpy(np.linspace(-1.0, 1.0, D).astype(np.float32))[b:b + c].contiguous()
    yl = torch.from_numpy(y[b:b + c].copy())
    theta = torch.zeros(THETA_N, dtype=torch.float64, requires_grad=True)
    loss = ((adjoint.project(theta, xt, sp) - yl) ** 2).sum()
    loss.backward()
    res = dict(rows=(b, c), proj=sp.project(xt).numpy(), vjp=sp.vjp(xt, u).numpy(),
               bp=sp.backproject(u).numpy(), mlem=adjoint.mlem(sp, yl, 5).numpy(), grad=theta.grad.numpy())
    q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_projector_equals_single_process():
    import torch.multiprocessing as mp
    adjoint = _load("sysmat_adjoint", os.path.join(PKG_DIR, "adjoint.py"))
    ref = _single_process(adjoint)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    out = dict(q.get() for _ in range(2))
    A, _, x, _ = _system()
    assert [out[r]["rows"] for r in (0, 1)] == [(0, 4), (4, 3)]
    proj = np.concatenate([out[0]["proj"], out[1]["proj"]])
    assert np.allclose(proj, A @ x.astype(np.float64), rtol=1e-12, atol=0)
    for r in (0, 1):                          # every rank holds the same totals
        for key in ("vjp", "bp", "grad"):
            assert np.allclose(out[r][key], ref[key], rtol=1e-12, atol=1e-12), (r, key)
        assert np.allclose(out[r]["mlem"], ref["mlem"], rtol=1e-5, atol=0), r
    assert np.array_equal(out[0]["mlem"], out[1]["mlem"])
