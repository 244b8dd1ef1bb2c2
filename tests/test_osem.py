"""CPU tests of OSEM and MLEM (adjoint.osem / adjoint.mlem) and of the all-rotations
projector (adjoint.RotationProjector) on dense stand-ins.

Both functions only call the projector's project / backproject (over row blocks for OSEM),
which on a GPU are sysmat_project / sysmat_backproject (tested against the dense matrix in
test_gpu_adjoint.py).  Here a seeded dense A stands in for them, so the update rules are
checked on CPU: OSEM against an independent numpy OSEM, one subset against MLEM."""
import os
import types

import numpy as np

from conftest import PKG_DIR, _load

adjoint = _load("sysmat_adjoint", os.path.join(PKG_DIR, "adjoint.py"))

D, V = 23, 17


class DenseProjector:
    def __init__(self, A):
        import torch
        self.A = torch.from_numpy(A)
        self.det_count = A.shape[0]
        self.geo = types.SimpleNamespace(n_det=A.shape[0], n_vox=A.shape[1])

    def _block(self, rows):
        b, n = (0, self.det_count) if rows is None else rows
        return self.A[b:b + n]

    def project(self, x, theta=None, rows=None):
        return self._block(rows) @ x.double()

    def backproject(self, u, theta=None, rows=None):
        return self._block(rows).T @ u.double()


def _problem():
    rng = np.random.default_rng(23)
    A = rng.uniform(0.0, 1.0, (D, V))
    A[rng.random((D, V)) < 0.4] = 0.0
    A[:, 5] = 0.0                                          # a voxel no row sees
    x_true = rng.uniform(0.5, 3.0, V)
    y = rng.poisson(A @ x_true * 40.0) / 40.0
    return A, y


def _numpy_osem(A, y, n_iter, n_subsets):
    x = np.ones(A.shape[1], dtype=np.float32)
    blocks = [adjoint.sharding.detector_slab(A.shape[0], s, n_subsets) for s in range(n_subsets)]
    for _ in range(n_iter):
        for b, n in blocks:
            As, ys = A[b:b + n], y[b:b + n]
            sens = As.sum(0)
            p = As @ x.astype(np.float64)
            ratio = np.where(p > 0, ys / np.where(p > 0, p, 1.0), 0.0).astype(np.float32)
            bp = As.T @ ratio.astype(np.float64)
            x = np.where(sens > 0, x.astype(np.float64) * bp / np.where(sens > 0, sens, 1.0), 0.0).astype(np.float32)
    return x


def test_osem_matches_numpy_osem():
    import torch
    A, y = _problem()
    P = DenseProjector(A)
    for n_subsets in (1, 3, 5):
        x = adjoint.osem(P, torch.from_numpy(y), 4, n_subsets).numpy()
        ref = _numpy_osem(A, y, 4, n_subsets)
        assert np.allclose(x, ref, rtol=1e-6, atol=0), n_subsets
        assert x[5] == 0.0                                  # unseen voxel


def test_one_subset_is_mlem():
    import torch
    A, y = _problem()
    P = DenseProjector(A)
    yt = torch.from_numpy(y)
    assert np.allclose(adjoint.osem(P, yt, 3, 1).numpy(), adjoint.mlem(P, yt, 3).numpy(), rtol=1e-6, atol=0)


def test_osem_raises_the_likelihood_faster_than_mlem():
    """One OSEM iteration with 4 subsets reaches at least the Poisson likelihood of two MLEM
    iterations (each subset update is an EM step on a quarter of the data)."""
    import torch
    A, y = _problem()
    P = DenseProjector(A)
    yt = torch.from_numpy(y)

    def nll(x):
        p = A @ x.astype(np.float64)
        return float((p - y * np.log(np.maximum(p, 1e-300))).sum())

    assert nll(adjoint.osem(P, yt, 1, 4).numpy()) <= nll(adjoint.mlem(P, yt, 2).numpy())


# ---- all rotations as one projector (adjoint.RotationProjector) -------------------------

R = 3


class DenseContext:
    """sysmat.Context's projection methods over dense per-rotation matrices A[r] (and
    derivative matrices dA[r, i] for the VJP)."""

    def __init__(self, A, dA):
        import torch
        self.A, self.dA = torch.from_numpy(A), torch.from_numpy(dA)

    def project(self, x, rotation, det_begin, det_count):
        return self.A[int(rotation), det_begin:det_begin + det_count] @ x.double()

    def backproject(self, u, rotation, det_begin, det_count):
        return self.A[int(rotation), det_begin:det_begin + det_count].T @ u.double()

    def vjp(self, x, u, rotation, det_begin, det_count):
        import torch
        r, rows = int(rotation), slice(det_begin, det_begin + det_count)
        u, x = u.double(), x.double()
        return torch.stack([u @ (self.dA[r, i, rows] @ x) for i in range(7)] + [u @ (self.A[r, rows] @ x)])


def _rotations():
    rng = np.random.default_rng(29)
    A = rng.uniform(0.0, 1.0, (R, D, V))
    A[rng.random((R, D, V)) < 0.4] = 0.0
    dA = rng.normal(size=(R, 7, D, V))
    geo = types.SimpleNamespace(n_det=D, n_vox=V, n_rot=R)
    return A, dA, adjoint.RotationProjector(geo, context=lambda theta: DenseContext(A, dA))


def test_rotation_projector_stacks_rotations():
    import torch
    A, dA, P = _rotations()
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.uniform(0.5, 2.0, V).astype(np.float32))
    u = torch.from_numpy(rng.normal(size=R * D).astype(np.float32))
    stacked = A.reshape(R * D, V)
    assert P.det_count == R * D
    assert np.allclose(P.project(x).numpy(), stacked @ x.numpy(), rtol=1e-12)
    assert np.allclose(P.backproject(u).numpy(), stacked.T @ u.numpy(), rtol=1e-12)
    b, n = D - 5, D + 9                                   # spans all three rotations
    assert np.allclose(P.project(x, rows=(b, n)).numpy(), stacked[b:b + n] @ x.numpy(), rtol=1e-12)
    assert np.allclose(P.backproject(u[:n], rows=(b, n)).numpy(), stacked[b:b + n].T @ u[:n].numpy(), rtol=1e-12)
    g = P.vjp(x, u).numpy()
    uu = u.numpy().astype(np.float64).reshape(R, D)
    ref = [sum(uu[r] @ dA[r, i] @ x.numpy() for r in range(R)) for i in range(7)]
    assert np.allclose(g[:7], ref, rtol=1e-10) and np.isclose(g[7], u.numpy() @ stacked @ x.numpy(), rtol=1e-10)


def test_osem_by_rotation_matches_numpy():
    import torch
    A, _, P = _rotations()
    stacked = A.reshape(R * D, V)
    y = np.random.default_rng(2).poisson(stacked @ np.full(V, 2.0) * 30.0) / 30.0
    x = adjoint.osem(P, torch.from_numpy(y), 3, R).numpy()
    assert np.allclose(x, _numpy_osem(stacked, y, 3, R), rtol=1e-6, atol=0)   # one rotation per subset
