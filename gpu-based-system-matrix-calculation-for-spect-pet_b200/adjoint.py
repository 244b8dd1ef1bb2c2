"""Differentiable forward projection and MLEM reconstruction over libsysmat's on-the-fly
projector (sysmat_project / sysmat_vjp / sysmat_backproject).

The reference only writes the dense system matrix (PEGen_RayTracing_CircularHole/
PESysMatGen.cu:1368-1437); its consumers multiply it.  Here the matrix is recomputed brick by
brick inside each product, so a calibration loop over collimator parameters theta, or an MLEM
reconstruction, needs no matrix memory.  theta = (mu_W, mu_crystal, hole radius, dx, dy, dz,
tilt), as geometry.apply_theta applies it to the parameter arrays.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


sysmat = _load("sysmat_binding", os.path.join(HERE, "sysmat.py"))
geometry = _load("sysmat_geometry", os.path.join(HERE, "geometry.py"))
sharding = _load("sysmat_sharding", os.path.join(HERE, "sharding.py"))


class Projector:
    """A system whose parameters theta may change; keeps the context of the last theta.
    shapes: optional (n_holes, 3) rows (rho_x, rho_z, theta_h) of elliptical holes
    (sysmat_set_hole_shapes); the tilt turns their frames with the pattern."""

    def __init__(self, geo, device=0, rotation=0.0, det_begin=0, det_count=None, shapes=None):
        self.geo = geo
        self.device = device
        self.rotation = float(rotation)
        self.det_begin = det_begin
        self.det_count = geo.n_det - det_begin if det_count is None else det_count
        self.shapes = None if shapes is None else np.asarray(shapes, dtype=np.float32).reshape(-1, 3)
        self._theta = None
        self._ctx = None

    def context(self, theta=None):
        theta = geometry.theta_of(self.geo) if theta is None else np.asarray(theta, dtype=np.float64)
        if self._ctx is None or not np.array_equal(theta, self._theta):
            if self._ctx is not None:
                self._ctx.close()
            self._ctx = sysmat.Context(geometry.apply_theta(self.geo, theta), device=self.device)
            if self.shapes is not None:
                self._ctx.set_hole_shapes(geometry.apply_theta_shapes(self.shapes, theta))
            self._theta = theta.copy()
        return self._ctx

    def project(self, x, theta=None, rows=None):
        """A x over the projector's rows, or over rows = (first, count) relative to them."""
        b, n = self._rows(rows)
        return self.context(theta).project(x, rotation=self.rotation, det_begin=b, det_count=n)

    def backproject(self, u, theta=None, rows=None):
        b, n = self._rows(rows)
        return self.context(theta).backproject(u, rotation=self.rotation, det_begin=b, det_count=n)

    def _rows(self, rows):
        if rows is None:
            return self.det_begin, self.det_count
        first, count = rows
        if first < 0 or count < 0 or first + count > self.det_count:
            raise ValueError("rows outside the projector's detector rows")
        return self.det_begin + first, count

    def vjp(self, x, u, theta=None):
        return self.context(theta).vjp(x, u, rotation=self.rotation, det_begin=self.det_begin,
                                       det_count=self.det_count)


class RotationProjector:
    """All rotations of one system as one projector: its rows are (rotation, detector) pairs,
    rotation-major, as the reference's matrix stacks them (A[rotation][detector][voxel]).
    project / backproject / vjp accept any block of rows (rows = (first, count)); a block that
    spans rotations is split into one device call per rotation, and back projections and
    gradients are summed over them.  OSEM with n_subsets = the number of rotations takes one
    rotation per subset.

    `context(theta)` may be given to supply the per-theta device context (an object with the
    sysmat.Context project / backproject / vjp methods); by default a Projector's is used."""

    def __init__(self, geo, rotations=None, device=0, context=None, shapes=None):
        self.geo = geo
        self.rotations = [float(r) for r in (range(geo.n_rot) if rotations is None else rotations)]
        self.n_det = geo.n_det
        self.det_count = len(self.rotations) * self.n_det
        self._context = context if context is not None else Projector(geo, device=device, shapes=shapes).context

    def _pieces(self, rows):
        first, count = (0, self.det_count) if rows is None else rows
        if first < 0 or count < 0 or first + count > self.det_count:
            raise ValueError("rows outside the projector's rows")
        pos, end, out = first, first + count, []
        while pos < end:
            r, d0 = divmod(pos, self.n_det)
            n = min(self.n_det - d0, end - pos)
            out.append((self.rotations[r], d0, n, pos - first))
            pos += n
        return out

    def project(self, x, theta=None, rows=None):
        ctx = self._context(theta)
        return torch.cat([ctx.project(x, rotation=rot, det_begin=d0, det_count=n)
                          for rot, d0, n, _ in self._pieces(rows)])

    def backproject(self, u, theta=None, rows=None):
        ctx = self._context(theta)
        q = None
        for rot, d0, n, off in self._pieces(rows):
            part = ctx.backproject(u[off:off + n].contiguous(), rotation=rot, det_begin=d0, det_count=n)
            q = part if q is None else q + part
        return q

    def vjp(self, x, u, theta=None):
        ctx = self._context(theta)
        g = None
        for rot, d0, n, off in self._pieces(None):
            part = ctx.vjp(x, u[off:off + n].contiguous(), rotation=rot, det_begin=d0, det_count=n)
            g = part if g is None else g + part
        return g


class ShardedProjector:
    """A projector whose detector rows are split across the ranks of a process group
    (sharding.detector_slab), one GPU per rank.  Each rank recomputes only its own rows of A.
    Projections stay local (a rank's rows of A x); the products that sum over detector rows
    are completed with one all-reduce each: the back projection (n_vox values) and the theta
    gradient with u^T A x (8 values).  Every rank then holds the same totals, so an MLEM loop
    or a calibration step proceeds identically on all ranks.

    `local` builds the rank's own projector (default: Projector on this rank's rows); any
    object with project / backproject / vjp over rows det_begin .. det_begin + det_count
    will do."""

    def __init__(self, geo, group=None, rotation=0.0, device=None, local=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.geo = geo
        self.det_begin, self.det_count = sharding.detector_slab(geo.n_det, self.rank, self.world)
        if local is None:
            dev = torch.cuda.current_device() if device is None else device
            local = Projector(geo, device=dev, rotation=rotation, det_begin=self.det_begin,
                              det_count=self.det_count)
        self.local = local

    def _sum(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def project(self, x, theta=None):
        return self.local.project(x, theta)

    def backproject(self, u, theta=None):
        return self._sum(self.local.backproject(u, theta))

    def vjp(self, x, u, theta=None):
        return self._sum(self.local.vjp(x, u, theta))


class Projection(torch.autograd.Function):
    """p = A(theta) x.  theta: CPU float64 tensor of 7; x: CUDA float32 tensor of n_vox;
    p: CUDA float64 tensor of the projector's detector rows.  Backward gives d/d theta through
    sysmat_vjp and d/d x through sysmat_backproject."""

    @staticmethod
    def forward(fctx, theta, x, projector):
        th = theta.detach().cpu().numpy().astype(np.float64)
        x = x.detach().to(torch.float32).contiguous()
        fctx.projector = projector
        fctx.theta = th
        fctx.save_for_backward(x)
        return projector.project(x, th)

    @staticmethod
    def backward(fctx, grad_p):
        (x,) = fctx.saved_tensors
        u = grad_p.detach().to(torch.float32).contiguous()
        g_theta = g_x = None
        if fctx.needs_input_grad[0]:
            g = fctx.projector.vjp(x, u, fctx.theta)
            g_theta = g[:sysmat.THETA_N].cpu().to(torch.float64)
        if fctx.needs_input_grad[1]:
            g_x = fctx.projector.backproject(u, fctx.theta).to(torch.float32)
        return g_theta, g_x, None


def project(theta, x, projector):
    return Projection.apply(theta, x, projector)


def osem(projector, y, n_iter, n_subsets, x0=None, theta=None):
    """OSEM: the MLEM update applied subset by subset, the subsets being contiguous blocks
    of the projector's detector rows (sharding.detector_slab); n_subsets = 1 is mlem.
    y: CUDA tensor of the projector's detector rows; returns a float32 CUDA tensor of n_vox.
    One iteration visits every subset once, in order."""
    dev = y.device
    n_rows = projector.det_count
    subsets = [sharding.detector_slab(n_rows, s, n_subsets) for s in range(n_subsets)]
    subsets = [r for r in subsets if r[1] > 0]
    sens = [projector.backproject(torch.ones(n, dtype=torch.float32, device=dev), theta, rows=(b, n))
            for b, n in subsets]
    x = torch.ones(projector.geo.n_vox, dtype=torch.float32, device=dev) if x0 is None else x0.clone()
    yd = y.to(torch.float64)
    for _ in range(n_iter):
        for (b, n), sn in zip(subsets, sens):
            p = projector.project(x, theta, rows=(b, n))
            ys = yd[b:b + n]
            ratio = torch.where(p > 0, ys / p, torch.zeros_like(p)).to(torch.float32)
            bp = projector.backproject(ratio, theta, rows=(b, n))
            x = torch.where(sn > 0, x.to(torch.float64) * bp / sn, torch.zeros_like(sn)).to(torch.float32)
    return x


def mlem(projector, y, n_iter, x0=None, theta=None):
    """MLEM reconstruction x <- x / (A^T 1) * A^T (y / A x) with the on-the-fly projector.
    y: CUDA tensor of the projector's detector rows; returns a float32 CUDA tensor of n_vox.
    With a ShardedProjector, y holds this rank's rows and every rank returns the same x."""
    dev = y.device
    sens = projector.backproject(torch.ones(projector.det_count, dtype=torch.float32, device=dev), theta)
    x = torch.ones(projector.geo.n_vox, dtype=torch.float32, device=dev) if x0 is None else x0.clone()
    yd = y.to(torch.float64)
    for _ in range(n_iter):
        p = projector.project(x, theta)
        ratio = torch.where(p > 0, yd / p, torch.zeros_like(p)).to(torch.float32)
        bp = projector.backproject(ratio, theta)
        x = torch.where(sens > 0, x.to(torch.float64) * bp / sens, torch.zeros_like(sens)).to(torch.float32)
    return x
