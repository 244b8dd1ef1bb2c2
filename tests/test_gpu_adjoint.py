"""GPU tests of the on-the-fly projector: forward projection, back projection, the
vector-Jacobian product with respect to the collimator/crystal parameters theta, the
torch.autograd shim and MLEM, all through the C ABI.

Products are checked against the dense matrix from sysmat_pe (precise mode).  The VJP is
checked against an FP64 CPU gradient: central differences of the FP64 oracle with steps that
the float parameter arrays represent exactly (h = 2^-20), and for the tilt the identity
d/dtilt = sum_h (-z_h d/dx_h + x_h d/dz_h) over per-hole differences (a rotated hole centre
is rounded to float, so a tilt step is not exact).  Small steps matter: the reference's
cylinder chord is continuous but very steep for near-axial rays (the wall crossing moves
~1/sqrt(kk) times faster than the hole), with kinks where a crossing moves onto a cap, so a
difference over h ~ 1e-4 averages slopes from both sides of nearby kinks.  The finite
differences of the GPU projection on configuration 5 (h = 2^-13) are checked to the accuracy
that allows."""
import importlib.util
import os

import numpy as np
import pytest

from conftest import PKG_DIR, geometry, oracle, sysmat

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("sysmat_adjoint", os.path.join(PKG_DIR, "adjoint.py"))
adjoint = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(adjoint)


def _dense(torch, ctx, rotation=0.0):
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    ctx.pe(out, rotation=rotation, mode=sysmat.MODE_PRECISE)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64)


def _ellipses(geo, every=2):
    """Every `every`-th hole elliptical (semi-axes 0.8 and 0.55 of its radius, seeded frame
    angles in [0.3, 3.5) rad); the others circular."""
    r = geo.collimator[104:104 + 9 * geo.n_holes:9]
    sh = np.zeros((geo.n_holes, 3), dtype=np.float32)
    k = np.arange(geo.n_holes)
    e = k % every == 0
    sh[e, 0] = 0.8 * r[e]
    sh[e, 1] = 0.55 * r[e]
    sh[e, 2] = (0.3 + (0.37 * k[e]) % 3.2).astype(np.float32)
    return sh


@pytest.mark.parametrize("case", ["mini_rot", "config1", "mini_ell"])
def test_products_equal_dense_matrix_products(gpu, case):
    torch = gpu
    if case == "mini_rot":
        geo = geometry.mini(seed=31, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))
        rot = 3.0
    elif case == "mini_ell":
        geo = geometry.mini(seed=31, rotated=True, layers=2, n_rot=8, nvox=(6, 5, 3), ncry=(5, 4))
        rot = 5.0
    else:
        geo, rot = geometry.config1(), 0.0
    ctx = sysmat.Context(geo)
    if case == "mini_ell":
        ctx.set_hole_shapes(_ellipses(geo))
    A = _dense(torch, ctx, rot)
    rng = np.random.default_rng(7)
    x = rng.uniform(0.0, 2.0, ctx.n_vox).astype(np.float32)
    x[rng.random(ctx.n_vox) < 0.3] = 0.0                 # zero voxels are skipped
    u = rng.normal(size=ctx.n_det).astype(np.float32)
    xt, ut = torch.from_numpy(x).cuda(), torch.from_numpy(u).cuda()
    p = ctx.project(xt, rotation=rot).cpu().numpy()
    q = ctx.backproject(ut, rotation=rot).cpu().numpy()
    g = ctx.vjp(xt, ut, rotation=rot).cpu().numpy()
    p_ref = A @ x.astype(np.float64)
    q_ref = A.T @ u.astype(np.float64)
    assert np.abs(p - p_ref).max() <= 1e-6 * np.abs(p_ref).max()
    assert np.abs(q - q_ref).max() <= 1e-6 * np.abs(q_ref).max()
    s_ref = float(u.astype(np.float64) @ p_ref)
    assert abs(g[sysmat.THETA_N] - s_ref) <= 1e-6 * float(np.abs(u) @ np.abs(p_ref))
    # a detector-row block equals the same rows of the full product
    pb = ctx.project(xt, rotation=rot, det_begin=3, det_count=5).cpu().numpy()
    assert np.allclose(pb, p[3:8], rtol=1e-12, atol=0)


def test_vjp_matches_fp64_oracle_gradient(gpu):
    torch = gpu
    geo = geometry.mini(seed=41, layers=2, nvox=(6, 5, 2), ncry=(4, 4), nholes=3)
    rng = np.random.default_rng(1)
    x = rng.uniform(0.5, 2.0, geo.n_vox).astype(np.float32)
    u = rng.normal(size=geo.n_det).astype(np.float32)
    x64, u64 = x.astype(np.float64), u.astype(np.float64)
    P = adjoint.Projector(geo)
    t0 = geometry.theta_of(geo)
    g = P.vjp(torch.from_numpy(x).cuda(), torch.from_numpy(u).cuda(), t0).cpu().numpy()

    def s_of(gg):
        return float(u64 @ oracle.pe(gg, prec=64) @ x64)

    h = 2.0 ** -20
    for i in range(6):                                   # mu_W .. dz
        tp, tm = t0.copy(), t0.copy()
        tp[i] += h
        tm[i] -= h
        fd = (s_of(geometry.apply_theta(geo, tp)) - s_of(geometry.apply_theta(geo, tm))) / (2 * h)
        assert abs(g[i] - fd) <= 1e-3 * abs(fd), (sysmat.THETA_NAMES[i], g[i], fd)
    tilt = 0.0
    for k in range(geo.n_holes):
        d = []
        for col in (100 + 9 * k, 103 + 9 * k):           # hole x, hole z
            cp, cm = geo.collimator.copy(), geo.collimator.copy()
            cp[col] += np.float32(h)
            cm[col] -= np.float32(h)
            d.append((s_of(geometry.Geometry(geo.name, cp, geo.detector, geo.image, geo.physics)) -
                      s_of(geometry.Geometry(geo.name, cm, geo.detector, geo.image, geo.physics))) / (2 * h))
        tilt += -float(geo.collimator[103 + 9 * k]) * d[0] + float(geo.collimator[100 + 9 * k]) * d[1]
    assert abs(g[6] - tilt) <= 1e-3 * abs(tilt), (g[6], tilt)


def test_vjp_with_elliptical_holes_matches_fp64_oracle_gradient(gpu):
    """Elliptical holes: the VJP against central differences of the FP64 oracle with the same
    shapes; the tilt against the identity sum_h (-z_h d/dx_h + x_h d/dz_h) plus the frame
    angle d/dtheta_h of every elliptical hole (the tilt turns their frames)."""
    torch = gpu
    geo = geometry.mini(seed=41, layers=2, nvox=(6, 5, 2), ncry=(4, 4), nholes=3)
    shapes = _ellipses(geo)
    rng = np.random.default_rng(1)
    x = rng.uniform(0.5, 2.0, geo.n_vox).astype(np.float32)
    u = rng.normal(size=geo.n_det).astype(np.float32)
    x64, u64 = x.astype(np.float64), u.astype(np.float64)
    P = adjoint.Projector(geo, shapes=shapes)
    t0 = geometry.theta_of(geo)
    g = P.vjp(torch.from_numpy(x).cuda(), torch.from_numpy(u).cuda(), t0).cpu().numpy()

    def s_of(gg, sh=shapes):
        return float(u64 @ oracle.pe(gg, prec=64, shapes=sh) @ x64)

    assert abs(g[sysmat.THETA_N] - s_of(geo)) <= 1e-6 * abs(s_of(geo))
    h = 2.0 ** -20
    for i in range(6):                                   # mu_W .. dz
        tp, tm = t0.copy(), t0.copy()
        tp[i] += h
        tm[i] -= h
        fd = (s_of(geometry.apply_theta(geo, tp)) - s_of(geometry.apply_theta(geo, tm))) / (2 * h)
        if i == 2:                                       # circular holes only move with the radius
            assert abs(g[i] - fd) <= 1e-3 * abs(fd) + 1e-9 * abs(s_of(geo)), (g[i], fd)
        else:
            assert abs(g[i] - fd) <= 1e-3 * abs(fd), (sysmat.THETA_NAMES[i], g[i], fd)
    tilt = 0.0
    for k in range(geo.n_holes):
        for col, wgt in ((100 + 9 * k, -float(geo.collimator[103 + 9 * k])),
                         (103 + 9 * k, float(geo.collimator[100 + 9 * k]))):
            cp, cm = geo.collimator.copy(), geo.collimator.copy()
            cp[col] += np.float32(h)
            cm[col] -= np.float32(h)
            tilt += wgt * (s_of(geometry.Geometry(geo.name, cp, geo.detector, geo.image, geo.physics)) -
                           s_of(geometry.Geometry(geo.name, cm, geo.detector, geo.image, geo.physics))) / (2 * h)
        if shapes[k, 0] > 0:                             # the frame turns with the pattern
            sp, sm = shapes.copy(), shapes.copy()
            sp[k, 2] += np.float32(h)
            sm[k, 2] -= np.float32(h)
            tilt += (s_of(geo, sp) - s_of(geo, sm)) / (2 * h)
    assert abs(g[6] - tilt) <= 1e-3 * abs(tilt), (g[6], tilt)


def test_vjp_matches_finite_differences_config5(gpu):
    """Configuration 5: loss = |A(theta) x - y|^2, y = A(theta*) x; d loss / d theta by the VJP
    with u = 2 (A x - y) against central differences of u^T A(theta) x (h = 2^-13, the FP32
    projection).  The attenuation coefficients move no geometry: tight agreement.  For the
    geometric parameters the difference step straddles chord kinks (module docstring), which
    bounds the agreement; the FP64 oracle test above checks them with small steps."""
    torch = gpu
    geo, x, t0, ts = geometry.config5()
    P = adjoint.Projector(geo)
    xt = torch.from_numpy(x).cuda()
    y = P.project(xt, ts)
    u = (2.0 * (P.project(xt, t0) - y)).float()
    g = P.vjp(xt, u, t0).cpu().numpy()
    h = 2.0 ** -13
    fd = np.zeros(sysmat.THETA_N)
    for i in range(sysmat.THETA_N):
        tp, tm = t0.copy(), t0.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (float((u.double() * P.project(xt, tp)).sum()) - float((u.double() * P.project(xt, tm)).sum())) / (2 * h)
    rel = np.abs(g[:sysmat.THETA_N] - fd) / np.abs(fd)
    assert rel[0] < 1e-4 and rel[1] < 1e-4, rel            # mu_W, mu_crystal
    assert np.all(rel[2:] < 3e-2), rel
    assert np.abs(g[:sysmat.THETA_N] - fd).max() < 1e-2 * np.abs(fd).max(), (g, fd)


def test_autograd_shim_gives_vjp_and_backprojection(gpu):
    torch = gpu
    geo = geometry.mini(seed=32, layers=1, nvox=(6, 6, 2), ncry=(5, 5))
    P = adjoint.Projector(geo)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.uniform(0.5, 2.0, geo.n_vox).astype(np.float32)).cuda().requires_grad_(True)
    t0 = geometry.theta_of(geo)
    theta = torch.tensor(t0, dtype=torch.float64, requires_grad=True)
    y = P.project(x.detach(), t0 + np.array([0, 0, 0.01, 0.05, 0, -0.03, 0.002]))
    loss = ((adjoint.project(theta, x, P) - y) ** 2).sum()
    loss.backward()
    r = (P.project(x.detach(), t0) - y)
    u = (2.0 * r).float()
    g = P.vjp(x.detach(), u, t0).cpu().numpy()
    q = P.backproject(u, t0).float()
    assert np.allclose(theta.grad.numpy(), g[:sysmat.THETA_N], rtol=1e-12, atol=0)
    assert torch.allclose(x.grad, q, rtol=1e-6, atol=0)


def test_mlem_matches_dense_mlem_and_raises_likelihood(gpu):
    torch = gpu
    geo = geometry.config1()
    ctx = sysmat.Context(geo)
    A = _dense(torch, ctx)
    rng = np.random.default_rng(11)
    x_true = geometry.ellipsoid_phantom((32, 32, 1), (1.0, 1.0, 1.0), 3, seed=2).astype(np.float64) + 0.1
    y = rng.poisson(A @ x_true * 1e6 / (A @ x_true).sum()).astype(np.float64)
    P = adjoint.Projector(geo)
    n_iter = 4
    x = adjoint.mlem(P, torch.from_numpy(y).cuda(), n_iter).cpu().numpy().astype(np.float64)
    sens = A.sum(0)
    xd = np.ones(geo.n_vox)
    nll = []
    for _ in range(n_iter):
        p = A @ xd
        nll.append(float((p - y * np.log(np.maximum(p, 1e-300))).sum()))
        xd = np.where(sens > 0, xd * (A.T @ np.where(p > 0, y / p, 0.0)) / np.where(sens > 0, sens, 1), 0.0)
    assert np.abs(x - xd).max() <= 1e-4 * np.abs(xd).max()
    assert all(b <= a + 1e-9 * abs(a) for a, b in zip(nll, nll[1:]))   # MLEM never lowers the likelihood


def test_osem_matches_dense_osem(gpu):
    """OSEM over 4 row-block subsets with the on-the-fly projector equals the same OSEM on the
    dense matrix."""
    torch = gpu
    geo = geometry.config1()
    A = _dense(torch, sysmat.Context(geo))
    rng = np.random.default_rng(12)
    x_true = geometry.ellipsoid_phantom((32, 32, 1), (1.0, 1.0, 1.0), 3, seed=3).astype(np.float64) + 0.1
    y = rng.poisson(A @ x_true * 1e6 / (A @ x_true).sum()).astype(np.float64)
    P = adjoint.Projector(geo)
    x = adjoint.osem(P, torch.from_numpy(y).cuda(), 2, 4).cpu().numpy().astype(np.float64)
    xd = np.ones(geo.n_vox)
    blocks = [adjoint.sharding.detector_slab(geo.n_det, s, 4) for s in range(4)]
    for _ in range(2):
        for b, n in blocks:
            As, ys = A[b:b + n], y[b:b + n]
            sens, p = As.sum(0), As @ xd
            xd = np.where(sens > 0, xd * (As.T @ np.where(p > 0, ys / np.where(p > 0, p, 1), 0.0)) /
                          np.where(sens > 0, sens, 1), 0.0)
    assert np.abs(x - xd).max() <= 1e-4 * np.abs(xd).max()


def test_rotation_osem_matches_dense_stacked_osem(gpu):
    """OSEM with one rotation per subset on the all-rotations projector (RotationProjector: rows
    (rotation, detector), rotation-major as the reference stacks its matrices) equals the same
    OSEM on the dense stacked matrix."""
    torch = gpu
    geo = geometry.mini(seed=23, rotated=True, layers=2, n_rot=4, nvox=(6, 5, 2), ncry=(5, 4))
    ctx = sysmat.Context(geo)
    A = np.concatenate([_dense(torch, ctx, float(r)) for r in range(geo.n_rot)])
    rng = np.random.default_rng(13)
    x_true = rng.uniform(0.5, 2.0, geo.n_vox)
    y = rng.poisson(A @ x_true * 1e6 / (A @ x_true).sum()).astype(np.float64)
    P = adjoint.RotationProjector(geo)
    x = adjoint.osem(P, torch.from_numpy(y).cuda(), 3, geo.n_rot).cpu().numpy().astype(np.float64)
    xd = np.ones(geo.n_vox)
    n = geo.n_det
    for _ in range(3):
        for r in range(geo.n_rot):
            As, ys = A[r * n:(r + 1) * n], y[r * n:(r + 1) * n]
            sens, p = As.sum(0), As @ xd
            xd = np.where(sens > 0, xd * (As.T @ np.where(p > 0, ys / np.where(p > 0, p, 1), 0.0)) /
                          np.where(sens > 0, sens, 1), 0.0)
    assert np.abs(x - xd).max() <= 1e-4 * np.abs(xd).max()


def test_invalid_adjoint_calls_raise(gpu):
    torch = gpu
    geo = geometry.mini(seed=33)
    ctx = sysmat.Context(geo)
    x = torch.ones(ctx.n_vox, dtype=torch.float32, device="cuda")
    u = torch.ones(ctx.n_det, dtype=torch.float32, device="cuda")
    with pytest.raises(sysmat.SysmatError):
        ctx.project(x, det_begin=ctx.n_det - 1, det_count=2)
    with pytest.raises(sysmat.SysmatError):
        ctx.vjp(x, u, det_begin=-1, det_count=1)
    p = ctx.project(x, det_count=0)
    assert p.numel() == 0
