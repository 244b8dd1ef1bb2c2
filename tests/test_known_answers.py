"""Analytic known answers for the photoelectric element, on the oracle (CPU) and on every
device mode (GPU).

A single crystal 1000 mm from a one-voxel image, on its axis.  Every sub-element ray is then
within 1e-3 rad of the axis, so it enters its crystal column through the top faces: its path
in the crystal before its sub-element is iy * (t/16) * d/dy and its absorption chord is
(t/16) * d/dy, with d the ray length and dy its depth component.  The element is therefore,
per sub-element s (PESysMatGen.cu:1196-1357),

    Omega_s * exp(-mu_W T d/dy [plate]) * exp(-mu iy (t/16) d/dy) * (1 - exp(-mu (t/16) d/dy))
    * mu_pe / mu,

with Omega_s the largest of the sub-element's three face projections.  Three collimators:
none (no layer: the plate penalty and layer terms are absent), a plain tungsten plate of
thickness T (the layer term T/cos(theta), no hole chord), and the same plate with a hole on
the axis wide enough to pass every ray (the hole chord cancels T/cos(theta) exactly, below
the layer term's threshold, so the element equals the bare one)."""
import numpy as np
import pytest

from conftest import geometry, oracle, sysmat

R, W, T, H = 1000.0, 2.0, 5.0, 2.0          # crystal distance and size (x, depth, z), mm
# the parameter arrays hold float32: the closed form uses the values they store
MU, MU_PE = float(np.float32(0.23)), float(np.float32(0.18))
MU_W, PLATE_T, PLATE_Y = float(np.float32(3.4)), 1.0, 500.0


def _geometry(collimator):
    cb = geometry._CollimatorBuilder()
    if collimator in ("plate", "hole"):
        holes = [(0.0, 0.0, 5.0)] if collimator == "hole" else []
        cb.add_layer(40.0, PLATE_T, 40.0, PLATE_Y, MU_W, MU_W * 0.87, MU_W * 0.13, holes)
    det = geometry._detector([(0.0, R, 0.0)], (W, T, H), mu=(MU, MU_PE))
    img = geometry._image((1, 1, 1), (1.0, 1.0, 1.0), 0.0)
    return geometry.Geometry(f"known_{collimator}", cb.build(), det, img, geometry._physics())


def closed_form(collimator, div=(8, 16, 8)):
    nx, ny, nz = div
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = -W / 2 + (ix + 0.5) / nx * W
    y = R - T / 2 + (iy + 0.5) / ny * T
    z = -H / 2 + (iz + 0.5) / nz * H
    d = np.sqrt(x * x + y * y + z * z)
    sec = d / y                                       # 1 / cos(theta) of each ray
    four_pi_d3 = 4.0 * np.pi * d ** 3
    omega = np.maximum.reduce([T * H / nz / ny * np.abs(x) / four_pi_d3,
                               W * T / nx / ny * np.abs(z) / four_pi_d3,
                               W * H / nx / nz * np.abs(y) / four_pi_d3])
    step = T / ny * sec
    val = omega * np.exp(-MU * iy * step) * (1.0 - np.exp(-MU * step)) * MU_PE / MU
    if collimator == "plate":
        val = val * np.exp(-MU_W * PLATE_T * sec)
    return float(val.sum())


@pytest.mark.parametrize("collimator", ["none", "plate", "hole"])
@pytest.mark.parametrize("prec, tol", [(64, 1e-10), (32, 2e-6), ("local", 2e-7)])
def test_oracle_known_answer(collimator, prec, tol):
    g = _geometry(collimator)
    a = float((oracle.pe_local(g) if prec == "local" else oracle.pe(g, prec=prec))[0, 0])
    b = closed_form("none" if collimator == "hole" else collimator)
    assert abs(a - b) <= tol * b, (a, b, abs(a - b) / b)


def test_known_answers_differ_as_the_physics_says():
    bare, plate = closed_form("none"), closed_form("plate")
    assert np.isclose(plate / bare, np.exp(-MU_W * PLATE_T), rtol=1e-5)   # near-axial rays


@pytest.mark.gpu
@pytest.mark.parametrize("collimator", ["none", "plate", "hole"])
def test_device_known_answer(gpu, collimator):
    torch = gpu
    ctx = sysmat.Context(_geometry(collimator))
    b = closed_form("none" if collimator == "hole" else collimator)
    out = torch.empty((1, 1), dtype=torch.float32, device="cuda")
    for mode, tol in ((sysmat.MODE_REFERENCE, 2e-6), (sysmat.MODE_PRECISE, 2e-6), (sysmat.MODE_FP64, 1e-7),
                      (sysmat.MODE_LOCAL, 2e-7)):
        ctx.pe(out, mode=mode)
        a = float(out.cpu()[0, 0])
        assert abs(a - b) <= tol * b, (mode, a, b, abs(a - b) / b)
    out_s = torch.empty((1, 1), dtype=torch.float32, device="cuda")
    ctx.pe_sampled(out_s, (4, 4, 4), (1, 1, 1))
    b4 = closed_form("none" if collimator == "hole" else collimator, div=(4, 4, 4))
    assert abs(float(out_s.cpu()[0, 0]) - b4) <= 2e-6 * b4
