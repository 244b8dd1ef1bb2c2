"""CPU tests of the host-side pieces of batching and differentiation: the parameter map theta
-> parameter arrays, the configuration 4 and 5 generators, and the batch item layout."""
import ctypes
import math

import numpy as np

from conftest import geometry, sysmat


def test_apply_theta_is_identity_at_nominal():
    geo, _, t0, _ = geometry.config5()
    g = geometry.apply_theta(geo, t0)
    assert np.array_equal(g.collimator, geo.collimator)
    assert np.array_equal(g.detector, geo.detector)


def test_apply_theta_moves_what_it_names():
    geo = geometry.mini(seed=3, layers=2)
    t = geometry.theta_of(geo)
    t2 = t + np.array([0.5, 0.01, -0.1, 0.25, -0.5, 0.125, 0.0])
    g = geometry.apply_theta(geo, t2)
    H = geo.n_holes
    h0 = geo.collimator[100:100 + 9 * H].reshape(H, 9).astype(np.float64)
    h1 = g.collimator[100:100 + 9 * H].reshape(H, 9).astype(np.float64)
    assert np.array_equal(h1[:, 0], (h0[:, 0] + 0.25).astype(np.float32))
    assert np.array_equal(h1[:, 3], (h0[:, 3] + 0.125).astype(np.float32))
    assert np.array_equal(h1[:, 1], (h0[:, 1] - 0.5).astype(np.float32))
    assert np.all(h1[:, 4] == np.float32(t2[2]))
    for m in range(2):
        assert g.collimator[(m + 1) * 10 + 5] == np.float32(t2[0])
        assert g.collimator[(m + 1) * 10 + 4] == np.float32(geo.collimator[(m + 1) * 10 + 4] - 0.5)
    d = g.detector[1:1 + 12 * geo.n_det].reshape(geo.n_det, 12)
    assert np.all(d[:, 6] == np.float32(t2[1]))
    assert np.allclose(d[:, 8], t2[1] - d[:, 7], atol=1e-7)


def test_tilt_rotates_hole_centres_about_y():
    geo = geometry.mini(seed=4)
    t = geometry.theta_of(geo)
    t[6] = math.radians(30.0)
    g = geometry.apply_theta(geo, t)
    H = geo.n_holes
    h0 = geo.collimator[100:100 + 9 * H].reshape(H, 9).astype(np.float64)
    h1 = g.collimator[100:100 + 9 * H].reshape(H, 9).astype(np.float64)
    c, s = math.cos(t[6]), math.sin(t[6])
    assert np.allclose(h1[:, 0], h0[:, 0] * c - h0[:, 3] * s, atol=1e-5)
    assert np.allclose(h1[:, 3], h0[:, 0] * s + h0[:, 3] * c, atol=1e-5)
    r0 = np.hypot(h0[:, 0], h0[:, 3])
    assert np.allclose(np.hypot(h1[:, 0], h1[:, 3]), r0, atol=1e-5)


def test_config4_instances_are_seeded_and_in_range():
    a, b = geometry.config4(8, seed=4), geometry.config4(8, seed=4)
    for ga, gb in zip(a, b):
        assert np.array_equal(ga.collimator, gb.collimator)
        m = ga.meta
        assert 0.8 <= m["hole_diameter"] <= 2.0 and 5.0 <= m["thickness"] <= 25.0
        assert 12 <= m["n_rot"] <= 60 and ga.n_rot == m["n_rot"]
        assert ga.n_det == 1024 and ga.n_vox == 32 * 32 * 16 and ga.n_holes == 1024
        assert abs(float(ga.image[7]) - 2 * math.pi / m["n_rot"]) < 1e-6


def test_config5_problem():
    geo, x, t0, ts = geometry.config5()
    assert geo.n_det == 48 * 48 and geo.n_vox == 64 * 64 * 16 and geo.n_holes == 32 * 32
    assert x.shape == (geo.n_vox,) and x.dtype == np.float32
    assert 0.0 < (x > 0).mean() < 1.0 and x.max() <= 5 * 4.0
    assert np.array_equal(ts[:3], t0[:3]) and np.all(np.abs(ts[3:6]) < 0.5)
    assert abs(ts[6]) < math.radians(1.0)


def test_batch_item_layout_matches_the_c_struct():
    # int, float, int, int, long long, long long, pointer, long long (x86-64 alignment)
    assert ctypes.sizeof(sysmat.BatchItem) == 48
    assert sysmat.BatchItem.vox_begin.offset == 16 and sysmat.BatchItem.d_out.offset == 32
