"""The float64 Ewald restatement (oracle/ewald.py) behind the periodic force
law: independent of the splitting parameter, periodic, odd, zero normal
component on the box faces, and d/|d|^3 - (4 pi/3) d + O(|d|^3) near d = 0."""
import math

import numpy as np

from oracle import ewald as E


def test_independent_of_splitting():
    d = np.random.default_rng(0).uniform(-0.5, 0.5, (40, 3))
    np.testing.assert_allclose(E.f_per(d, 2.0), E.f_per(d, 2.7), rtol=0, atol=1e-11)


def test_periodic_and_odd():
    d = np.random.default_rng(1).uniform(-0.5, 0.5, (40, 3))
    f = E.f_per(d)
    for shift in ([1, 0, 0], [0, -1, 0], [1, 1, -1]):
        np.testing.assert_allclose(E.f_per(d + np.array(shift)), f, atol=1e-10)
    np.testing.assert_allclose(E.f_per(-d), -f, atol=1e-12)


def test_face_and_corner_symmetry():
    # on the face d_x = 1/2 the x component vanishes (periodic and odd)
    d = np.random.default_rng(2).uniform(-0.5, 0.5, (20, 3))
    d[:, 0] = 0.5
    assert np.abs(E.f_per(d)[:, 0]).max() < 1e-12
    assert np.abs(E.f_per(np.array([[0.5, 0.5, 0.5]]))).max() < 1e-12


def test_small_distance_expansion():
    for r in (1e-3, 1e-2):
        d = np.array([[r, 0.3 * r, -0.2 * r]])
        corr = E.f_per(d)[0] - d[0] / np.linalg.norm(d[0]) ** 3
        np.testing.assert_allclose(corr / d[0], -4 * math.pi / 3, rtol=3e-3 if r > 5e-3 else 1e-4)
    # g is O(|d|^3)
    for r in (0.05, 0.1, 0.2):
        g = E.g_corr(np.array([[r, 0.5 * r, 0.25 * r]]))
        assert 5 < np.linalg.norm(g) / r ** 3 < 20


def test_direct_sum_is_periodic_in_the_target():
    rng = np.random.default_rng(3)
    p = rng.random((64, 3))
    m = np.full(64, 1 / 64)
    a = E.direct_sum_ewald(p[:, 0], p[:, 1], p[:, 2], m, [5], 1.0, 0.01)
    q = p.copy()
    q[:, 1] = (q[:, 1] + 0.37) % 1.0     # the whole system translated
    b = E.direct_sum_ewald(q[:, 0], q[:, 1], q[:, 2], m, [5], 1.0, 0.01)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12)
