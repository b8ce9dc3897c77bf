"""The oracle's beam pushers other than Vay (<beam>.pusher = boris | hc | imp, src/Pushers.hpp:54-95), pinned
by the checks of the reference's tests/test_pushers.cpp:
  1. algebraic identity (test_pushers.cpp:29-50): the implicit midpoint push (note eqs. 19-36) equals
     Higuera-Cary to 1e-12 relative to 1 + |u| + 2 eps (|E| + |B|), on random u, E, B, eps spanning
     many decades (1e5 samples here; 1e6 there);
  2. force-free particle (test_pushers.cpp:69-82): E = v_d B with gamma_d = 2e4, B = 60, dt = 20; after
     1000 steps the spurious transverse momentum stays below 1e-6 for Vay, HC and IMP (Boris is not
     force-free, as the reference prints);
  3. gyration in a uniform B (test_pushers.cpp:52-67, gamma = 10, 64 steps per period, 100 periods): every
     pusher keeps |u| to round-off;
and kind 0 is the Vay push of qzo_vay."""
import numpy as np
import pytest

import oracle as O

KINDS = {"vay": 0, "boris": 1, "hc": 2, "imp": 3}


def test_imp_equals_higuera_cary():
    rng = np.random.default_rng(7)
    n = 100000
    su = 10.0 ** rng.uniform(-3, 6, n)
    sf = 10.0 ** (rng.uniform(-3, 6, n) - 2)
    u = su[:, None] * rng.uniform(-1, 1, (n, 3))
    E = sf[:, None] * rng.uniform(-1, 1, (n, 3))
    B = sf[:, None] * rng.uniform(-1, 1, (n, 3))
    eps = 0.5 * 10.0 ** (rng.uniform(-3, 6, n) - 3)
    a = O.push(KINDS["imp"], u, E, B, eps)
    b = O.push(KINDS["hc"], u, E, B, eps)
    sc = 1.0 + np.linalg.norm(u, axis=1) + 2 * eps * (np.linalg.norm(E, axis=1) + np.linalg.norm(B, axis=1))
    assert (np.linalg.norm(a - b, axis=1) / sc).max() < 1e-12


def test_kind_zero_is_vay():
    rng = np.random.default_rng(3)
    for _ in range(50):
        u, E, B = rng.normal(size=3) * 100, rng.normal(size=3), rng.normal(size=3)
        want = O.vay(u, E, B, 0.3)
        np.testing.assert_array_equal(O.push(0, u, E, B, 0.3)[0], want)


@pytest.mark.parametrize("kind", ["vay", "hc", "imp", "boris"])
def test_force_free_drift(kind):
    gd, Bm, dt = 2e4, 60.0, 20.0
    vd = np.sqrt(1 - 1 / gd ** 2)
    E, B = np.array([vd * Bm, 0, 0]), np.array([0, Bm, 0])
    u = np.array([[0.0, 0.0, gd * vd]])
    for _ in range(1000):
        u = O.push(KINDS[kind], u, E, B, -0.5 * dt)
    if kind == "boris":
        assert abs(u[0, 0]) > 1e-6          # Boris is not force-free here (the reference prints it, unchecked)
    else:
        assert abs(u[0, 0]) < 1e-6, (kind, u)


@pytest.mark.parametrize("kind", list(KINDS))
def test_gyration_keeps_momentum(kind):
    Bz, g = 1.0, 10.0
    up = np.sqrt(g * g - 1)
    dt = 2 * np.pi / (Bz / g) / 64
    u = np.array([[up, 0.0, 0.0]])
    for _ in range(64 * 100):
        u = O.push(KINDS[kind], u, np.zeros(3), np.array([0, 0, Bz]), -0.5 * dt)
    assert abs(np.linalg.norm(u) - up) / up < 1e-11, kind
