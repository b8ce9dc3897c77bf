"""The oracle's adjoint of an m = 0 run (oracle/qz_oracle_adj.c) against central differences of the
oracle's own forward: the FP64 reference gradient the CUDA adjoint is checked against.

Deck: 24 uniform cells on r in [0, 6], xi in [-7, 0] with dxi 0.1 (71 slices), ppc 1, AB3, driver
(n_b 5, sigma_r 0.5, sigma_xi 1) and witness (n_b 20, sigma_r 0.2, sigma_xi 0.3, 3 behind) with 300
particles each, dt 5, 2 steps.

The deck runs as it is, with plasma.smooth_length = 0.3 (the radial smoothing filter of the plasma
sources, S+ and the background, whose transpose the adjoint applies) and with beams.xi_shape = ngp (the
nearest-slice deposit and gather, and the backward difference of rho - J_z along xi). The ngp shape is
piecewise constant in xi, so the xi direction leaves out the particles within 0.01 slices of a half-slice
boundary, which a step of +-h could move to the other slice.

Checks:
- directional derivatives of a random linear functional of the last step's moment sums along a
  random direction in each particle component of each beam: central differences with h = 1e-5 of
  the component's scale (their error is set by roundoff and the few cell crossings inside +-h), to
  2e-5 relative;
- the gradients of the witness energy gain and energy spread with respect to 3 bins of the 64-bin
  driver profile and the witness delay, against central differences with h = 1e-6 (profile bins of the
  smoothed deck: h = 1e-4 of the bin's value), to 1e-5 relative."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from quarz_b200 import adjoint as A
from quarz_b200 import deck

TEXT = """
xi.convention = z-t
grid.type = uniform
grid.rmax = 6
grid.dr = 0.25
xi.min = -7
xi.max = 0
xi.step = 0.1
time.dt = 5
time.steps = 2
plasma.species = electrons
electrons.ppc = 1
beams = driver witness
driver.n0 = 5
driver.sigma_r = 0.5
driver.sigma_xi = 1
driver.xi0 = -2
driver.gamma = 1000
driver.espread = 0.001
driver.emit_n = 0.05
driver.nparticles = 300
witness.n0 = 20
witness.sigma_r = 0.2
witness.sigma_xi = 0.3
witness.xi0 = -5
witness.gamma = 1000
witness.emit_n = 1e-2
witness.nparticles = 300
"""


@pytest.fixture(scope="module", params=["plain", "smoothed", "ngp"])
def case(request):
    over = {"plain": [], "smoothed": ["plasma.smooth_length=0.3"], "ngp": ["beams.xi_shape=ngp"]}[request.param]
    spec = deck.run_spec(deck.parse_deck(TEXT, over))
    beams = [Q.sample_beam(b) for b in spec.beams]
    return spec, beams


def _last_sums(spec, beams):
    return O.OracleSim(spec, beams=beams).run(spec.steps, spec.dt)


def test_adjoint_matches_central_differences_per_component(case):
    spec, beams = case
    T, dt = spec.steps, spec.dt
    mom0 = _last_sums(spec, beams)
    scale = np.abs(mom0[-1]) + 1e-30
    rng = np.random.default_rng(3)
    seeds = rng.normal(size=(2, 17)) / scale
    seeds[:, 16] = 0.0
    lam, mom = O.OracleSim(spec, beams=beams).adjoint(T, dt, seeds)
    np.testing.assert_array_equal(mom, mom0)          # the adjoint's forward is the plain forward
    for b in range(2):
        for c in range(7):
            d = rng.normal(size=len(beams[b][0]))
            h = 1e-5 * (np.abs(beams[b][0][:, c]).mean() + 1e-3)
            if spec.ngp and c == 5:
                sl = (beams[b][0][:, 5] - spec.xi_min) / spec.dxi + 0.5
                d[np.abs(sl - np.rint(sl)) < 0.01] = 0.0

            def J(sign):
                rows = [bm[0].copy() for bm in beams]
                rows[b][:, c] += sign * h * d
                m = _last_sums(spec, [(rows[q], beams[q][1], beams[q][2]) for q in range(2)])
                return float(np.sum(seeds * m[-1]))

            fd = (J(1) - J(-1)) / (2 * h)
            ad = float(lam[b][:, c] @ d)
            assert abs(fd - ad) <= 2e-5 * abs(fd), (b, c, fd, ad)


def test_profile_and_delay_gradients(case):
    spec, beams = case
    T, dt = spec.steps, spec.dt
    drv, wit = spec.beams
    prof = A.DriverProfile.gaussian(-drv.xi0_user, drv.sigma_xi, drv.cut, 64)
    (ds, dg, dx), (ws, wg, wx) = beams

    def run(f, shift):
        bm = [(A.driver_rows(ds, prof, f), dg, dx), (A.witness_rows(ws, shift), wg, wx)]
        m = _last_sums(spec, bm)
        return A.gain(m[-1, 1], m[0, 1], wg), A.spread(m[-1, 1])

    mom = _last_sums(spec, beams)
    for name, seed in (("gain", A.gain_seed(mom[-1, 1])), ("spread", A.spread_seed(mom[-1, 1]))):
        seeds = np.zeros((2, 17))
        seeds[1] = seed
        lam, _ = O.OracleSim(spec, beams=beams).adjoint(T, dt, seeds)
        gf = A.profile_gradient(lam[0], ds, prof)
        gd = A.delay_gradient(lam[1])
        k = 0 if name == "gain" else 1
        for b in (26, 32, 38):
            # smoothed: h = 1e-4 f0 (at 1e-6 f0 the quotient of bin 26, whose gradient is 3e-3 of the largest,
            # is round-off; at 1e-3 .. 1e-5 f0 it agrees with the adjoint to 3e-9 .. 7e-7)
            h = (1e-4 if spec.smooth_length > 0 else 1e-6) * prof.f0[b]
            fp, fm = prof.f0.copy(), prof.f0.copy()
            fp[b] += h
            fm[b] -= h
            fd = (run(fp, 0.0)[k] - run(fm, 0.0)[k]) / (2 * h)
            assert abs(fd - gf[b]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gf).max()), (name, b, fd, gf[b])
        h = 1e-6
        fd = (run(prof.f0, h)[k] - run(prof.f0, -h)[k]) / (2 * h)
        assert abs(fd - gd) <= 1e-5 * abs(fd), (name, "delay", fd, gd)
