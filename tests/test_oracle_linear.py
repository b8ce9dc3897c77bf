"""The CPU oracle against the reference's validation sections 1 (linear wake against its Green's
function) and 4 (witness energy gain, the full-length run), printed in validation/reference_full.txt
and reference_quick.txt (fixtures in tests/golden/validation_numbers.json).

Section 1 (validation/run_validation.sh:24-31, the comparison of validation/check_linear.py): a weak
Gaussian driver (n_b = 0.001) in a conducting cylinder. Linear theory gives the density response
dn(r, s) = rho_b(r) Int sin(s - s') f(s') ds' (s = distance behind the box head) and the wake
potential psi = -Int r' G(r, r') dn(r') dr' with the Green's function of (lap_perp - 1) under
psi(R) = 0: G = I0(r<) [K0(r>) - K0(R) I0(r>) / I0(R)]; E_z = d psi / ds, E_r - B_theta = -d psi / dr.
The printed numbers are the maximum errors of E_z and psi on the axis and of E_r - B_theta at r = 0.5,
relative to the analytic maxima, on the uniform grid (dr 0.01) and on a stretched one (0.002 -> 0.05).
The analytic side uses the same quadratures as the reference's check (trapezoid on 4001 radial
points, a Riemann sum on 4001 points across the truncated Gaussian), so that the printed four digits
are comparable.

Section 4 (run_validation.sh:59-67): the witness's mean energy gain rate in the rigid-driver
blowout over 20 steps with 5e5 driver particles, d<gamma>/dt = 0.4477.
"""
import numpy as np
import pytest
from scipy.special import i0e, k0e

import oracle as O
from helpers import user_xi
from test_oracle_pins import VAL, _deck


def linear_wake_numbers(spec, fld, diag, nb, sr=0.5, sx=1.0, s0=4.0, cut=4.0):
    """(max|E_z|, rel. err E_z(r=0), rel. err psi(0), rel. err (E_r - B_theta)(r=0.5)) of the fields
    of one sweep against the linear wake of the truncated Gaussian driver."""
    r = spec.nodes
    R = r[-1]
    s = -user_xi(spec)                          # distance behind the head, rows in file order
    ez = fld[::-1, :, 4]
    wr = fld[::-1, :, 0] - fld[::-1, :, 3]
    psi = diag[::-1, :, 0]
    rq = np.linspace(0.0, R, 4001)
    wq = np.full(rq.shape, rq[1] - rq[0])
    wq[0] *= 0.5
    wq[-1] *= 0.5
    prof_r = np.where(rq <= cut * sr, np.exp(-rq ** 2 / (2 * sr ** 2)), 0.0)
    sg = np.linspace(s0 - cut * sx, s0 + cut * sx, 4001)
    fg = np.exp(-(sg - s0) ** 2 / (2 * sx ** 2))
    dsg = sg[1] - sg[0]

    def along(kernel):
        return np.array([np.sum(np.where(sg <= x, kernel(x - sg), 0.0) * fg) * dsg for x in s])

    dn_s, ddn_s = along(np.sin), along(np.cos)
    lo = np.minimum(r[:, None], rq[None, :])
    hi = np.maximum(r[:, None], rq[None, :])
    # exponentially scaled Bessel functions keep every factor finite: I0(a) = i0e(a) e^a, K0(a) = k0e(a) e^-a
    with np.errstate(invalid="ignore", over="ignore"):      # K0(0) is infinite; its column has weight 0
        g = i0e(lo) * np.exp(lo - hi) * k0e(hi) - i0e(lo) * i0e(hi) * k0e(R) / i0e(R) * np.exp(lo + hi - 2 * R)
        g = np.nan_to_num(g * (rq * wq)[None, :], nan=0.0, posinf=0.0)
    psi_r = -g @ (-nb * prof_r)                # electron driver: rho_b = -n_b exp(-r^2 / 2 sr^2)
    ez_ref = np.outer(ddn_s, psi_r)
    psi_ref = np.outer(dn_s, psi_r)
    wr_ref = -np.outer(dn_s, np.gradient(psi_r, r))
    ir = int(np.argmin(abs(r - 0.5)))
    amp = abs(ez_ref[:, 0]).max()
    return (amp, abs(ez[:, 0] - ez_ref[:, 0]).max() / amp,
            abs(psi[:, 0] - psi_ref[:, 0]).max() / abs(psi_ref[:, 0]).max(),
            abs(wr[:, ir] - wr_ref[:, ir]).max() / abs(wr_ref[:, ir]).max())


LINEAR_DECKS = {
    "uniform": ["driver.n0=0.001"],
    "stretched": ["driver.n0=0.001", "grid.type=regions", "grid.regions=0.3:0.002 2:0.02 8:0.05",
                  "grid.max_ratio=1.05"],
}


def check_linear(name, fld, diag, spec):
    amp, e_ez, e_psi, e_wr = linear_wake_numbers(spec, fld, diag, 0.001)
    want = VAL[f"linear_{name}_full"]
    assert VAL[f"linear_{name}_quick"] == want
    assert f"{amp:.4e}" == want["max|Ez|"]
    assert f"{e_ez:.3e}" == want["rel.err Ez(r=0)"]
    assert f"{e_psi:.3e}" == want["psi(0)"]
    assert f"{e_wr:.3e}" == want["(Er-Bth)(r=0.5)"]


@pytest.mark.parametrize("name", ["uniform", "stretched"])
def test_validation_linear_wake(name):
    spec = _deck("linear.in", LINEAR_DECKS[name])
    sim = O.OracleSim(spec)
    sim.step_fields(0.0)
    check_linear(name, sim.fld(), sim.diag(), spec)


def test_validation_gain_full():
    spec = _deck("gain.in")
    assert spec.steps == 20 and spec.beams[0].nparticles == 500000
    sim = O.OracleSim(spec)
    mom = sim.run(spec.steps, spec.dt)
    bi = [b.name for b in spec.beams].index("witness")
    _, gref, xiref = sim.beam_data[bi]
    t = np.arange(spec.steps + 1) * spec.dt
    g = np.array([O.from_sums(mom[n, bi], gref, xiref)["gamma_mean"] for n in range(spec.steps + 1)])
    assert f"{np.polyfit(t, g, 1)[0]:.4f}" == VAL["gain_full"]
