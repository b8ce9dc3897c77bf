"""The CPU oracle against the reference's own known answers (no GPU).

Unit tests restated from the reference's tests/test_solvers.cpp, tests/test_pushers.cpp and
tests/test_ab.cpp (same cases, same thresholds), and the printed numbers of its validation suite
(validation/reference_full.txt / reference_quick.txt, sections 2-4 and 7, fixtures in tests/golden)
reproduced from the same decks with the same sampled beams.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import GOLDEN, bsum_numbers, spec_from_text
from quarz_b200 import deck

VAL = json.load(open(os.path.join(GOLDEN, "validation_numbers.json")))


def _deck(name, overrides=()):
    with open(os.path.join(GOLDEN, "decks", name)) as f:
        cfg = deck.parse_deck(f.read(), overrides)
    for k in [k for k in cfg if k.startswith("output.")]:       # output settings: not part of the path
        cfg.pop(k, None)
    return deck.run_spec(cfg)


# ------------------------------------------------------------------ tests/test_solvers.cpp:34-56
@pytest.mark.parametrize("M", [16, 17, 100, 1537, 3841, 9001])
@pytest.mark.parametrize("method", ["thomas", "pcr", "partition"])
def test_tridiag_random_diagonally_dominant(M, method):
    rng = np.random.default_rng(3)
    a = rng.uniform(-1, 1, M); a[0] = 0
    c = rng.uniform(-1, 1, M); c[-1] = 0
    b = 2.5 + rng.uniform(-1, 1, M)
    x = rng.uniform(-1, 1, M)
    d = b * x
    d[1:] += a[1:] * x[:-1]
    d[:-1] += c[:-1] * x[1:]
    xs = O.tridiag(a, b, c, d, method)
    assert np.max(np.abs(xs - x)) < 1e-12


# ------------------------------------------------------------------ tests/test_solvers.cpp:58-124
def _op_errors(nodes):
    R = nodes[-1]
    r = nodes
    ex = np.exp(-r * r)
    eR = np.exp(-R * R)
    chi = 1 + r * r
    rhs = (4 * r * r - 4) * ex
    rhsB = (4 * r ** 3 - 8 * r) * ex - chi * r * ex
    rhs1 = r * ex * (4 * r * r - 8) - chi * r * (ex - eR)
    rhs2 = r * r * ex * (4 * r * r - 12) - chi * r * r * (ex - eR)
    jz = np.zeros_like(r)
    jz[-1] = (2 - 2 * R * R) * eR
    psi = O.field_solve(nodes, "L0", rhs)
    B = O.field_solve(nodes, "L1F", rhsB, chi=chi, wall=jz)
    f1 = O.field_solve(nodes, "L1D", rhs1, chi=chi)
    f2 = O.field_solve(nodes, "L2D", rhs2, chi=chi)
    return np.array([np.max(np.abs(psi - (ex - eR))), np.max(np.abs(B - r * ex)),
                     np.max(np.abs(f1 - r * (ex - eR))), np.max(np.abs(f2 - r * r * (ex - eR)))])


@pytest.mark.parametrize("stretched", [False, True])
def test_operators_second_order(stretched):
    errs = []
    for f in (1, 2, 4, 8):
        if stretched:
            nodes = O.make_regions(4.0, [(0.3, 0.01 / f), (1.5, 0.05 / f), (4.0, 0.2 / f)], 1.05 ** (1.0 / f))
        else:
            nodes = O.make_uniform(4.0, 0.04 / f)
        errs.append(_op_errors(nodes))
    order = np.log2(errs[-2] / errs[-1])
    assert np.all(order > 1.7), order


# ------------------------------------------------------------------ tests/test_solvers.cpp:126-143
def test_uniform_plasma_deposit_on_stretched_grid():
    nodes = O.make_regions(3.0, [(0.2, 0.002), (3.0, 0.05)], 1.08)
    spec = deck.RunSpec(nodes=nodes, K=2, dxi=0.01, xi_min=0.0)
    spec.species.append(deck.SpeciesSpec(name="electrons", ppc=2))
    spec.neutralize = True
    sim = O.OracleSim(spec, beams=[])
    sim.step_fields(0.0)
    ni = sim.diag()[0, :, 2]          # neutralising background = density of the freshly loaded electrons
    assert np.max(np.abs(ni[:-1] - 1.0)) < 2e-3


# ------------------------------------------------------------------ tests/test_pushers.cpp:73-86
def test_vay_force_free_drift():
    gd = 2e4
    vd = np.sqrt(1 - 1 / (gd * gd))
    Bm, dt = 60.0, 20.0
    E = np.array([vd * Bm, 0.0, 0.0])
    B = np.array([0.0, Bm, 0.0])
    u = np.array([0.0, 0.0, gd * vd])
    for _ in range(1000):
        u = O.vay(u, E, B, -0.5 * dt)
    assert abs(u[0]) < 1e-6


def test_vay_gyration_conserves_momentum():
    Bz, g = 1.0, 10.0
    uperp = np.sqrt(g * g - 1)
    T = 2 * np.pi * g / Bz
    u = np.array([uperp, 0.0, 0.0])
    for _ in range(64 * 20):
        u = O.vay(u, np.zeros(3), np.array([0.0, 0.0, Bz]), -0.5 * T / 64)
    assert abs(np.linalg.norm(u) - uperp) / uperp < 1e-12


# ------------------------------------------------------------------ tests/test_ab.cpp:13-48
def test_adams_bashforth_coefficients():
    h = 0.01
    worst = 0.0
    for p in range(1, 6):
        t = np.array([3.0 - m * h for m in range(p)] + [0.0] * (5 - p))
        u, v = O.ab_coeffs(p), O.ab_variable(p, t, h)
        worst = max(worst, np.max(np.abs(u[:p] - v[:p])))
        tn = np.array([1.0, 1.0 - h, 1.0 - 2.5 * h, 1.0 - 2.75 * h, 1.0 - 3.5 * h])
        hn = 0.7 * h
        w = O.ab_variable(p, tn, hn)
        a = [0.3, -1.2, 2.0, 0.7, -0.4]
        num = sum(hn * w[m] * sum(a[k] * tn[m] ** k for k in range(p)) for m in range(p))
        exact = sum(a[k] * ((tn[0] + hn) ** (k + 1) - tn[0] ** (k + 1)) / (k + 1) for k in range(p))
        assert abs(num - exact) / abs(exact) < 1e-11
        assert abs(sum(w[:p]) - 1) < 1e-12
    assert worst < 1e-11


# ------------------------------------------------------------------ beam generator = the reference's stream
def test_rng_matches_libstdcxx():
    g = json.load(open(os.path.join(GOLDEN, "rng_golden.json")))
    for seed in (12345, 1, 987654321):
        r = O.Rng(seed)
        assert [r.u64() for _ in range(8)] == [int(x) for x in g[f"raw_{seed}"]]
        r = O.Rng(seed)
        assert [r.normal() for _ in range(64)] == g[f"normal_{seed}"]
        r = O.Rng(seed)
        assert [r.canonical() for _ in range(16)] == g[f"uniform_{seed}"]


# ------------------------------------------------------------------ validation/reference_*.txt, section 2
@pytest.mark.parametrize("case,over", [
    ("blowout_uniform_dr0.01_dxi0.01", []),
    ("blowout_stretched_dxi0.005", ["xi.step=0.005", "grid.type=regions", "grid.regions=0.5:0.0025 2.5:0.01 8:0.05",
                                    "grid.max_ratio=1.05"]),
    ("blowout_stretched_dxi0.005_PCR", ["xi.step=0.005", "grid.type=regions",
                                        "grid.regions=0.5:0.0025 2.5:0.01 8:0.05", "grid.max_ratio=1.05",
                                        "solver.tridiag=pcr"]),
])
def test_validation_blowout(case, over):
    spec = _deck("blowout.in", ["xi.min=-10"] + over)
    sim = O.OracleSim(spec)
    sim.step_fields(0.0)
    got = bsum_numbers(spec, sim.fld())
    ref = VAL[case]
    assert f"{got['Ez(-5)']:+.4f}" == ref["Ez(-5)"]
    assert f"{got['Ez(-7)']:+.4f}" == ref["Ez(-7)"]
    assert f"{got['Ez(-8)']:+.4f}" == ref["Ez(-8)"]
    assert f"{got['Ezmin']:+.3f}" == ref["Ezmin"]
    assert f"{got['xi_min']:.3f}" == ref["xi_min"]
    assert f"{got['Wr/r']:.4f}" == ref["Wr/r"]


# ------------------------------------------------------------------ section 3 (betatron) and 4 (gain, quick)
def test_validation_betatron():
    spec = _deck("betatron.in")
    sim = O.OracleSim(spec)
    mom = sim.run(spec.steps, spec.dt)
    _, gref, xiref = sim.beam_data[0]
    t = np.arange(spec.steps + 1) * spec.dt
    rr = np.array([O.from_sums(mom[n, 0], gref, xiref)["r_rms"] for n in range(spec.steps + 1)])
    w = 1 / np.sqrt(2 * 1000)
    val = abs(rr - rr[0] * abs(np.cos(w * t))).max() / rr[0]
    assert f"{val:.2e}" == VAL["betatron_full"]


def test_validation_gain_quick():
    spec = _deck("gain.in", ["time.steps=8", "driver.nparticles=100000"])
    sim = O.OracleSim(spec)
    mom = sim.run(spec.steps, spec.dt)
    bi = [b.name for b in spec.beams].index("witness")
    _, gref, xiref = sim.beam_data[bi]
    t = np.arange(spec.steps + 1) * spec.dt
    g = np.array([O.from_sums(mom[n, bi], gref, xiref)["gamma_mean"] for n in range(spec.steps + 1)])
    assert f"{np.polyfit(t, g, 1)[0]:.4f}" == VAL["gain_quick"]


# ------------------------------------------------------------------ section 7: azimuthal mode 1
def test_validation_m1_centroid_betatron():
    # validation/run_validation.sh:101-109: betatron.in with modes = 1 and the witness offset by 0.05
    spec = _deck("betatron.in", ["modes=1", "witness.x0=0.05", "witness.nsym=4"])
    sim = O.OracleSim(spec)
    mom = sim.run(spec.steps, spec.dt)
    _, gref, xiref = sim.beam_data[0]
    t = np.arange(spec.steps + 1) * spec.dt
    d = [O.from_sums(mom[n, 0], gref, xiref, m1=True) for n in range(spec.steps + 1)]
    xc = np.array([q["x_mean"] for q in d])
    yc = np.array([q["y_mean"] for q in d])
    w = 1 / np.sqrt(2 * 1000)
    ref = VAL["m1_centroid_full"]
    assert f"{abs(xc - xc[0] * np.cos(w * t)).max() / xc[0]:.2e}" == ref["x"]
    assert f"{abs(yc).max() / xc[0]:.1e}" == ref["y"]
