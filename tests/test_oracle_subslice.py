"""The oracle's adaptive sub-slicing (pusher.max_cells_per_step; src/Simulation.cpp:755-781, :837-847,
src/PlasmaSpecies.cpp:814-830, variable-step Adams-Bashforth :30-48, :561-580) against the reference's
validation section 13 (validation/run_validation.sh:264-281): the paper case conv_s1 (pinched witness
with mobile ions, analytic driver and witness, axis cell 5e-4, ppc 4) in a box to xi = -12 with
dxi = 0.01. The reference prints the number of extra sub-slices of that sweep, 1642 with
max_cells_per_step = 1 and none without; the count follows every sub-slice decision (the cells-crossed
estimate, the doubling rule, the variable-step pushes after a sub-sliced step), so it pins them all.

It also prints, for the runs with and without sub-slicing (validation/subslice_check.py), the relative
r.m.s. errors of E_z and psi on the axis behind the closure spike (s = -xi in [9.2, 11.9]) and around the
witness ([6.4, 7.2]) against a fine-step run (dxi = 0.0025 quick, 0.000625 full), and the integral of E_z
over the spike ([8.9, 9.2]) of all three runs. Those are restated here on the oracle's axis values and
agree to every printed digit, full and quick. The check reads xi back from the axis file, written with
ten significant digits (Simulation::write_axis, src/Simulation.cpp:995-1029): rounded the same way here,
the slice at s = 9.2 lies inside the spike's window as it does there."""
import numpy as np

import oracle as O
from helpers import user_xi
from test_oracle_pins import VAL, _deck

CONV = ["xi.min=-12", "xi.step=0.01"]


def _axis(extra):
    """(s, E_z(0), psi(0)) of one sweep of the box to xi = -12, head first, s as the axis file gives it."""
    spec = _deck("conv_s1.in", ["xi.min=-12"] + extra)
    sim = O.OracleSim(spec)
    sim.step_fields(0.0)
    s = -np.array([float(f"{x:+.10e}") for x in user_xi(spec)])
    return s[::-1], sim.fld()[:, 0, 4], sim.diag()[:, 0, 0], sim.subslices()


def _rms(a, b, lo, hi, c):
    xs = np.arange(lo, hi, 0.005)
    r0, r1 = np.interp(xs, a[0], a[c]), np.interp(xs, b[0], b[c])
    return np.sqrt(np.mean((r1 - r0) ** 2) / np.mean(r0 ** 2))


def _spike(a):
    m = (a[0] >= 8.9) & (a[0] <= 9.2)
    return np.trapezoid(a[1][m], a[0][m])


def test_validation_subslice_errors_and_spike():
    runs = {"plain": _axis(["xi.step=0.01"]), "sub": _axis(["xi.step=0.01", "pusher.max_cells_per_step=1"])}
    assert runs["sub"][3] == 1642 and runs["plain"][3] == 0
    for tag, dref in (("quick", 0.0025), ("full", 0.000625)):
        ref = _axis([f"xi.step={dref}"])
        assert f"{_spike(ref):.3f}" == VAL[f"subslice_ref_{tag}"]["spike"], tag
        for name, a in runs.items():
            want = VAL[f"subslice_{name}_{tag}"]
            got = {"behind Ez": _rms(ref, a, 9.2, 11.9, 1), "behind psi": _rms(ref, a, 9.2, 11.9, 2),
                   "witness Ez": _rms(ref, a, 6.4, 7.2, 1), "witness psi": _rms(ref, a, 6.4, 7.2, 2)}
            for key, v in got.items():
                assert f"{v:.1e}" == want[key], (tag, name, key, v)
            assert f"{_spike(a):.3f}" == want["spike"], (tag, name)


def test_validation_subslice_count():
    for key, extra in (("subslice_sub_full", ["pusher.max_cells_per_step=1"]), ("subslice_plain_full", [])):
        spec = _deck("conv_s1.in", CONV + extra)
        assert spec.K == 1201
        sim = O.OracleSim(spec)
        sim.step_fields(0.0)
        assert sim.subslices() == int(VAL[key]["extra"]), key
        assert VAL[key.replace("full", "quick")]["extra"] == VAL[key]["extra"]


def test_subslicing_off_below_the_threshold():
    # a threshold above every particle's cells crossed: the same fields bit for bit as without sub-slicing
    spec = _deck("conv_s1.in", ["xi.min=-4", "xi.step=0.01"])
    a = O.OracleSim(spec)
    a.step_fields(0.0)
    spec2 = _deck("conv_s1.in", ["xi.min=-4", "xi.step=0.01", "pusher.max_cells_per_step=1e6"])
    b = O.OracleSim(spec2)
    b.step_fields(0.0)
    assert b.subslices() == 0
    assert np.array_equal(a.fld(), b.fld()) and np.array_equal(a.diag(), b.diag())
