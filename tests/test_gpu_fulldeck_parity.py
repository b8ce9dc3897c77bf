"""GPU parity on the benchmarked decks at their full sizes, against the serial CPU oracle.

The serial oracle finishes a full pinched-witness sweep (512 stretched nodes, 2400 slices) in about
0.6 s and a push of 2 x 1e6 beam particles in about 0.5 s; the hosing sweep (modes 0, 1, 8 azimuths,
4088 plasma particles per slice) takes about 5 s. So the bars are checked on the decks the bench
numbers come from, not only on cut boxes.

- Pinched witness (512 stretched nodes, 2400 slices, dxi 0.005, 1e6 driver + 1e6 witness particles):
  (a) the beam sources of the initial beams 1e-12 relative L2 per component; one sweep: every stored
      field and diagnostic within 1e-10 relative L2, raised to 4x the reference algorithm's own
      round-off floor where that is higher (the difference between its Thomas and partition
      tridiagonal solvers on the same input, computed here and printed). On this deck the plasma
      electrons cross the axis where the bubble closes behind the witness (xi < -9, slices >= 1800),
      and round-off differences of 1e-16 grow there by six orders: the reference's own partition
      solver differs from its Thomas solver by 1.5e-10 (psi) and 2.2e-10 (E_z) over the whole box.
      Ahead of that point (xi in (-9, 0], slices < 1800) psi, E_z and B_z must meet 1e-10 outright,
      relative to the whole component's norm; over the whole box they meet the floor rule;
  (b) 10 time steps through the pipelined run: derived beam moments of every step within 1e-8
      relative to their natural scale; E_z, B_z after the last sweep 1e-8 relative L2.
- Hosing (the same grid and box with modes 0, 1, Picard 3, 8 azimuths, 2e6 + 2e6 particles):
  one sweep at the same field bar; 3 pipelined time steps with moments at 1e-8 (the oracle needs
  about 30 s for them); E_z, B_z of modes 0 and 1 after the last sweep 1e-8.
"""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import rel_l2
from quarz_b200 import workloads
from test_gpu_m1 import KEYS as KEYS_M1
from test_gpu_m1 import _gpu_sweep as _gpu_sweep_m1
from test_gpu_parity import _floor, _gpu_sweep
from test_gpu_pipeline import _close

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10
MOMENT_TOL = 1e-8
AHEAD_OF_CLOSURE = 1800     # slices of xi in (-9, 0]: ahead of where the bubble closes behind the witness


def test_pinched_witness_full_deck_one_sweep():
    spec = workloads.pinched_witness(steps=10)
    assert (spec.K, spec.M) == (2400, 512)
    beams = [Q.sample_beam(b) for b in spec.beams]
    assert sum(len(b[0]) for b in beams) == 2000000
    ref, floor = _floor(spec, beams)
    bs, fld, diag, lost, sw = _gpu_sweep(spec, beams)
    for c in range(5):
        assert rel_l2(bs[..., c], ref.bsrc()[..., c]) < 1e-12, f"bsrc comp {c}"
    F, D = ref.fld(), ref.diag()
    got = {f"fld{c}": fld[..., c] for c in range(6)}
    got.update({f"diag{c}": diag[..., c] for c in range(3)})
    want = {f"fld{c}": F[..., c] for c in range(6)}
    want.update({f"diag{c}": D[..., c] for c in range(3)})
    errs = {k: rel_l2(got[k], want[k]) for k in got if np.any(want[k])}
    print("pinched witness, one sweep (error / reference floor):",
          {k: f"{v:.2e}/{floor[k]:.2e}" for k, v in errs.items()})
    bad = {k: (v, floor[k]) for k, v in errs.items() if not v < max(FIELD_TOL, 4.0 * floor[k])}
    assert not bad, f"field mismatch {bad}"
    ahead = slice(0, AHEAD_OF_CLOSURE)
    for k in ("diag0", "fld4", "fld5"):            # psi, E_z, B_z ahead of the bubble closure
        e = np.linalg.norm(got[k][ahead] - want[k][ahead]) / np.linalg.norm(want[k])
        print(f"{k} ahead of the closure: {e:.2e}")
        assert e < FIELD_TOL, (k, e)
    assert lost == ref.lost()


def test_pinched_witness_full_deck_10_pipelined_steps():
    spec = workloads.pinched_witness(steps=10)
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(spec.steps, spec.dt)
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(True)
    mom = sim.run(spec.steps, spec.dt)
    assert sim.schedule()["pipelined"] == 1
    worst = 0.0
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(spec.steps + 1):
            d, dr = O.from_sums(mom[n, q], gref, xiref), O.from_sums(mom_ref[n, q], gref, xiref)
            _close(spec, d, dr, MOMENT_TOL, (q, n))
            worst = max(worst, max(abs(d[k] - dr[k]) / max(abs(dr[k]), 1e-300) for k in ("gamma_mean", "charge_w")))
    fld, _ = sim.fields()
    F = ref.fld()
    for c in (4, 5):
        assert rel_l2(fld[..., c], F[..., c]) < 1e-8, c
    print(f"pinched witness, 10 pipelined steps: worst relative <gamma> / charge difference {worst:.2e}")


def test_hosing_full_deck_one_sweep():
    spec = workloads.hosing(steps=3)
    assert (spec.K, spec.M, spec.modes) == (2400, 512, 1)
    beams = [Q.sample_beam(b) for b in spec.beams]
    a = O.OracleSim(spec, beams=beams, tridiag="thomas")
    a.step_fields(0.0)
    b = O.OracleSim(spec, beams=beams, tridiag="partition")
    b.step_fields(0.0)
    bs, fld, diag, lost = _gpu_sweep_m1(spec, beams)
    B = a.bsrc()
    for c in range(15):
        if np.any(B[..., c]):
            assert rel_l2(bs[..., c], B[..., c]) < 1e-12, f"bsrc comp {c}"
    errs, bad = {}, {}
    for name, got, ra, rb, nc in (("fld", fld, a.fld(), b.fld(), 18), ("diag", diag, a.diag(), b.diag(), 9)):
        for c in range(nc):
            if not np.any(ra[..., c]):
                assert not np.any(got[..., c]), (name, c)
                continue
            e = rel_l2(got[..., c], ra[..., c])
            floor = rel_l2(rb[..., c], ra[..., c])
            errs[f"{name}{c}"] = (e, floor)
            if not e < max(FIELD_TOL, 4.0 * floor):
                bad[f"{name}{c}"] = (e, floor)
    assert not bad, f"hosing field mismatch {bad}; all {errs}"
    for k in ("diag0", "fld4", "fld5"):         # psi, E_z, B_z of mode 0
        assert errs[k][0] < FIELD_TOL, (k, errs[k])
    assert lost == a.lost()
    print("hosing, one sweep (error, floor):", {k: f"{e:.1e}/{f:.1e}" for k, (e, f) in errs.items()})


def test_hosing_full_deck_3_pipelined_steps():
    spec = workloads.hosing(steps=3)
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(spec.steps, spec.dt)
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(True)
    mom = sim.run(spec.steps, spec.dt)
    assert sim.schedule()["pipelined"] == 1
    L, R = spec.K * spec.dxi, spec.nodes[-1]
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(spec.steps + 1):
            d = O.from_sums(mom[n, q], gref, xiref, m1=True)
            dr = O.from_sums(mom_ref[n, q], gref, xiref, m1=True)
            scale = {"gamma_rms": abs(dr["gamma_mean"]), "xi_mean": L, "xi_rms": L, "x_mean": R, "y_mean": R,
                     "sigma_x": R}
            for k in KEYS_M1:
                tol = MOMENT_TOL * max(abs(dr[k]), scale.get(k, 0.0), 1e-300)
                assert abs(d[k] - dr[k]) <= tol, (q, n, k, d[k], dr[k])
    fld, _ = sim.fields()
    F = ref.fld()
    for c in (4, 5, 14, 15):
        assert rel_l2(fld[..., c], F[..., c]) < 1e-8, c
