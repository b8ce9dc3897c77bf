"""The pipelined run against the step-by-step run and the oracle.

The pipelined qz_sim_run puts all sweeps and pushes of a run into ONE cooperative launch: sweeps of
consecutive time steps run concurrently on different SMs, each slice waiting for the beam pushes of
the previous step that can deposit into it. The arithmetic is that of the step-by-step run (one sweep
launch, then one push launch per beam, per step); only the order in which beam deposits are summed
differs. Tolerances against the step-by-step run: derived beam moments 1e-10 relative (to their
natural scale, see _scale), E_z / B_z 1e-9 relative L2 and particles 1e-9 (the round-off of the
deposit order carried through the sweeps)."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import CONFIG0, config1_deck, rel_l2, spec_from_text

pytestmark = pytest.mark.gpu

MOM_TOL = 1e-10
FLD_TOL = 1e-9
KEYS = ("gamma_mean", "gamma_rms", "xi_mean", "xi_rms", "r_rms", "emit_nx", "charge_w", "alive")


def _scale(spec, d):
    """Absolute floor of each derived quantity: the tolerance is relative to max(|value|, scale), so that
    a spread that is itself pure round-off (a beam without energy spread has gamma_rms ~ 1e-13) is
    compared on the scale of the quantity it is the spread of."""
    L = spec.K * spec.dxi
    R = spec.nodes[-1]
    return {"gamma_mean": 0.0, "gamma_rms": abs(d["gamma_mean"]), "xi_mean": L, "xi_rms": L, "r_rms": R,
            "emit_nx": 0.0, "charge_w": 0.0, "alive": 0.0}


def _close(spec, d, dr, tol, where):
    sc = _scale(spec, dr)
    for k in KEYS:
        assert abs(d[k] - dr[k]) <= tol * max(abs(dr[k]), sc[k], 1e-300), (where, k, d[k], dr[k])


def _spec(name, steps):
    if name == "config0":
        spec = spec_from_text(CONFIG0, [f"time.steps={steps}"])
    else:   # the stretched 512-node grid with driver + witness, box cut to xi in [-9, 0]
        spec = spec_from_text(config1_deck(xi_min=-9.0, driver_np=40000, witness_np=40000, steps=steps))
    return spec, [Q.sample_beam(b) for b in spec.beams]


def _run(spec, beams, steps, pipelined=True, **sched):
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(pipelined, **sched)
    mom = sim.run(steps, spec.dt)
    info = sim.schedule()
    assert info["pipelined"] == (1 if pipelined else 0), info
    fld, _ = sim.fields()
    parts = [sim.beam(b) for b in range(len(spec.beams))]
    return mom, fld, parts, info


def _same(spec, beams, a, b, mtol=MOM_TOL, ftol=FLD_TOL):
    mom_a, fld_a, parts_a = a[:3]
    mom_b, fld_b, parts_b = b[:3]
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(mom_a.shape[0]):
            da, db = O.from_sums(mom_a[n, q], gref, xiref), O.from_sums(mom_b[n, q], gref, xiref)
            _close(spec, da, db, mtol, (q, n))
    for c in (4, 5):
        assert rel_l2(fld_a[..., c], fld_b[..., c]) < ftol, c
    for pa, pb in zip(parts_a, parts_b):
        assert np.array_equal(pa[:, 6] == 0, pb[:, 6] == 0)
        for c in range(6):
            assert rel_l2(pa[:, c], pb[:, c]) < ftol, c


@pytest.mark.parametrize("name,steps", [("config0", 6), ("config1", 4)])
def test_pipelined_equals_step_by_step(name, steps):
    spec, beams = _spec(name, steps)
    seq = _run(spec, beams, steps, pipelined=False)
    pip = _run(spec, beams, steps)
    assert pip[3]["sweep_ctas"] == steps + 1 and pip[3]["buckets"] > 10
    _same(spec, beams, pip, seq)


@pytest.mark.parametrize("sched", [{"sweep_ctas": 1}, {"sweep_ctas": 2, "bucket": 97}, {"bucket": 4096}])
def test_pipeline_schedules(sched):
    # fewer sweep CTAs than steps (a CTA runs several sweeps in turn), odd and large buckets
    spec, beams = _spec("config0", 5)
    seq = _run(spec, beams, 5, pipelined=False)
    pip = _run(spec, beams, 5, **sched)
    if "sweep_ctas" in sched:
        assert pip[3]["sweep_ctas"] == sched["sweep_ctas"]
    _same(spec, beams, pip, seq)


def test_pipelined_run_against_oracle():
    spec, beams = _spec("config1", 3)
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(3, spec.dt)
    mom, fld, parts, _ = _run(spec, beams, 3)
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(4):
            d, dr = O.from_sums(mom[n, q], gref, xiref), O.from_sums(mom_ref[n, q], gref, xiref)
            _close(spec, d, dr, 1e-8, (q, n))
    F = ref.fld()
    for c in (4, 5):
        assert rel_l2(fld[..., c], F[..., c]) < 1e-8, c
    for q in range(len(beams)):
        got, want = parts[q], ref.beam(q)
        for c in range(6):
            assert rel_l2(got[:, c], want[:, c]) < 1e-9, (q, c)


def test_run_host_keeps_caller_order():
    spec, beams = _spec("config0", 3)
    sim = Q.Simulation(spec, beams=beams)
    cols = [np.ascontiguousarray(p.T) for p, _, _ in beams]
    mom_h = sim.run_host(3, spec.dt, cols)
    seq = _run(spec, beams, 3, pipelined=False)
    for q in range(len(beams)):
        got = cols[q].T
        for c in range(6):
            assert rel_l2(got[:, c], seq[2][q][:, c]) < FLD_TOL, c
        # and the device copy is back in the caller's order too
        assert np.array_equal(sim.beam(q), got)
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(4):
            _close(spec, O.from_sums(mom_h[n, q], gref, xiref), O.from_sums(seq[0][n, q], gref, xiref), MOM_TOL,
                   (q, n))


def test_pipeline_wait_limit_reports_error_and_device_stays_usable():
    # every wait inside the pipelined launch is bounded; with a limit of 100 ns the first wait that is
    # not satisfied at once gives up, the launch ends, and the host gets an error (no hang, no fault)
    spec, beams = _spec("config0", 3)
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(True, timeout_s=1e-7)
    with pytest.raises(Q.QZError) as e:
        sim.run(3, spec.dt)
    assert "timed out" in str(e.value)
    # the same device and a fresh simulation afterwards: correct results
    seq = _run(spec, beams, 3, pipelined=False)
    pip = _run(spec, beams, 3)
    _same(spec, beams, pip, seq)
