"""The CUDA adjoint of an m = 0 run (qz_sim_adjoint) against the oracle's adjoint on the same inputs,
and the gradients of witness energy gain and spread against central differences of the CUDA forward.

Deck: the one of tests/test_oracle_adjoint.py (24 uniform cells, 71 slices, AB3, driver and witness
with 300 particles each, 2 steps) and a stretched-grid variant with 3 steps, each also with the smoothing
filter (plasma.smooth_length 0.3 and 0.05: the adjoint then runs the filters in reverse), and both with
the nearest-slice beam shape (beams.xi_shape = ngp; the stretched one with the filter). Tolerances: every
component of the particle adjoint 1e-8 relative L2 against the oracle (the forwards differ in the
order of their deposit sums, about 1e-13); the profile and delay gradients 1e-5 relative against
central differences with h = 1e-6 (their error is that of the differences). Both schedules: the
pipelined passes (the default) and step by step."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from quarz_b200 import adjoint as A
from quarz_b200 import deck, workloads
from test_oracle_adjoint import TEXT

pytestmark = pytest.mark.gpu


def _specs():
    spec = deck.run_spec(deck.parse_deck(TEXT))
    st = deck.run_spec(deck.parse_deck(TEXT, ["time.steps=3"]))
    st.nodes = workloads.scan_nodes(129, 2e-3)
    sm = deck.run_spec(deck.parse_deck(TEXT, ["plasma.smooth_length=0.3"]))
    sms = deck.run_spec(deck.parse_deck(TEXT, ["time.steps=3", "plasma.smooth_length=0.05"]))
    sms.nodes = workloads.scan_nodes(129, 2e-3)
    ngp = deck.run_spec(deck.parse_deck(TEXT, ["beams.xi_shape=ngp"]))
    ngps = deck.run_spec(deck.parse_deck(TEXT, ["beams.xi_shape=ngp", "time.steps=3", "plasma.smooth_length=0.05"]))
    ngps.nodes = workloads.scan_nodes(129, 2e-3)
    return [spec, st, sm, sms, ngp, ngps]


@pytest.mark.parametrize("pipelined", [True, False])
@pytest.mark.parametrize("which", [0, 1, 2, 3, 4, 5])
def test_adjoint_against_oracle(which, pipelined):
    spec = _specs()[which]
    beams = [Q.sample_beam(b) for b in spec.beams]
    T, dt = spec.steps, spec.dt
    rng = np.random.default_rng(5)
    mom0 = O.OracleSim(spec, beams=beams).run(T, dt)
    seeds = rng.normal(size=(2, 17)) / (np.abs(mom0[-1]) + 1e-30)
    seeds[:, 16] = 0.0
    lam_ref, mom_ref = O.OracleSim(spec, beams=beams).adjoint(T, dt, seeds)
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(pipelined)
    lam, mom, ms = sim.adjoint(T, dt, seeds)
    assert ms[0] > 0 and ms[1] > 0
    np.testing.assert_allclose(mom, mom_ref, rtol=1e-10, atol=1e-12 * np.abs(mom_ref).max())
    for b in range(2):
        for c in range(7):
            ref = lam_ref[b][:, c]
            err = np.linalg.norm(lam[b][:, c] - ref) / max(np.linalg.norm(ref), 1e-300)
            assert err < 1e-8, (which, b, c, err)


@pytest.mark.parametrize("every", [0, 5, 71])
def test_checkpointed_adjoint_equals_full_record(every):
    # slice checkpointing (qz_sim_set_adjoint_checkpoint): the reverse sweeps push the plasma again from
    # every C-th slice (0: C = ceil(sqrt(71)) = 9; 5; 71: one segment per sweep) and reproduce the
    # forward's states, so the gradient is the one of the fully recorded trajectory (C = 1) up to the
    # summation order of the reverse pass's atomic adds
    spec = _specs()[3]
    beams = [Q.sample_beam(b) for b in spec.beams]
    T, dt = spec.steps, spec.dt
    seeds = np.random.default_rng(9).normal(size=(2, 17))
    seeds[:, 16] = 0.0
    out = []
    for c in (1, every):
        sim = Q.Simulation(spec, beams=beams)
        sim.set_adjoint_checkpoint(c)
        out.append(sim.adjoint(T, dt, seeds))
    assert np.array_equal(out[0][1], out[1][1])          # the forwards' moments
    for b in range(2):
        for c in range(7):
            ref = out[0][0][b][:, c]
            err = np.linalg.norm(out[1][0][b][:, c] - ref) / max(np.linalg.norm(ref), 1e-300)
            assert err < 1e-12, (every, b, c, err)


def test_gain_and_spread_gradients_against_differences():
    spec = _specs()[0]
    beams = [Q.sample_beam(b) for b in spec.beams]
    T, dt = spec.steps, spec.dt
    drv = spec.beams[0]
    prof = A.DriverProfile.gaussian(-drv.xi0_user, drv.sigma_xi, drv.cut, 64)
    (ds, dg, dx), (ws, wg, wx) = beams

    def run(f, shift):
        bm = [(A.driver_rows(ds, prof, f), dg, dx), (A.witness_rows(ws, shift), wg, wx)]
        sim = Q.Simulation(spec, beams=bm)
        sim.set_schedule(False)
        m = sim.run(T, dt)
        return A.gain(m[-1, 1], m[0, 1], wg), A.spread(m[-1, 1])

    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(False)
    mom = sim.run(T, dt)
    for k, seed in enumerate((A.gain_seed(mom[-1, 1]), A.spread_seed(mom[-1, 1]))):
        seeds = np.zeros((2, 17))
        seeds[1] = seed
        lam, _, _ = Q.Simulation(spec, beams=beams).adjoint(T, dt, seeds)
        gf = A.profile_gradient(lam[0], ds, prof)
        gd = A.delay_gradient(lam[1])
        for b in (26, 32, 38):
            h = 1e-6 * prof.f0[b]
            fp, fm = prof.f0.copy(), prof.f0.copy()
            fp[b] += h
            fm[b] -= h
            fd = (run(fp, 0.0)[k] - run(fm, 0.0)[k]) / (2 * h)
            assert abs(fd - gf[b]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gf).max()), (k, b, fd, gf[b])
        h = 1e-6
        fd = (run(prof.f0, h)[k] - run(prof.f0, -h)[k]) / (2 * h)
        assert abs(fd - gd) <= 1e-5 * abs(fd), (k, "delay", fd, gd)


def test_torch_function_matches_adjoint_and_differences():
    import torch

    spec = _specs()[0]
    samples = [Q.sample_beam(b) for b in spec.beams]
    drv = spec.beams[0]
    prof = A.DriverProfile.gaussian(-drv.xi0_user, drv.sigma_xi, drv.cut, 64)
    obj = A.WitnessObjective(spec, samples, prof, "gain")
    f = torch.tensor(prof.f0, dtype=torch.float64, requires_grad=True)
    d = torch.tensor(0.0, dtype=torch.float64, requires_grad=True)
    J = obj(f, d)
    (2.0 * J).backward()
    h = 1e-6
    Jp = float(obj(torch.tensor(prof.f0), torch.tensor(h)))
    Jm = float(obj(torch.tensor(prof.f0), torch.tensor(-h)))
    assert abs(float(d.grad) - 2.0 * (Jp - Jm) / (2 * h)) <= 1e-5 * abs(float(d.grad))
    b = 32
    fp, fm = prof.f0.copy(), prof.f0.copy()
    fp[b] += h * prof.f0[b]
    fm[b] -= h * prof.f0[b]
    fd = (float(obj(torch.tensor(fp), torch.tensor(0.0))) - float(obj(torch.tensor(fm), torch.tensor(0.0)))) / (
        2 * h * prof.f0[b])
    assert abs(float(f.grad[b]) - 2.0 * fd) <= 1e-5 * abs(2.0 * fd)
