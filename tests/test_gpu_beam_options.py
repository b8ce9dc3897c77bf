"""GPU parity of the beam options beyond the default path: the pushers other than Vay (<beam>.pusher =
boris | hc | imp, src/Pushers.hpp:64-95) and the per-slice beam diagnostics, through the C ABI against the
oracle on the same inputs.

- one push of config 0's driver (1e5 particles, explicit start-up kick included) with the oracle's own field
  store, for every pusher: every particle column within 1e-13 relative L2, as for Vay;
- a 10-step run with the driver pushed by Higuera-Cary and an m = 1 run with Boris, through qz_sim (which
  goes step by step for them): moments within 1e-8 of the oracle's relative to their natural scale;
- the adjoint refuses a beam whose pusher is not Vay;
- the per-slice beam sums of output.beam_slices (qz_beam_slice_sums, src/Beam.cpp:1195-1217) against the
  oracle's;
- the field file of a run (qz_sim_write_fields) against the run's own arrays."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import CONFIG0, rel_l2, spec_from_text
from quarz_b200 import workloads
from test_gpu_pipeline import _close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pusher", ["boris", "hc", "imp", "vay"])
def test_beam_push_against_oracle(pusher):
    import torch

    spec = spec_from_text(CONFIG0, [f"driver.pusher={pusher}"])
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    ref.step_fields(0.0)
    F = ref.fld()
    ref.push_beams(spec.dt, spec.dt)
    want = ref.beam(0)
    grid = Q.RadialGrid(spec.nodes)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, spec.K)
    fld = torch.from_numpy(F.reshape(-1).copy()).cuda()
    cols = torch.from_numpy(np.ascontiguousarray(beams[0][0].T)).cuda().contiguous()
    assert Q.BeamOps.push(grid, cols, -1.0, 1.0, box, fld, spec.dt, spec.dt, 0, pusher=spec.beams[0].pusher) == 1
    got = cols.cpu().numpy().T
    for c in range(7):
        assert rel_l2(got[:, c], want[:, c]) < 1e-13, (pusher, c)
    if pusher != "vay":             # the pusher matters: a Vay push of the same particles differs
        ref2 = O.OracleSim(spec_from_text(CONFIG0), beams=beams)
        ref2.step_fields(0.0)
        ref2.push_beams(spec.dt, spec.dt)
        assert rel_l2(ref2.beam(0)[:, 2], want[:, 2]) > 1e-12


def _run(spec, steps):
    beams = [Q.sample_beam(b) for b in spec.beams]
    mom_ref = O.OracleSim(spec, beams=beams).run(steps, spec.dt)
    sim = Q.Simulation(spec, beams=beams)
    mom = sim.run(steps, spec.dt)
    assert sim.schedule()["pipelined"] == 0          # non-Vay beams run step by step
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(steps + 1):
            m1 = spec.modes == 1
            _close(spec, O.from_sums(mom[n, q], gref, xiref, m1=m1), O.from_sums(mom_ref[n, q], gref, xiref, m1=m1),
                   1e-8, (q, n))


def test_run_hc_config0():
    _run(spec_from_text(CONFIG0, ["driver.pusher=hc", "driver.nparticles=20000"]), 10)


def test_run_boris_m1():
    text = workloads.hosing_deck(xi_min=-9.0, driver_np=10000, witness_np=10000, steps=3)
    _run(workloads.spec_from_text(text, ["xi.step=0.01", "pusher.beam=boris"]), 3)


def test_adjoint_refuses_other_pushers():
    spec = spec_from_text(CONFIG0, ["driver.pusher=imp", "driver.nparticles=1000"])
    with pytest.raises(Q.QZError) as e:
        Q.Simulation(spec).adjoint(1, spec.dt, np.zeros((1, 17)))
    assert e.value.code == 3


# ---------------------------------------------------------------- slice diagnostics (src/Beam.cpp:1195-1236)
def test_slice_sums_against_oracle():
    """qz_beam_slice_sums of config 0's driver (1e5 particles, 240 bins over the user xi in [-6, 0)) and of the
    sim's beams after a pipelined run of the pinched-witness deck cut to xi in [-9, 0] (beams kept in xi-cell
    order on the device): every bin's 9 sums within 1e-12 of the oracle's, relative to the bin's scale."""
    import torch

    spec = spec_from_text(CONFIG0)
    parts = Q.sample_beam(spec.beams[0])[0]
    want = O.slice_sums(parts, -6.0, 0.0, 240)
    cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
    out = torch.zeros(9 * 240, dtype=torch.float64, device="cuda")
    for _ in range(2):                                 # the output is overwritten, not accumulated
        Q.BeamOps.slice_sums(cols, -6.0, 0.0, 240, out)
    got = out.cpu().numpy().reshape(240, 9)
    scale = np.abs(want).max(axis=0) + 1e-300
    assert np.all(np.abs(got - want) <= 1e-12 * scale), np.abs(got - want).max(axis=0) / scale
    assert want[:, 0].sum() > 0.99 * parts[:, 6].sum()

    text = workloads.pinched_witness_deck(xi_min=-9.0, driver_np=20000, witness_np=20000, steps=2)
    spec = workloads.spec_from_text(text)
    beams = [Q.sample_beam(b) for b in spec.beams]
    sim = Q.Simulation(spec, beams=beams)
    sim.run(2, spec.dt)
    for b in range(2):
        want = O.slice_sums(sim.beam(b), -9.0, 0.0, 180)
        got = sim.slice_sums(b, -9.0, 0.0, 180)
        scale = np.abs(want).max(axis=0) + 1e-300
        assert np.all(np.abs(got - want) <= 1e-12 * scale), (b, np.abs(got - want).max(axis=0) / scale)
        tab = Q.slice_table(got, spec.beams[b].q, -9.0, 0.0)
        assert tab.shape[1] == 8 and len(tab) > 0


# ---------------------------------------------------------------- field files (src/Simulation.cpp:878-993)
def test_sim_write_fields(tmp_path):
    """qz_sim_write_fields after a run: the field values are those of qz_sim_fields bit for bit, and rhob (the
    beam sources the last sweep read, re-deposited from the beams as they stand) equals the oracle's beam
    deposit of the same particles to 1e-12 relative L2."""
    from test_fields_file import read_fields

    text = workloads.pinched_witness_deck(xi_min=-9.0, driver_np=20000, witness_np=20000, steps=2)
    spec = workloads.spec_from_text(text)
    beams = [Q.sample_beam(b) for b in spec.beams]
    sim = Q.Simulation(spec, beams=beams)
    sim.run(2, spec.dt)
    path = tmp_path / "fields_000002.bin"
    sim.write_fields(path, t=10.0)
    got = read_fields(path)
    F, D = sim.fields()
    np.testing.assert_array_equal(got["psi"], D[::-1, :, 0])
    np.testing.assert_array_equal(got["ez"], F[::-1, :, 4])
    np.testing.assert_array_equal(got["bth"], F[::-1, :, 3])
    ref = O.OracleSim(spec, beams=[(sim.beam(b), g, x) for b, (_, g, x) in enumerate(beams)])
    ref.deposit_beams()
    assert rel_l2(got["rhob"], ref.bsrc()[::-1, :, 4]) < 1e-12
