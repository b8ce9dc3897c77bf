"""Bit-for-bit reproducibility of the m = 0 path.

The plasma deposits of the sweep (the slice deposit, the S deposit, the background and neutralising
deposits) and the beam deposits of qz_sim runs are exact sums of integers (fixed-point quanta), so
their results do not depend on the order in which warps and CTAs add. Consequences checked here on the
full pinched-witness deck (512 stretched nodes, 2400 slices, 2 x 1e6 beam particles):

- one stand-alone sweep, run twice on the same beam sources: fields, diagnostics and the plasma state
  at the end of the box are identical (np.array_equal);
- the whole run (10 time steps), pipelined, twice from the same beams: moments of every step, the last
  fields and every particle identical; the same for the step-by-step schedule;
- the two schedules agree to rounding (the pipeline sums each warp's runs of equal cells in FP64 before
  quantising them, the step-by-step push quantises every particle's contribution): derived moments
  1e-10 relative to their natural scale, E_z / B_z and particles 1e-9, as for the cut boxes.
"""
import numpy as np
import pytest

import quarz_b200 as Q
from test_gpu_pipeline import _same
from quarz_b200 import workloads

pytestmark = pytest.mark.gpu


def test_sweep_is_bitwise_reproducible():
    import torch

    spec = workloads.pinched_witness(steps=1)
    beams = [Q.sample_beam(b) for b in spec.beams]
    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    K, M = spec.K, spec.M
    f64 = dict(dtype=torch.float64, device="cuda")
    bsrc = torch.zeros(K * M * 5, **f64)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    for b, (parts, _, _) in zip(spec.beams, beams):
        cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
        Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    out = []
    for _ in range(2):
        fld, diag = torch.zeros(K * M * 6, **f64), torch.zeros(K * M * 3, **f64)
        lost = sw.run(bsrc, fld, diag)
        torch.cuda.synchronize()
        out.append((fld.cpu().numpy(), diag.cpu().numpy(), sw.plasma(), lost))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert out[0][3] == out[1][3]


def _run(spec, beams, pipelined):
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(pipelined)
    mom = sim.run(spec.steps, spec.dt)
    assert sim.schedule()["pipelined"] == (1 if pipelined else 0)
    fld, diag = sim.fields()
    return mom, fld, diag, [sim.beam(b) for b in range(len(beams))]


@pytest.mark.parametrize("pipelined", [True, False])
def test_run_is_bitwise_reproducible(pipelined):
    spec = workloads.pinched_witness(steps=10)
    beams = [Q.sample_beam(b) for b in spec.beams]
    a = _run(spec, beams, pipelined)
    b = _run(spec, beams, pipelined)
    assert np.array_equal(a[0], b[0]), "moments"
    assert np.array_equal(a[1], b[1]), "fields"
    assert np.array_equal(a[2], b[2]), "diagnostics"
    for pa, pb in zip(a[3], b[3]):
        assert np.array_equal(pa, pb), "particles"


def test_schedules_agree():
    spec = workloads.pinched_witness(steps=4)
    beams = [Q.sample_beam(b) for b in spec.beams]
    p = _run(spec, beams, True)
    s = _run(spec, beams, False)
    _same(spec, beams, (p[0], p[1], p[3]), (s[0], s[1], s[3]))
