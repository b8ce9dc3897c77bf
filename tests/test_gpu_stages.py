"""The xi-pipelined run (the reference's multi-rank mode) on one GPU: slabs of the box run one after
the other through qz_sweep_run_stage, each taking the plasma state and the guard row of the slab ahead.

- One sweep cut into 2 and 3 slabs equals the whole-box sweep bit for bit (np.array_equal): fields,
  diagnostics, the plasma at the end of the box and the removal count. This is the reference's claim for
  its pipelined MPI run with the ngp xi shape (README.md:1755-1758); here it holds because the sweep's
  plasma deposits are exact sums. Checked on the pinched-witness deck with beams.xi_shape = ngp, cut box
  and full box.
- A staged run of 5 time steps (quarz_b200.stages, stages run in turn in one process) with exact beam
  sources (qz_beam_deposit_fx with the quanta the single-GPU run derives from the same beams) equals the
  single-GPU step-by-step run bit for bit in the last fields and diagnostics and in every particle; the
  moment sums, added over the stages, agree to rounding (1e-10 relative to their natural scale). With
  exact=False (FP64 reductions) the whole run agrees to rounding: moments 1e-10, E_z / B_z and particles
  1e-9.
- The entry point refuses what a stage cannot do: a guard row with the linear xi shape, a plasma state of
  the wrong shape.
"""
import numpy as np
import pytest

import quarz_b200 as Q
from quarz_b200 import stages, workloads
from test_gpu_pipeline import _same

pytestmark = pytest.mark.gpu


def _ngp_spec(full, steps=1, n=100000):
    text = workloads.pinched_witness_deck(xi_min=-11.995 if full else -9.0, driver_np=n * (10 if full else 1),
                                          witness_np=n * (10 if full else 1), steps=steps)
    return workloads.spec_from_text(text, ["beams.xi_shape=ngp"])


def _sources(spec, beams):
    import torch

    grid = Q.RadialGrid(spec.nodes)
    bsrc = torch.zeros((spec.K, spec.M, 5), dtype=torch.float64, device="cuda")
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, spec.K, spec.ngp, spec.modes)
    for b, (parts, _, _) in zip(spec.beams, beams):
        cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
        Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    return grid, bsrc


@pytest.mark.parametrize("full", [False, True])
def test_stage_sweeps_equal_the_whole_sweep_bit_for_bit(full):
    import torch

    spec = _ngp_spec(full)
    assert spec.ngp
    beams = [Q.sample_beam(b) for b in spec.beams]
    grid, bsrc = _sources(spec, beams)
    K, M = spec.K, spec.M
    f64 = dict(dtype=torch.float64, device="cuda")
    whole = Q.Sweep(grid, Q.sweep_params(spec))
    fld, diag = torch.zeros((K, M, 6), **f64), torch.zeros((K, M, 3), **f64)
    lost = whole.run(bsrc, fld, diag)
    torch.cuda.synchronize()
    F, D, P = fld.cpu().numpy(), diag.cpu().numpy(), whole.plasma()
    for ns in (2, 3):
        parts_f, parts_d, nlost, state = [], [], 0, None
        for r, (k0, kl) in enumerate(stages.slabs(K, ns)):
            sw = Q.Sweep(grid, Q.sweep_params(stages.slab_spec(spec, k0, kl)))
            f, d = torch.zeros((kl, M, 6), **f64), torch.zeros((kl, M, 3), **f64)
            out = sw.new_state() if r < ns - 1 else None
            cnt = sw.run_stage(bsrc[k0:k0 + kl], f, d, guard=bsrc[k0 - 1].contiguous() if r else None,
                               state_in=state, state_out=out)
            nlost += cnt["lost"]
            parts_f.append(f.cpu().numpy())
            parts_d.append(d.cpu().numpy())
            state = out
        torch.cuda.synchronize()
        assert np.array_equal(np.concatenate(parts_f), F), ns
        assert np.array_equal(np.concatenate(parts_d), D), ns
        assert np.array_equal(sw.plasma(), P), ns
        assert nlost == lost, (ns, nlost, lost)


@pytest.mark.parametrize("ns,exact", [(2, True), (3, True), (2, False)])
def test_staged_run_equals_the_single_gpu_run(ns, exact):
    spec = _ngp_spec(False, steps=5, n=50000)
    beams = [Q.sample_beam(b) for b in spec.beams]
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(False)
    mom = sim.run(spec.steps, spec.dt)
    fld, diag = sim.fields()
    run = stages.Stages(spec, ns, beams, exact=exact)
    smom = run.run(spec.steps, spec.dt)
    sfld, sdiag = run.fields()
    # particles per beam: the staged run keeps them grouped by slab; compare in the caller's order of ids
    single = [sim.beam(q) for q in range(len(beams))]
    staged = [run.beam(q) for q in range(len(beams))]
    order = []
    for q in range(len(beams)):
        a, b = single[q], staged[q]
        assert a.shape == b.shape
        ka = np.lexsort(a.T[::-1])
        kb = np.lexsort(b.T[::-1])
        order.append((a[ka], b[kb]))
    _same(spec, beams, (smom, sfld, [b for _, b in order]), (mom, fld, [a for a, _ in order]))
    if exact:
        assert np.array_equal(sfld, fld) and np.array_equal(sdiag, diag)
        for a, b in order:
            assert np.array_equal(a, b)


def test_stage_entry_point_refuses_what_a_stage_cannot_do():
    import torch

    spec = workloads.spec_from_text(workloads.pinched_witness_deck(xi_min=-2.0, driver_np=1000, witness_np=1000))
    assert not spec.ngp
    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    f64 = dict(dtype=torch.float64, device="cuda")
    bsrc = torch.zeros((spec.K, spec.M, 5), **f64)
    fld, diag = torch.zeros((spec.K, spec.M, 6), **f64), torch.zeros((spec.K, spec.M, 3), **f64)
    with pytest.raises(Q.QZError, match="ngp"):
        sw.run_stage(bsrc, fld, diag, guard=torch.zeros((spec.M, 5), **f64))
    spec2 = workloads.spec_from_text(workloads.pinched_witness_deck(xi_min=-2.0, driver_np=1000, witness_np=1000),
                                     ["beams.xi_shape=ngp"])
    sw2 = Q.Sweep(grid, Q.sweep_params(spec2))
    bad = torch.zeros((3, 7), **f64)
    with pytest.raises(Q.QZError, match="state"):
        sw2.run_stage(bsrc, fld, diag, state_in=bad)
