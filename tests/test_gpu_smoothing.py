"""GPU parity of the radial smoothing filter (plasma.smooth_length) and of analytic rigid beams: the CUDA
path through the C ABI against the oracle on the same inputs.

Decks: the plain blowout (config 0's deck, 257 uniform nodes, one thread row per node) and a finer
uniform grid of 801 nodes (two rows per thread, plasma state in global memory), both with
plasma.smooth_length = 0.05 and 2e4 driver particles, box cut to xi in [-8, 0]; an analytic driver
(m = 0) with a particle witness on the stretched 512-node grid; and an analytic driver displaced by
0.05 in x with modes = 1; the hosing deck (modes = 1, 8 azimuths, Picard 3) cut to xi in [-9, 0] with
plasma.smooth_length = 0.02.

Tolerances as in the other parity tests: beam sources 1e-12 (FP64 reductions in another order); fields
and diagnostics after one sweep, relative L2 per stored component, within max(1e-10, 4 x the reference
algorithm's own round-off floor on the input, its Thomas-vs-partition difference), psi / E_z / B_z
within 1e-10 outright; beam moments after a run 1e-8 relative to their natural scale, pipelined and
step by step."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import CONFIG0, rel_l2
from quarz_b200 import workloads
from test_gpu_pipeline import _close

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10


def _blowout(extra=()):
    return workloads.spec_from_text(CONFIG0, ["xi.min=-8", "driver.nparticles=20000", "time.steps=3",
                                              "plasma.smooth_length=0.05"] + list(extra))


def _analytic_m0(steps=3):
    text = workloads.pinched_witness_deck(xi_min=-9.0, driver_np=1000, witness_np=20000, steps=steps)
    return workloads.spec_from_text(text, ["driver.analytic=1"])


def _analytic_m1():
    text = workloads.hosing_deck(xi_min=-9.0, driver_np=1000, witness_np=20000, steps=2)
    return workloads.spec_from_text(text, ["xi.step=0.01", "driver.analytic=1", "driver.x0=0.05",
                                           "driver.x_slope=0.002"])


def _gpu_sweep(spec, beams):
    import torch

    assert torch.cuda.is_available(), "CUDA device required"
    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    K, M = spec.K, spec.M
    bnc, fnc, dnc = (15, 18, 9) if spec.modes else (5, 6, 3)
    f64 = dict(dtype=torch.float64, device="cuda")
    bsrc, fld, diag = torch.zeros(K * M * bnc, **f64), torch.zeros(K * M * fnc, **f64), torch.zeros(K * M * dnc, **f64)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    for b, (parts, _, _) in zip(spec.beams, beams):
        if b.analytic:
            Q.BeamOps.deposit_analytic(grid, b, box, bsrc)
        else:
            cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
            Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    lost = sw.run(bsrc, fld, diag)
    torch.cuda.synchronize()
    return (bsrc.cpu().numpy().reshape(K, M, bnc), fld.cpu().numpy().reshape(K, M, fnc),
            diag.cpu().numpy().reshape(K, M, dnc), lost)


def _one_sweep(spec, bsrc_tol=1e-12):
    beams = [Q.sample_beam(b) for b in spec.beams]
    a = O.OracleSim(spec, beams=beams, tridiag="thomas")
    a.step_fields(0.0)
    b = O.OracleSim(spec, beams=beams, tridiag="partition")
    b.step_fields(0.0)
    bs, fld, diag, lost = _gpu_sweep(spec, beams)
    B = a.bsrc()
    for c in range(B.shape[-1]):
        if np.any(B[..., c]):
            assert rel_l2(bs[..., c], B[..., c]) < bsrc_tol, ("bsrc", c)
    errs, bad = {}, {}
    for name, got, want, alt in (("fld", fld, a.fld(), b.fld()), ("diag", diag, a.diag(), b.diag())):
        for c in range(want.shape[-1]):
            if not np.any(want[..., c]):
                continue
            e = rel_l2(got[..., c], want[..., c])
            floor = rel_l2(alt[..., c], want[..., c])
            errs[f"{name}{c}"] = e
            if not e < max(FIELD_TOL, 4.0 * floor):
                bad[f"{name}{c}"] = (e, floor)
    assert not bad, (bad, errs)
    for k in ("diag0", "fld4"):                               # psi, E_z
        assert errs[k] < FIELD_TOL, (k, errs[k])
    if spec.modes == 0:
        assert errs["fld5"] < FIELD_TOL, errs["fld5"]         # B_z
    assert lost == a.lost()
    return errs


def _runs_against_oracle(spec, steps):
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(steps, spec.dt)
    F = ref.fld()
    for pipelined in (True, False):
        sim = Q.Simulation(spec, beams=beams)
        sim.set_schedule(pipelined)
        mom = sim.run(steps, spec.dt)
        assert mom.shape == mom_ref.shape
        for q, (b, (_, gref, xiref)) in enumerate(zip(spec.beams, beams)):
            if b.analytic:
                assert np.all(mom[:, q] == 0) and np.all(mom_ref[:, q] == 0)
                continue
            m1 = spec.modes == 1
            for n in range(steps + 1):
                d, dr = O.from_sums(mom[n, q], gref, xiref, m1=m1), O.from_sums(mom_ref[n, q], gref, xiref, m1=m1)
                _close(spec, d, dr, 1e-8, (pipelined, q, n))
        fld, _ = sim.fields()
        for c in (4, 5):
            assert rel_l2(fld[..., c], F[..., c]) < 1e-8, (pipelined, c)


def test_filter_one_sweep_257_nodes():
    _one_sweep(_blowout())


def test_filter_one_sweep_801_nodes_two_rows_per_thread():
    _one_sweep(_blowout(["grid.dr=0.0075"]))


def test_filter_runs_against_oracle():
    _runs_against_oracle(_blowout(), 3)


def test_analytic_driver_m0_one_sweep_and_runs():
    spec = _analytic_m0()
    _one_sweep(spec)
    _runs_against_oracle(spec, 3)


def test_analytic_driver_m1_displaced_one_sweep():
    _one_sweep(_analytic_m1())


def _hosing_filtered():
    text = workloads.hosing_deck(xi_min=-9.0, driver_np=20000, witness_np=20000, steps=2)
    return workloads.spec_from_text(text, ["xi.step=0.01", "plasma.smooth_length=0.02"])


def test_filter_m1_one_sweep():
    _one_sweep(_hosing_filtered())


def test_filter_m1_runs_against_oracle():
    _runs_against_oracle(_hosing_filtered(), 2)
