"""Azimuthal modes m = 0, 1 (the hosing workload): the CUDA m = 1 sweep and whole runs against the
oracle on the same inputs.

Workload: the pinched-witness grid (512 stretched nodes) with modes = 1, Picard 3, 8 azimuths per
plasma ring (4088 particles per slice), the driver offset 0.1 in x and tilted 1e-3, the witness offset
0.02; box cut to xi in [-9, 0] with dxi 0.01 (901 slices) and 2 x 20000 beam particles so that the
oracle finishes in seconds. The wide cases put the same deck on geometric grids of 700 and 1024 nodes
(axis cell 1e-3, wall r = 6): the m = 1 sweep then runs in a CTA of 1024 threads, one node per thread.

Tolerances (relative L2 per stored component): beam sources 1e-12; fields and diagnostics after one
sweep max(1e-10, 4 x the reference algorithm's own round-off floor on this input, i.e. the difference
between its Thomas and partition tridiagonal solvers); beam moments after a run 1e-8 relative to
their natural scale."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import rel_l2
from quarz_b200 import workloads

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10
MOMENT_TOL = 1e-8
KEYS = ("gamma_mean", "gamma_rms", "xi_mean", "xi_rms", "x_mean", "y_mean", "sigma_x", "emit_nx", "charge_w", "alive")


def _spec(steps=3, n=20000, M=None):
    text = workloads.hosing_deck(xi_min=-9.0, driver_np=n, witness_np=n, steps=steps)
    spec = workloads.spec_from_text(text, ["xi.step=0.01"])
    if M is not None:
        spec.nodes = workloads.scan_nodes(M, 1e-3)
    return spec


def _gpu_sweep(spec, beams):
    import torch

    assert torch.cuda.is_available(), "CUDA device required"
    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    K, M = spec.K, spec.M
    f64 = dict(dtype=torch.float64, device="cuda")
    bsrc, fld, diag = torch.zeros(K * M * 15, **f64), torch.zeros(K * M * 18, **f64), torch.zeros(K * M * 9, **f64)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    for b, (parts, _, _) in zip(spec.beams, beams):
        cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
        Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    lost = sw.run(bsrc, fld, diag)
    torch.cuda.synchronize()
    return (bsrc.cpu().numpy().reshape(K, M, 15), fld.cpu().numpy().reshape(K, M, 18),
            diag.cpu().numpy().reshape(K, M, 9), lost)


@pytest.mark.parametrize("M", [None, 700, 1024])
def test_sweep_m1_one_step_against_oracle(M):
    spec = _spec(M=M)
    beams = [Q.sample_beam(b) for b in spec.beams]
    a = O.OracleSim(spec, beams=beams, tridiag="thomas")
    a.step_fields(0.0)
    b = O.OracleSim(spec, beams=beams, tridiag="partition")
    b.step_fields(0.0)
    bs, fld, diag, lost = _gpu_sweep(spec, beams)
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
    assert not bad, f"m = 1 field mismatch {bad}; all {errs}"
    assert lost == a.lost()


@pytest.mark.parametrize("pipelined,M", [(True, None), (False, None), (True, 700)])
def test_run_m1_moments_against_oracle(pipelined, M):
    # the whole run as one pipelined launch (sweeps of consecutive steps concurrent), and step by step;
    # with more than 512 nodes the run goes step by step (the pipeline's sweep CTAs have 512 threads)
    spec = _spec(steps=3, M=M)
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(spec.steps, spec.dt)
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(pipelined)
    mom = sim.run(spec.steps, spec.dt)
    assert sim.schedule()["pipelined"] == (1 if pipelined and spec.M <= 512 else 0)
    L = spec.K * spec.dxi
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(spec.steps + 1):
            d = O.from_sums(mom[n, q], gref, xiref, m1=True)
            dr = O.from_sums(mom_ref[n, q], gref, xiref, m1=True)
            scale = {"gamma_rms": abs(dr["gamma_mean"]), "xi_mean": L, "xi_rms": L, "x_mean": spec.nodes[-1],
                     "y_mean": spec.nodes[-1], "sigma_x": spec.nodes[-1]}
            for k in KEYS:
                tol = MOMENT_TOL * max(abs(dr[k]), scale.get(k, 0.0), 1e-300)
                assert abs(d[k] - dr[k]) <= tol, (q, n, k, d[k], dr[k])
    fld, _ = sim.fields()
    F = ref.fld()
    for c in (4, 5, 14, 15):                 # E_z, B_z modes 0 and 1 after the last sweep
        assert rel_l2(fld[..., c], F[..., c]) < 1e-8, c
    for q in range(len(beams)):
        got, want = sim.beam(q), ref.beam(q)
        for c in range(6):
            assert rel_l2(got[:, c], want[:, c]) < 1e-9, (q, c)
