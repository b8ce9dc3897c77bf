"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the same inputs.

Tolerances (relative L2 over each stored component): beam deposit 1e-12 (FP64 reductions in a
different order), one sweep 1e-10 (the bar stated for the fields after one step), beam moments
after a run 1e-8."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import CONFIG0, bsum_numbers, config1_deck, rel_l2, spec_from_text

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10
MOMENT_TOL = 1e-8


def _torch():
    import torch

    assert torch.cuda.is_available(), "CUDA device required"
    return torch


def _gpu_sweep(spec, beams):
    """deposit + one sweep on the GPU through the granular C ABI; returns bsrc, fld, diag (numpy)."""
    torch = _torch()
    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    K, M = spec.K, spec.M
    bsrc = torch.zeros(K * M * 5, dtype=torch.float64, device="cuda")
    fld = torch.zeros(K * M * 6, dtype=torch.float64, device="cuda")
    diag = torch.zeros(K * M * 3, dtype=torch.float64, device="cuda")
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    for b, (parts, gref, xiref) in zip(spec.beams, beams):
        cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
        Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    lost = sw.run(bsrc, fld, diag)
    torch.cuda.synchronize()
    return (bsrc.cpu().numpy().reshape(K, M, 5), fld.cpu().numpy().reshape(K, M, 6),
            diag.cpu().numpy().reshape(K, M, 3), lost, sw)


def _floor(spec, beams):
    """Round-off noise floor of the reference algorithm itself: relative L2 between the oracle with
    the reference's CPU tridiagonal solver (Thomas) and with its GPU one (partition), per component."""
    a = O.OracleSim(spec, beams=beams, tridiag="thomas")
    a.step_fields(0.0)
    b = O.OracleSim(spec, beams=beams, tridiag="partition")
    b.step_fields(0.0)
    fl = {f"fld{c}": rel_l2(b.fld()[..., c], a.fld()[..., c]) for c in range(6)}
    fl.update({f"diag{c}": rel_l2(b.diag()[..., c], a.diag()[..., c]) for c in range(3)})
    return a, fl


def _compare_fields(spec, beams, tol=FIELD_TOL):
    """Per component: GPU vs oracle within max(1e-10, 4 x the reference's own Thomas-vs-partition
    difference on the same input); psi, E_z and B_z within 1e-10 outright."""
    ref, floor = _floor(spec, beams)
    bs, fld, diag, lost, sw = _gpu_sweep(spec, beams)
    for c in range(5):
        assert rel_l2(bs[..., c], ref.bsrc()[..., c]) < 1e-12, f"bsrc comp {c}"
    F, D = ref.fld(), ref.diag()
    errs = {f"fld{c}": rel_l2(fld[..., c], F[..., c]) for c in range(6) if np.any(F[..., c])}
    errs.update({f"diag{c}": rel_l2(diag[..., c], D[..., c]) for c in range(3) if np.any(D[..., c])})
    bad = {k: (v, floor[k]) for k, v in errs.items() if not v < max(tol, 4.0 * floor[k])}
    assert not bad, f"field mismatch {bad} (all: {errs}, floor: {floor})"
    for k in ("diag0", "fld4", "fld5"):          # psi, E_z, B_z
        assert errs[k] < tol, (k, errs[k])
    assert lost == ref.lost()
    # plasma state at the end of the box
    P = sw.plasma()
    Po = ref.plasma(0)
    assert P.shape == Po.shape
    assert rel_l2(P[:5], Po[:5]) < 1e-6
    return errs


def test_sweep_config0_one_step():
    spec = spec_from_text(CONFIG0)
    beams = [Q.sample_beam(b) for b in spec.beams]
    _compare_fields(spec, beams)


def test_sweep_config1_grid_short_box():
    # the stretched 512-node grid of config 1 with both beams, box cut to xi in [-9, 0]
    spec = spec_from_text(config1_deck(xi_min=-9.0, driver_np=100000, witness_np=100000))
    beams = [Q.sample_beam(b) for b in spec.beams]
    _compare_fields(spec, beams)


def test_sweep_ab4_ppc4_blowout_validation():
    # validation/blowout.in (uniform dr 0.01, xi in [-10, 0]); the printed numbers of
    # validation/reference_full.txt:5 must come out of the GPU sweep too
    import os
    import json

    from helpers import GOLDEN
    with open(os.path.join(GOLDEN, "decks", "blowout.in")) as f:
        spec = spec_from_text(f.read(), ["xi.min=-10"])
    beams = [Q.sample_beam(b) for b in spec.beams]
    bs, fld, diag, lost, sw = _gpu_sweep(spec, beams)
    ref = json.load(open(os.path.join(GOLDEN, "validation_numbers.json")))["blowout_uniform_dr0.01_dxi0.01"]
    got = bsum_numbers(spec, fld)
    assert f"{got['Ez(-5)']:+.4f}" == ref["Ez(-5)"]
    assert f"{got['Ez(-7)']:+.4f}" == ref["Ez(-7)"]
    assert f"{got['Ez(-8)']:+.4f}" == ref["Ez(-8)"]
    assert f"{got['Ezmin']:+.3f}" == ref["Ezmin"]
    assert f"{got['xi_min']:.3f}" == ref["xi_min"]
    assert f"{got['Wr/r']:.4f}" == ref["Wr/r"]


def test_beam_push_against_oracle():
    torch = _torch()
    spec = spec_from_text(CONFIG0)
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    ref.step_fields(0.0)
    F = ref.fld()
    ref.push_beams(spec.dt, spec.dt)
    out_ref = ref.beam(0)
    grid = Q.RadialGrid(spec.nodes)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, spec.K)
    fld = torch.from_numpy(F.reshape(-1).copy()).cuda()
    parts = beams[0][0]
    cols = torch.from_numpy(np.ascontiguousarray(parts.T)).cuda().contiguous()
    st = Q.BeamOps.push(grid, cols, -1.0, 1.0, box, fld, spec.dt, spec.dt, 0)
    assert st == 1
    got = cols.cpu().numpy().T
    for c in range(7):
        assert rel_l2(got[:, c], out_ref[:, c]) < 1e-13, f"column {c}"


def test_run_config0_moments_10_steps():
    spec = spec_from_text(CONFIG0)
    beams = [Q.sample_beam(b) for b in spec.beams]
    ref = O.OracleSim(spec, beams=beams)
    mom_ref = ref.run(spec.steps, spec.dt)
    sim = Q.Simulation(spec, beams=beams)
    mom = sim.run(spec.steps, spec.dt)
    parts, gref, xiref = beams[0]
    for n in range(spec.steps + 1):
        d_ref = O.from_sums(mom_ref[n, 0], gref, xiref)
        d = O.from_sums(mom[n, 0], gref, xiref)
        for key in ("gamma_mean", "gamma_rms", "xi_mean", "xi_rms", "r_rms", "emit_nx", "charge_w", "alive"):
            a, b = d[key], d_ref[key]
            assert abs(a - b) <= MOMENT_TOL * max(abs(b), 1e-300), (n, key, a, b)
    fld, diag = sim.fields()
    F = ref.fld()
    for c in (4, 5):                               # E_z, B_z after the last sweep
        assert rel_l2(fld[..., c], F[..., c]) < 1e-8, f"fields after {spec.steps} steps, comp {c}"
