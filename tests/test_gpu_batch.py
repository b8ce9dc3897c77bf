"""Batched parameter scan: every instance of one persistent launch (a CTA per instance) against the
same instance run on its own (step by step) and, for two of them, against the oracle.

Instances are drawn like the scan workload (quarz_b200.workloads.scan_instances: 128-1024 cells,
stretched grids, xi lengths 8-16) with 4000 beam particles and 3 steps. Tolerances: derived beam
moments 1e-10 relative to their natural scale against the single runs (only the summation order of
the beam deposits differs), 1e-8 against the oracle. The m = 1 case draws the same way with modes 0, 1
(Picard 3, 4 azimuths per ring, 128-1023 cells: two of the three above 512 nodes, run by the 1024-thread
batch kernel after the 512-thread one), mixed in one batch with m = 0 instances; and a batch of
m = 0 and m = 1 instances of which three smooth their plasma sources (plasma.smooth_length = 0.02), run by
the kernel variant with the filter."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from quarz_b200 import workloads

pytestmark = pytest.mark.gpu

KEYS = ("gamma_mean", "gamma_rms", "xi_mean", "xi_rms", "r_rms", "emit_nx", "charge_w", "alive")


def _close(spec, mom, ref, beams, tol):
    L, R = spec.K * spec.dxi, spec.nodes[-1]
    for q, (_, gref, xiref) in enumerate(beams):
        for n in range(mom.shape[0]):
            d, dr = O.from_sums(mom[n, q], gref, xiref), O.from_sums(ref[n, q], gref, xiref)
            sc = {"gamma_rms": abs(dr.get("gamma_mean", 0.0)), "xi_mean": L, "xi_rms": L, "r_rms": R}
            for k in KEYS:
                if k not in dr:
                    continue
                assert abs(d[k] - dr[k]) <= tol * max(abs(dr[k]), sc.get(k, 0.0), 1e-300), (q, n, k, d[k], dr[k])


def test_batch_equals_single_runs_and_oracle():
    specs = workloads.scan_instances(6, seed=7, beam_particles=4000, steps=3)
    assert min(s.M for s in specs) <= 513 < max(s.M for s in specs)      # both sweep variants
    beams = [[Q.sample_beam(b) for b in s.beams] for s in specs]
    batch = Q.Batch()
    for s, bm in zip(specs, beams):
        batch.add(s, bm)
    moms = batch.run(3, specs[0].dt)
    info = batch.info()
    assert info["instances"] == 6 and info["ctas"] == 6
    for s, bm, mom in zip(specs, beams, moms):
        sim = Q.Simulation(s, beams=bm)
        sim.set_schedule(False)
        _close(s, mom, sim.run(3, s.dt), bm, 1e-10)
    for s, bm, mom in list(zip(specs, beams, moms))[:2]:
        ref = O.OracleSim(s, beams=bm)
        _close(s, mom, ref.run(3, s.dt), bm, 1e-8)


def test_batch_m1_and_mixed_modes():
    m1 = workloads.scan_instances(3, seed=4, beam_particles=2000, steps=2, modes=1)
    assert sorted(s.M > 512 for s in m1) == [False, True, True]
    m0 = workloads.scan_instances(2, seed=12, beam_particles=2000, steps=2)
    specs = m1 + m0
    beams = [[Q.sample_beam(b) for b in s.beams] for s in specs]
    batch = Q.Batch()
    for s, bm in zip(specs, beams):
        batch.add(s, bm)
    moms = batch.run(2, specs[0].dt)
    for s, bm, mom in zip(specs, beams, moms):
        sim = Q.Simulation(s, beams=bm)
        sim.set_schedule(False)
        _close(s, mom, sim.run(2, s.dt), bm, 1e-10)
    ref = O.OracleSim(specs[0], beams=beams[0])
    _close(specs[0], moms[0], ref.run(2, specs[0].dt), beams[0], 1e-8)


def test_batch_m1_refuses_wide_grids():
    spec = workloads.scan_instances(1, seed=3, beam_particles=1000, steps=1, modes=1)[0]
    spec.modes = 1
    spec.nodes = workloads.scan_nodes(1100, 1e-3)
    with pytest.raises(Q.QZError, match="M <= 1024"):
        Q.Batch().add(spec)


def test_batch_with_smoothing():
    m0 = workloads.scan_instances(3, seed=21, beam_particles=2000, steps=2)
    m1 = workloads.scan_instances(2, seed=22, beam_particles=2000, steps=2, modes=1)
    specs = m0 + m1
    for i in (0, 2, 3):
        specs[i].smooth_length = 0.02
    beams = [[Q.sample_beam(b) for b in s.beams] for s in specs]
    batch = Q.Batch()
    for s, bm in zip(specs, beams):
        batch.add(s, bm)
    moms = batch.run(2, specs[0].dt)
    for s, bm, mom in zip(specs, beams, moms):
        sim = Q.Simulation(s, beams=bm)
        sim.set_schedule(False)
        _close(s, mom, sim.run(2, s.dt), bm, 1e-10)
    # the filtered m = 0 instance and the filtered m = 1 instance (the batch's m = 1 filter path, which
    # smooths the mode parts in place in the instance's scratch) against the independent oracle
    for i in (0, 3):
        s, bm, mom = specs[i], beams[i], moms[i]
        _close(s, mom, O.OracleSim(s, beams=bm).run(2, s.dt), bm, 1e-8)


def test_autotuned_batch_equals_default_batch():
    # the autotuner (quarz_b200.tune) measures every candidate layout of each size class on representatives
    # and reorders the queue by measured cost; the tuned batch computes the same runs: every layout gives
    # the same moments to rounding (1e-10 of their natural scale), the queue order none at all
    from quarz_b200 import tune

    specs = workloads.scan_instances(12, seed=21, beam_particles=4000, steps=3)
    assert min(s.M for s in specs) <= 513 < max(s.M for s in specs)
    beams = [[Q.sample_beam(b) for b in s.beams] for s in specs]
    base = Q.Batch()
    for s, bm in zip(specs, beams):
        base.add(s, bm)
    ref = base.run(3, specs[0].dt)
    tuned, t = tune.tuned_batch(specs, beams, 3, specs[0].dt, steps=1)
    assert set(t.layouts) == {tune.size_class(s) for s in specs}
    for i, s in enumerate(specs):
        lay, cost = tuned.tuning(i)
        assert lay == t.layout(s) and cost > 0
        if tune.plasma_per_slice(s) <= tune.REG_PARTICLES:
            assert not (lay & 4)
    tuned.set_trace(True)
    moms = tuned.run(3, specs[0].dt)
    tr = tuned.trace()
    assert np.all(tr[:, 2] >= tr[:, 1]) and np.all(tr[:, 3] > 0)
    for s, bm, mom, r in zip(specs, beams, moms, ref):
        _close(s, mom, r, bm, 1e-10)
    # a saved tuning gives the same choices
    again = tune.Tuning.from_json(t.to_json())
    assert again.layouts == t.layouts and again.sweep_us == t.sweep_us
