"""The batch autotuner's host logic (quarz_b200.tune), without a GPU: size classes, candidate layouts, the
choice from measurements, representatives, the cost model and its JSON form."""
import numpy as np

from quarz_b200 import tune, workloads


def test_classes_and_candidates():
    specs = workloads.scan_instances(40, seed=3, beam_particles=100, steps=2)
    for s in specs:
        c = tune.size_class(s)
        assert c[0] == 0 and c[3] == s.M // 128
        glob = tune.plasma_per_slice(s) > tune.REG_PARTICLES
        assert c[2] == int(glob)
        cands = tune.candidate_layouts(s)
        assert (4 in cands) == glob and all(0 <= l < 8 for l in cands)
    m1 = workloads.scan_instances(3, seed=4, beam_particles=100, steps=2, modes=1)
    assert all(tune.candidate_layouts(s) == [-1] for s in m1)


def test_choose_and_representatives():
    a, b = (0, 0, 0, 3), (0, 0, 1, 5)
    samples = [(a, 3, 10.0), (a, 3, 12.0), (a, 1, 11.5), (a, 1, 11.0), (b, 5, 40.0), (b, 4, 30.0), (b, 4, 60.0)]
    lay, rate = tune.choose(samples)
    assert lay == {a: 3, b: 5} and rate == {a: 11.0, b: 40.0}     # medians: a 11 (3) vs 11.25 (1); b 40 vs 45
    specs = workloads.scan_instances(30, seed=5, beam_particles=100, steps=2)
    reps = tune.representatives(specs, per_class=2)
    classes = {tune.size_class(s) for s in specs}
    assert len(reps) <= 2 * len(classes) and {tune.size_class(specs[i]) for i in reps} == classes
    for i in reps:       # each is among the two largest M of its class
        c = tune.size_class(specs[i])
        ms = sorted((s.M for s in specs if tune.size_class(s) == c), reverse=True)
        assert specs[i].M >= ms[min(1, len(ms) - 1)]


def test_cost_model_and_json():
    specs = workloads.scan_instances(30, seed=6, beam_particles=100, steps=2)
    t = tune.Tuning(beam_us=0.01, device="test")
    for s in specs:
        c = tune.size_class(s)
        t.layouts[c] = 3 if not c[2] else 5
        t.sweep_us[c] = (60.0 if c[2] else 25.0)
    # measured rates order the queue: plasma in global memory costs more per slice
    big = [s for s in specs if tune.size_class(s)[2]]
    small = [s for s in specs if not tune.size_class(s)[2]]
    if big and small:
        sb = max(big, key=lambda s: s.K)
        ss = min(small, key=lambda s: s.K)
        if sb.K >= ss.K:
            assert t.cost(sb, 100, 20) > t.cost(ss, 100, 20)
    assert np.isclose(t.cost(specs[0], 1000, 20), t.sweep_us[tune.size_class(specs[0])] * specs[0].K * 21 + 0.01 * 1000 * 20)
    # an unmeasured class borrows the nearest measured one of its kind, scaled by M
    kind = {}
    for s in specs:
        kind.setdefault(tune.size_class(s)[:3], {}).setdefault(tune.size_class(s)[3], s)
    pairs = [(v[min(v)], v[max(v)]) for v in kind.values() if len(v) > 1]
    assert pairs
    lo, hi = pairs[0]
    c0 = tune.size_class(lo)
    u = tune.Tuning(layouts={c0: 3}, sweep_us={c0: 20.0}, beam_us=0.0)
    c1 = tune.size_class(hi)
    assert np.isclose(u.cost(hi, 0, 1), 20.0 * (c1[3] + 1) / (c0[3] + 1) * hi.K * 2)
    back = tune.Tuning.from_json(t.to_json())
    assert back.layouts == t.layouts and back.sweep_us == t.sweep_us and back.beam_us == t.beam_us
