"""The scan sharded over ranks (quarz_b200.scan), on CPU with the gloo backend at world size 2.

The batch runner needs a GPU, so these tests give run_sharded a stand-in runner whose result is a
fixed function of each instance (its K, M and beam sizes). The gathered result on every rank must
equal the one-rank result, and the cost split must cover every instance once and stay balanced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from quarz_b200 import scan, workloads


def _fake_runner(nsteps):
    def run(specs, beams):
        out = []
        for s, bm in zip(specs, beams):
            m = np.zeros((nsteps + 1, len(bm), 17))
            for q, (p, g, x) in enumerate(bm):
                m[:, q, :] = s.K * 1e-3 + s.M * 1e-6 + len(p) * 1e-9 + q + np.arange(17)[None, :] * 1e-2
                m[:, q, 0] += np.arange(nsteps + 1)
            out.append(m)
        return out
    return run


def _scan(count=9):
    specs = workloads.scan_instances(count, seed=5, beam_particles=40, steps=2)
    rng = np.random.default_rng(1)
    beams = [[(rng.normal(size=(20 + 3 * i, 7)), 1000.0, 0.0) for _ in s.beams] for i, s in enumerate(specs)]
    return specs, beams


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 10, size=37))
    for world in (1, 2, 3, 8):
        parts = scan.partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)
        assert parts == scan.partition(costs, world)          # deterministic
    assert scan.partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        scan.partition([1.0], 0)


def test_cost_orders_m1_above_m0():
    m0 = workloads.scan_instances(1, seed=9, beam_particles=100, steps=1)[0]
    m1 = workloads.scan_instances(1, seed=9, beam_particles=100, steps=1, modes=1)[0]
    assert scan.instance_cost(m1, 100) > scan.instance_cost(m0, 100) * (m1.M / m0.M)


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs, beams = _scan()
        out = scan.run_sharded(specs, beams, _fake_runner(2))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_scan_gathers_the_single_rank_result():
    specs, beams = _scan()
    ref = scan.run_sharded(specs, beams, _fake_runner(2))
    assert ref.shape == (len(specs), scan.MAX_BEAMS, 17) and np.all(ref[:, :, 16] != 0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r, out = q.get(timeout=120)
        got[r] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        np.testing.assert_array_equal(got[r], ref)

