"""The xi-pipelined run's host side without a GPU: the cut of the box into slabs, and the message between
two ranks over torch.distributed (gloo, world size 2, CPU tensors): the plasma state, the guard row and the
particles that changed slab, including a beam with none, arrive unchanged and in order over several steps."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from quarz_b200 import stages


def test_slabs_cover_the_box_in_order():
    for K, n in ((2400, 1), (2400, 2), (2401, 3), (10, 10), (901, 4)):
        s = stages.slabs(K, n)
        assert s[0][0] == 0 and sum(kl for _, kl in s) == K
        assert all(s[i][0] + s[i][1] == s[i + 1][0] for i in range(n - 1))
        assert max(kl for _, kl in s) - min(kl for _, kl in s) <= 1
    with pytest.raises(ValueError):
        stages.slabs(3, 4)


def _message(step, rng_seed):
    import torch

    rng = np.random.default_rng(rng_seed + step)
    state = torch.from_numpy(rng.normal(size=(21, 512)))
    guard = torch.from_numpy(rng.normal(size=(2, 64, 5)))          # exact limbs: high row, low row
    beams = [torch.from_numpy(rng.normal(size=(7, 3 + step))), torch.zeros((7, 0), dtype=torch.float64)]
    return stages.Message(state, step > 0, guard, beams)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ch = stages.DistChannel(torch.device("cpu"), 2, (21, 512), 64)
        ok = True
        for step in range(3):
            if rank == 0:
                ch.send(1, step, _message(step, 7))
            else:
                got, want = ch.recv(0, 1, step), _message(step, 7)
                ok = ok and got.pushed == want.pushed and torch.equal(got.state, want.state)
                ok = ok and torch.equal(got.guard, want.guard)
                ok = ok and all(torch.equal(a, b) for a, b in zip(got.beams, want.beams))
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_stage_messages_between_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: True, 1: True}
