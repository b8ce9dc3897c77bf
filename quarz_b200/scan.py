"""A parameter scan over several GPUs.

The instances of a scan are independent runs, so they shard with no data-path exchange. Each rank
runs a cost-balanced share of the instances in one batch (qz_batch: one persistent launch, a CTA per
instance). The only collective is the final gather of every instance's last-step moment sums
(17 doubles per beam) onto every rank. The reference has no counterpart: it runs one deck per
process.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np

MAX_BEAMS = 2          # beams per batched instance


def instance_cost(spec, beam_particles: int) -> float:
    """Relative run time of an instance, the estimate the batch queue orders by: the sweep's slices
    times (nodes + 4 x plasma particles per slice), about 7x more per slice with modes = 1, plus the
    beam work."""
    np_slice = sum(sp.ppc * max(1, sp.ntheta if spec.modes else 1) for sp in spec.species) * (spec.M - 1)
    m1 = spec.modes == 1
    return (7.0 if m1 else 1.0) * spec.K * (spec.M + 4.0 * np_slice) + 2.0 * beam_particles * (3.0 if m1 else 1.0)


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time split: instances by decreasing cost, each to the least loaded rank
    (ties to the lower rank). Every rank's list is returned in increasing instance order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def batch_runner(nsteps: int, dt: float, stream=None) -> Callable:
    """The runner of `run_sharded` on a GPU: all of a rank's instances in one qz_batch launch."""
    from .api import Batch

    def run(specs, beams):
        b = Batch()
        for s, bm in zip(specs, beams):
            b.add(s, bm)
        return b.run(nsteps, dt, stream=stream)

    return run


def run_sharded(specs: Sequence, beams: Sequence, runner: Callable, group=None,
                device: Optional[str] = None) -> np.ndarray:
    """Runs this rank's share of the scan and gathers the last-step moment sums of every instance.

    specs, beams: the whole scan (every rank passes the same lists). runner(specs, beams) -> a list of
    (steps + 1, nbeams, 17) arrays for the given instances. Returns (len(specs), MAX_BEAMS, 17): the
    last step's sums per instance and beam (zero for an absent beam), identical on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    nb = [sum(len(p) for p, _, _ in bm) for bm in beams]
    parts = partition([instance_cost(s, n) for s, n in zip(specs, nb)], world)
    mine = parts[rank]
    moms = runner([specs[i] for i in mine], [beams[i] for i in mine]) if mine else []
    width = max(len(p) for p in parts)
    local = np.zeros((width, MAX_BEAMS, 17))
    for k, m in enumerate(moms):
        local[k, :m.shape[1]] = m[-1]
    out = np.zeros((len(specs), MAX_BEAMS, 17))
    if world == 1:
        out[mine] = local[:len(mine)]
        return out
    t = torch.from_numpy(local).to(device or "cpu")
    bufs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(bufs, t, group=group)
    for r, p in enumerate(parts):
        out[p] = bufs[r].cpu().numpy()[:len(p)]
    return out
