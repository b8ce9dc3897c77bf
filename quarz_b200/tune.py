"""Autotuner of the batched scan (qz_batch).

The batch runs every instance in one CTA of 512 threads, one slice of radial rows per scan step. What is
left to choose per instance is how its slice data are tiled into shared memory, and in which order the
queue hands instances to CTAs:

- the layout, a bit set: 1 double-buffered slice sources (the next slice's deposit lands in the free half
  while the current one is stored), 2 the per-node operator constants in shared memory (instead of L1-cached
  global loads), 4 a shared-memory copy of the plasma particles when they live in global memory (np > 512
  particles per slice). Which of them fit depends on M; which is fastest is measured;
- the queue cost: the largest-first queue wants each instance's run time. The built-in estimate
  K (M + 4 np) + 2 N_beam misses that plasma in global memory costs about twice as much per particle as
  plasma in registers, so those instances start late and leave a tail.

`calibrate` runs a short batch (a few steps) of representatives of every size class (modes, filter, plasma
in registers or not, M in steps of 128), each representative once per layout that fits, with the
per-instance timeline on (qz_batch_trace); it keeps per class the fastest layout and its sweep time per
slice-step, and a beam time per particle-step. `apply` sets every instance's layout and predicted cost
(qz_batch_set_tuning). The measurement runs the representatives side by side, one per SM, as the batch
itself does, so the times include the contention of a full device. A Tuning can be saved and loaded
(JSON) to skip the calibration on the next scan of the same shapes and device.
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

REG_PARTICLES = 512     # particles per slice kept one per thread in registers (the CTA's threads)
LAYOUTS = range(8)


def plasma_per_slice(spec) -> int:
    """Mobile plasma particles per slice (the sweep's np)."""
    return sum(sp.ppc * (sp.ntheta if spec.modes else 1) for sp in spec.species if sp.mobile) * (spec.M - 1)


def size_class(spec) -> Tuple[int, int, int, int]:
    """(modes, filter, plasma in global memory, M // 128): instances that share a layout and a rate."""
    return (int(spec.modes), int(getattr(spec, "smooth_length", 0.0) > 0.0),
            int(plasma_per_slice(spec) > REG_PARTICLES), int(spec.M) // 128)


def candidate_layouts(spec) -> List[int]:
    """The layouts to try (the library rejects those that do not fit): none for modes = 1, the particle
    copy only with plasma in global memory."""
    if spec.modes != 0:
        return [-1]
    glob = plasma_per_slice(spec) > REG_PARTICLES
    return [l for l in LAYOUTS if glob or not (l & 4)]


@dataclass
class Tuning:
    """Per size class the chosen layout and its measured sweep time (us per slice-step), and the beam
    time per particle-step (us); `cost` predicts an instance's run time from them (us)."""
    layouts: Dict[Tuple[int, int, int, int], int] = field(default_factory=dict)
    sweep_us: Dict[Tuple[int, int, int, int], float] = field(default_factory=dict)
    beam_us: float = 0.0
    device: str = ""

    def layout(self, spec) -> int:
        return self.layouts.get(size_class(spec), -1)

    def cost(self, spec, beam_particles: int, nsteps: int) -> float:
        """Predicted run time (us) of nsteps (nsteps + 1 sweeps): the class's measured slice time, or that
        of the nearest measured class of the same kind scaled by M, plus the beam work."""
        c = size_class(spec)
        rate = self.sweep_us.get(c)
        if rate is None:
            same = [(k, v) for k, v in self.sweep_us.items() if k[:3] == c[:3]]
            if not same:
                same = list(self.sweep_us.items())
            if not same:
                return 0.0
            k, v = min(same, key=lambda kv: abs(kv[0][3] - c[3]))
            rate = v * (c[3] + 1) / (k[3] + 1)
        return rate * spec.K * (nsteps + 1) + self.beam_us * beam_particles * nsteps

    def to_json(self) -> str:
        return json.dumps({"device": self.device, "beam_us": self.beam_us,
                           "classes": [[list(k), self.layouts[k], self.sweep_us[k]] for k in sorted(self.layouts)]})

    @staticmethod
    def from_json(text: str) -> "Tuning":
        d = json.loads(text)
        t = Tuning(beam_us=float(d["beam_us"]), device=d.get("device", ""))
        for k, lay, us in d["classes"]:
            t.layouts[tuple(k)] = int(lay)
            t.sweep_us[tuple(k)] = float(us)
        return t


def choose(samples: Sequence[Tuple[Tuple[int, int, int, int], int, float]]) -> Tuple[Dict, Dict]:
    """From (class, layout, us per slice-step) measurements: per class the layout with the lowest median
    time and that time."""
    by: Dict[Tuple, Dict[int, List[float]]] = {}
    for c, lay, us in samples:
        by.setdefault(c, {}).setdefault(lay, []).append(us)
    layouts, rates = {}, {}
    for c, per in by.items():
        lay, ts = min(per.items(), key=lambda kv: (float(np.median(kv[1])), kv[0]))
        layouts[c] = lay
        rates[c] = float(np.median(ts))
    return layouts, rates


def representatives(specs: Sequence, per_class: int = 2) -> List[int]:
    """Per size class the indices of its per_class largest instances (by M, then K): a layout that fits
    the largest M of a class fits the whole class."""
    groups: Dict[Tuple, List[int]] = {}
    for i, s in enumerate(specs):
        groups.setdefault(size_class(s), []).append(i)
    out = []
    for c in sorted(groups):
        idx = sorted(groups[c], key=lambda i: (-specs[i].M, -specs[i].K, i))
        out.extend(idx[:per_class])
    return out


def calibrate(specs: Sequence, beams: Sequence, dt: float, steps: int = 2, per_class: int = 2) -> Tuning:
    """Measures the candidate layouts of representatives of every size class on the device (one batch of
    `steps` steps) and returns the Tuning."""
    from .api import Batch, QZError

    b = Batch()
    entries = []                      # (batch index, class, layout, spec index)
    for i in representatives(specs, per_class):
        for lay in candidate_layouts(specs[i]):
            j = b.add(specs[i], beams[i])
            ok = True
            if lay >= 0:
                try:
                    b.set_tuning(j, lay)
                except QZError:
                    ok = False        # does not fit: runs with the default layout, not counted
            if ok:
                entries.append((j, size_class(specs[i]), lay, i))
    b.set_trace(True)
    b.run(steps, dt)
    tr = b.trace()
    samples, beam = [], []
    for j, c, lay, i in entries:
        s = specs[i]
        samples.append((c, lay, 1e3 * tr[j, 3] / (s.K * (steps + 1))))
        nb = sum(len(p) for p, _, _ in beams[i])
        if nb and steps:
            beam.append(1e3 * tr[j, 4] / (nb * steps))
    layouts, rates = choose(samples)
    import torch

    return Tuning(layouts=layouts, sweep_us=rates, beam_us=float(np.median(beam)) if beam else 0.0,
                  device=torch.cuda.get_device_name())


def apply(batch, specs: Sequence, beams: Sequence, nsteps: int, tuning: Tuning) -> None:
    """Sets every instance's layout and predicted cost (instances added to `batch` in the order of specs).
    A layout that does not fit an instance (a tuning loaded for other shapes) leaves its layout as it is."""
    from .api import QZError

    for i, s in enumerate(specs):
        nb = sum(len(p) for p, _, _ in beams[i])
        cost = tuning.cost(s, nb, nsteps)
        try:
            batch.set_tuning(i, tuning.layout(s), cost)
        except QZError:
            batch.set_tuning(i, -1, cost)


def tuned_batch(specs: Sequence, beams: Sequence, nsteps: int, dt: float, tuning: Optional[Tuning] = None,
                steps: int = 2):
    """A Batch of all instances with the autotuner's layouts and costs (calibrating first unless a Tuning
    is given); returns (batch, tuning)."""
    from .api import Batch

    t = tuning if tuning is not None else calibrate(specs, beams, dt, steps=steps)
    b = Batch()
    for s, bm in zip(specs, beams):
        b.add(s, bm)
    apply(b, specs, beams, nsteps, t)
    return b, t
