"""The xi-pipelined run over several GPUs: the reference's multi-rank mode (Simulation::run,
src/Simulation.cpp:1370-1448, with the message of Simulation::make_message, :851-870, taken apart by
step_fields, :714-731).

The box is cut into slabs of consecutive slices, one per stage (one rank per GPU). In every time step a
stage
  1. takes the message of the stage ahead of it (none for the first stage): the plasma state leaving that
     stage's last slice (particles and Adams-Bashforth history), the beam sources of that last slice (the
     guard row, for the xi-derivative of rho - J_z at this slab's first slice), and the beam particles that
     moved into this slab during the previous push;
  2. deposits its own beam particles into its slab's beam sources and sweeps its slices from the received
     plasma state (qz_sweep_run_stage);
  3. sends the next stage its message (the plasma after the push of its last slice, its last beam-source
     row, the particles that left it);
  4. pushes its particles with its own fields; those now past the slab's end go into the next message.
A stage only ever waits for the stage ahead of it, so with one rank per stage consecutive time steps run
concurrently, staggered by one slab per rank. The xi shape must be ngp (src/Beam.cpp:746, :980-983):
a particle then deposits into and gathers from its own slice only, so no slab needs another slab's
beams within a step. Every sweep gives the fields of the whole-box sweep bit for bit (its plasma deposits
are exact). With exact beam sources (the default; qz_beam_deposit_fx with the quanta qz_sim derives from
the same beams) every slab's beam sources are the whole box's bit for bit too, so a staged run equals the
single-GPU run in its fields and particles; its moment sums, added over the stages, agree to rounding.
exact=False deposits with FP64 reductions (the whole run then agrees to rounding).

Messages go over torch.distributed (send / recv of float64 tensors, NCCL between GPUs, gloo on CPU), or
between stages run one after the other in one process (Stages.run with a local channel), which is how it
is tested on one GPU. The beam moments of every step are summed over the stages at the end (one
all_reduce per run, not per step, so that no step waits for the last stage).
"""
from __future__ import annotations

import copy
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import api as Q


def slabs(K: int, nstages: int) -> List[Tuple[int, int]]:
    """(first slice, slices) of each stage: consecutive, as equal as possible, the first stages longer."""
    if nstages < 1 or nstages > K:
        raise ValueError(f"stages: {nstages} stages for {K} slices")
    base, extra = divmod(K, nstages)
    out, k0 = [], 0
    for r in range(nstages):
        n = base + (1 if r < extra else 0)
        out.append((k0, n))
        k0 += n
    return out


def slab_spec(spec, k0: int, kl: int):
    """The run spec of one slab: the same grid, plasma and beams, slices [k0, k0 + kl) of the box."""
    s = copy.copy(spec)
    s.xi_min = spec.xi_min + k0 * spec.dxi
    s.K = kl
    return s


class Message:
    """What a stage hands on in one step: the plasma state (a (6 + 5 order, npad) tensor and whether it was
    pushed), the guard row (M x 5, or 2 x M x 5 exact limbs) and the beam particles that entered the next
    slab, per beam (7, n)."""

    def __init__(self, state, pushed: bool, guard, beams):
        self.state, self.pushed, self.guard, self.beams = state, pushed, guard, beams


class LocalChannel:
    """Messages between stages run one after the other in one process."""

    def __init__(self):
        self.box = {}

    def send(self, dst: int, step: int, msg: Message):
        self.box[(dst, step)] = msg

    def recv(self, src: int, dst: int, step: int) -> Message:
        return self.box.pop((dst, step))


class DistChannel:
    """Messages between ranks over torch.distributed: a float64 header (pushed, beam counts) then the
    state, the guard row and each beam's particles, all on the rank's device."""

    def __init__(self, device, nbeams: int, state_shape, M: int, exact: bool = True):
        self.device, self.nbeams, self.state_shape, self.M = device, nbeams, state_shape, M
        self.guard_shape = (2, M, 5) if exact else (M, 5)

    def send(self, dst: int, step: int, msg: Message):
        import torch
        import torch.distributed as dist

        head = torch.tensor([1.0 if msg.pushed else 0.0] + [float(b.shape[1]) for b in msg.beams],
                            dtype=torch.float64, device=self.device)
        dist.send(head, dst)
        dist.send(msg.state.contiguous(), dst)
        dist.send(msg.guard.contiguous(), dst)
        for b in msg.beams:
            if b.shape[1]:
                dist.send(b.contiguous(), dst)

    def recv(self, src: int, dst: int, step: int) -> Message:
        import torch
        import torch.distributed as dist

        head = torch.empty(1 + self.nbeams, dtype=torch.float64, device=self.device)
        dist.recv(head, src)
        state = torch.empty(self.state_shape, dtype=torch.float64, device=self.device)
        dist.recv(state, src)
        guard = torch.empty(self.guard_shape, dtype=torch.float64, device=self.device)
        dist.recv(guard, src)
        beams = []
        for q in range(self.nbeams):
            n = int(head[1 + q].item())
            b = torch.empty((7, n), dtype=torch.float64, device=self.device)
            if n:
                dist.recv(b, src)
            beams.append(b)
        return Message(state, bool(head[0].item() != 0.0), guard, beams)


class Stage:
    """One slab of the box on one device: its sweep, beam sources, fields and beam particles."""

    def __init__(self, spec, rank: int, nstages: int, beams, device=None, bound=None):
        """bound: (wq, particles) of the whole run's beams for exact beam sources (ExactSources.bound), or
        None for FP64 reductions."""
        import torch

        if not spec.ngp:
            raise ValueError("stages: the xi-pipelined run needs beams.xi_shape = ngp")
        if spec.modes != 0:
            raise ValueError("stages: modes = 0 only")
        self.rank, self.nstages = rank, nstages
        self.first, self.last = rank == 0, rank == nstages - 1
        self.k0, self.kl = slabs(spec.K, nstages)[rank]
        self.spec = slab_spec(spec, self.k0, self.kl)
        self.xi_end = spec.xi_min + (spec.K - 1) * spec.dxi       # the box's last slice (internal xi)
        self.device = device if device is not None else torch.device("cuda")
        self.grid = Q.RadialGrid(spec.nodes)
        self.sweep = Q.Sweep(self.grid, Q.sweep_params(self.spec))
        self.box = Q.BeamOps.box(self.spec.xi_min, spec.dxi, self.kl, True, 0)
        M = spec.M
        f64 = dict(dtype=torch.float64, device=self.device)
        self.fx = Q.ExactSources(self.grid, spec.dxi, bound[0], bound[1]) if bound is not None else None
        self.sweep.set_exact_sources(self.fx)
        self.bsrc = torch.zeros((2, self.kl, M, 5) if self.fx else (self.kl, M, 5), **f64)
        self.fld = torch.zeros((self.kl, M, 6), **f64)
        self.diag = torch.zeros((self.kl, M, 3), **f64)
        self.state_out = None if self.last else self.sweep.new_state()
        self.bspec = spec.beams
        # this stage's particles of every beam: (7, n) columns, the ones whose ngp slice lies in the slab
        self.cols = []
        for b, (parts, gref, xiref) in zip(spec.beams, beams):
            c = torch.from_numpy(np.ascontiguousarray(parts.T)).to(self.device)
            self.cols.append(c[:, self._inside(c)].contiguous())
        self.started = [0] * len(beams)
        self.refs = [(gref, xiref) for _, gref, xiref in beams]
        self.outbox = [torch.zeros((7, 0), **f64) for _ in beams]
        self.moments = []
        self.counts = {"lost": 0, "trapped": 0, "nonfinite": 0}

    def _slice(self, cols):
        import torch

        return torch.floor((cols[5] - self.spec.xi_min) / self.spec.dxi + 0.5)

    def _inside(self, cols):
        k = self._slice(cols)
        return (k >= 0) & (k < self.kl)

    def step(self, n: int, dt: float, msg: Optional[Message], push: bool) -> Message:
        """Time step n: sweep (from msg), moments, push; returns the message for the next stage (None
        from the last stage)."""
        import torch

        if msg is not None:
            for q, b in enumerate(msg.beams):
                if b.shape[1]:
                    self.cols[q] = torch.cat([self.cols[q], b], dim=1).contiguous()
        self.bsrc.zero_()
        for b, c in zip(self.bspec, self.cols):
            if c.shape[1]:
                if self.fx is not None:
                    Q.BeamOps.deposit_fx(self.grid, c, b.q, b.m, self.box, self.fx, self.bsrc)
                else:
                    Q.BeamOps.deposit(self.grid, c, b.q, b.m, self.box, self.bsrc)
        state_in = None
        if msg is not None:
            state_in = msg.state
            state_in.pushed = msg.pushed
        cnt = self.sweep.run_stage(self.bsrc, self.fld, self.diag, guard=None if msg is None else msg.guard,
                                   state_in=state_in, state_out=self.state_out)
        for k in self.counts:
            self.counts[k] += cnt[k]
        out = None
        if not self.last:
            last = self.bsrc[:, self.kl - 1] if self.fx is not None else self.bsrc[self.kl - 1]
            out = Message(self.state_out, True, last.contiguous().clone(), self.outbox)
            self.outbox = [torch.zeros((7, 0), dtype=torch.float64, device=self.device) for _ in self.cols]
        mom = torch.zeros((len(self.cols), 17), dtype=torch.float64, device=self.device)
        for q, c in enumerate(self.cols):
            if c.shape[1]:
                Q.BeamOps.sums(c, self.refs[q][0], self.refs[q][1], mom[q])
        self.moments.append(mom)
        if push:
            fld = self.fld.reshape(-1)
            for q, (b, c) in enumerate(zip(self.bspec, self.cols)):
                if not c.shape[1] or b.rigid:
                    continue
                w0 = c[6].clone()
                self.started[q] = Q.BeamOps.push(self.grid, c, b.q, b.m, self.box, fld, dt, dt, self.started[q],
                                                 pusher=b.pusher)
                # the push removes what it finds outside the slab; a particle that is only outside the slab
                # (inside the wall and the box: its ngp slice lies half a slice ahead of the slab's first one,
                # or it moved past the slab's end) lives on, the latter in the next stage
                R = float(self.spec.nodes[-1])
                moved = (w0 != 0) & (c[6] == 0) & (c[0] * c[0] + c[1] * c[1] < R * R) & (c[5] <= self.xi_end)
                c[6] = torch.where(moved, w0, c[6])
                if not self.last:
                    gone = (self._slice(c) >= self.kl) & (c[6] != 0)
                    if bool(gone.any()):
                        self.outbox[q] = c[:, gone].contiguous()
                        self.cols[q] = c[:, ~gone].contiguous()
        return out


class Stages:
    """A staged run. With a DistChannel each rank holds one stage (rank = stage index); with a
    LocalChannel one process holds all the stages and runs them in turn within every step."""

    def __init__(self, spec, nstages: int, beams, ranks: Optional[Sequence[int]] = None, channel=None,
                 device=None, exact: bool = True):
        self.spec, self.nstages = spec, nstages
        self.local = channel is None or isinstance(channel, LocalChannel)
        self.channel = channel if channel is not None else LocalChannel()
        mine = list(range(nstages)) if ranks is None else list(ranks)
        bound = Q.ExactSources.bound([p for p, _, _ in beams], [b.q for b in spec.beams]) if exact else None
        if bound is not None and bound[1] > 1 << 25:
            bound = None                  # beyond 2^25 particles the run deposits with FP64 reductions
        self.stages = [Stage(spec, r, nstages, beams, device, bound) for r in mine]

    def run(self, nsteps: int, dt: float) -> np.ndarray:
        """nsteps time steps (nsteps + 1 sweeps); returns the moment sums (nsteps + 1, nbeams, 17) summed over
        the stages (on every rank)."""
        import torch

        for n in range(nsteps + 1):
            for st in self.stages:
                msg = None if st.first else self.channel.recv(st.rank - 1, st.rank, n)
                out = st.step(n, dt, msg, push=n < nsteps)
                if out is not None:
                    self.channel.send(st.rank + 1, n, out)
        mom = sum(torch.stack(st.moments) for st in self.stages)
        if not self.local:
            import torch.distributed as dist

            dist.all_reduce(mom)
        return mom.cpu().numpy()

    def fields(self):
        """Fields and diagnostics of the last sweep of this process's stages, slabs in box order."""
        import torch

        fld = torch.cat([st.fld for st in self.stages]).cpu().numpy()
        diag = torch.cat([st.diag for st in self.stages]).cpu().numpy()
        return fld, diag

    def beam(self, q: int) -> np.ndarray:
        """Beam q's particles of this process's stages, (n, 7)."""
        import torch

        return torch.cat([st.cols[q] for st in self.stages], dim=1).T.cpu().numpy()
