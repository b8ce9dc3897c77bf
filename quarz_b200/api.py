"""Python objects over the C ABI of libqz_b200 (names follow the reference's classes).

Device memory is handled with torch tensors (float64, cuda) purely as plumbing: the kernels receive
raw device pointers through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import deck as _deck
from ._lib import AnalyticBeam, BeamView, Box, Counters, PlasmaState, QZError, Species, SweepParams, check, lib

_dp = C.POINTER(C.c_double)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream))


def _dev(t) -> int:
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise QZError(1, "expected a contiguous float64 CUDA tensor")
    return t.data_ptr()


# ---------------------------------------------------------------- grid
class RadialGrid:
    """Radial grid, node volumes, operator rows and stencils on the device (qz_grid)."""

    def __init__(self, nodes: Sequence[float]):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        h = C.c_void_p()
        check(lib().qz_grid_create(_p(self.nodes), len(self.nodes), C.byref(h)))
        self.h = h

    @property
    def M(self) -> int:
        return len(self.nodes)

    def volumes(self) -> np.ndarray:
        V = np.zeros(self.M)
        check(lib().qz_grid_volumes(self.h, _p(V)))
        return V

    def operator(self, op: str):
        k = {"L0": 0, "L1D": 1, "L1F": 2, "L2D": 3}[op]
        a, b, c, fc = np.zeros(self.M), np.zeros(self.M), np.zeros(self.M), np.zeros(1)
        check(lib().qz_grid_operator(self.h, k, _p(a), _p(b), _p(c), _p(fc)))
        return a, b, c, float(fc[0])

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:
            try:
                lib().qz_grid_destroy(self.h)
            except Exception:
                pass
            self.h = None


def sweep_params(spec: "_deck.RunSpec") -> SweepParams:
    """qz_sweep_params from a RunSpec (quarz_b200.deck)."""
    p = SweepParams()
    p.modes = spec.modes
    p.picard = spec.picard
    p.ab_order = spec.ab_order
    p.delta_min = spec.delta_min
    p.max_qsa = spec.max_qsa
    p.xi_min = spec.xi_min
    p.dxi = spec.dxi
    p.K = spec.K
    p.ngp = 1 if spec.ngp else 0
    p.neutralize = 1 if spec.neutralize else 0
    p.smooth_length = float(getattr(spec, "smooth_length", 0.0))
    p.max_cells_per_step = float(getattr(spec, "max_cells", 0.0))
    p.substep_max = int(getattr(spec, "substep_max", 64))
    if len(spec.species) > 4:
        raise QZError(1, "at most 4 plasma species")
    p.nspecies = len(spec.species)
    for i, sp in enumerate(spec.species):
        p.species[i] = Species(q=sp.q, m=sp.m, ppc=sp.ppc, ntheta=sp.ntheta, mobile=1 if sp.mobile else 0,
                               density=sp.density, rmax=sp.rmax, channel_depth=sp.channel_depth,
                               channel_radius=sp.channel_radius)
    return p


# ---------------------------------------------------------------- sweep
class ExactSources:
    """The node quanta of exact (two-limb, order-independent) beam sources (qz_fx): for beams whose
    sum over beams of max |w q| is at most wq and that hold at most nparticles particles in all."""

    def __init__(self, grid: RadialGrid, dxi: float, wq: float, nparticles: int):
        self.grid = grid
        h = C.c_void_p()
        check(lib().qz_fx_create(grid.h, float(dxi), float(wq), int(nparticles), C.byref(h)))
        self.h = h

    @staticmethod
    def bound(beams, charges) -> Tuple[float, int]:
        """(wq, particles) of beams given as (n, 7) rows (weight last) with their charges, in the order
        qz_sim sums them."""
        wq, n = 0.0, 0
        for rows, q in zip(beams, charges):
            if len(rows):
                wq += float(np.max(np.abs(rows[:, 6]))) * abs(float(q))
            n += len(rows)
        return wq, n

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().qz_fx_destroy(self.h)
            except Exception:
                pass
            self.h = None


class Sweep:
    """One quasi-static sweep per call (qz_sweep)."""

    def __init__(self, grid: RadialGrid, params: SweepParams):
        self.grid = grid
        self.params = params
        h = C.c_void_p()
        check(lib().qz_sweep_create(grid.h, C.byref(params), C.byref(h)))
        self.h = h

    def run(self, bsrc, fld, diag, stream=None) -> int:
        cnt = Counters()
        check(lib().qz_sweep_run(self.h, _dev(bsrc), _dev(fld), _dev(diag), C.byref(cnt), _stream_ptr(stream)))
        self.last_counters = {"lost": int(cnt.lost), "nonfinite": int(cnt.nonfinite), "trapped": int(cnt.trapped),
                              "subslices": int(cnt.subslices)}
        return int(cnt.lost)

    def set_exact_sources(self, fx: Optional["ExactSources"]) -> None:
        """qz_sweep_set_exact_sources: read bsrc (2, K, M, 5) and the guard row (2, M, 5) as exact limbs
        (None: plain doubles)."""
        check(lib().qz_sweep_set_exact_sources(self.h, fx.h if fx is not None else None))
        self._fx = fx

    def run_async(self, bsrc, fld, diag, stream=None) -> None:
        check(lib().qz_sweep_run(self.h, _dev(bsrc), _dev(fld), _dev(diag), None, _stream_ptr(stream)))

    def state_shape(self) -> Tuple[int, int, int]:
        """(np, npad, AB order) of the plasma state a slab hands on (qz_sweep_state_shape)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().qz_sweep_state_shape(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def new_state(self):
        """An empty plasma state for this sweep: a (6 + 5 order, npad) float64 CUDA tensor with its pushed
        flag (attribute .pushed)."""
        import torch

        np_, npad, order = self.state_shape()
        t = torch.zeros((6 + 5 * order, npad), dtype=torch.float64, device="cuda")
        t.pushed = False
        return t

    def _state(self, t) -> PlasmaState:
        np_, npad, order = self.state_shape()
        if tuple(t.shape) != (6 + 5 * order, npad):
            raise QZError(1, f"plasma state of shape {tuple(t.shape)}, the sweep's is {(6 + 5 * order, npad)}")
        return PlasmaState(state=_dev(t), np=np_, npad=npad, order=order, pushed=1 if getattr(t, "pushed", False) else 0)

    def run_stage(self, bsrc, fld, diag, guard=None, state_in=None, state_out=None, stream=None) -> dict:
        """qz_sweep_run_stage: one slab of a xi-pipelined sweep. state_in / state_out: plasma states
        (new_state()); guard: the beam sources of the slice ahead of the slab (M x 5 CUDA tensor) or None.
        Returns the counters of the sweep."""
        cnt = Counters()
        sin = self._state(state_in) if state_in is not None else None
        sout = self._state(state_out) if state_out is not None else None
        check(lib().qz_sweep_run_stage(self.h, _dev(bsrc), _dev(guard) if guard is not None else None,
                                       C.byref(sin) if sin is not None else None, _dev(fld), _dev(diag),
                                       C.byref(sout) if sout is not None else None, C.byref(cnt), _stream_ptr(stream)))
        if state_out is not None:
            state_out.pushed = True
        return {"lost": int(cnt.lost), "nonfinite": int(cnt.nonfinite), "trapped": int(cnt.trapped),
                "subslices": int(cnt.subslices)}

    def plasma(self) -> np.ndarray:
        cap = 1 << 22
        out = np.zeros(6 * cap)
        n = C.c_int()
        check(lib().qz_sweep_plasma(self.h, _p(out), cap, C.byref(n)))
        return out[: 6 * n.value].reshape(6, n.value)

    def timing(self, enable: bool = True) -> np.ndarray:
        cyc = (C.c_ulonglong * 16)()
        check(lib().qz_sweep_timing(self.h, 1 if enable else 0, cyc))
        return np.array(list(cyc), dtype=np.float64)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().qz_sweep_destroy(self.h)
            except Exception:
                pass
            self.h = None


# ---------------------------------------------------------------- beams
class BeamOps:
    """Beam deposit / push / sums on 7 device columns (tensor (7, n): x y px py pz xi w)."""

    @staticmethod
    def view(cols, q: float, m: float, pusher: int = 0) -> BeamView:
        base = _dev(cols)
        n = cols.shape[1]
        v = BeamView()
        for c, name in enumerate(("x", "y", "px", "py", "pz", "xi", "w")):
            setattr(v, name, base + 8 * n * c)
        v.n, v.q, v.m, v.pusher = n, q, m, int(pusher)
        return v

    @staticmethod
    def box(xi_min: float, dxi: float, K: int, ngp: bool = False, modes: int = 0) -> Box:
        return Box(xi_min=xi_min, dxi=dxi, K=K, ngp=1 if ngp else 0, modes=modes)

    @staticmethod
    def deposit(grid: RadialGrid, cols, q, m, box: Box, bsrc, stream=None):
        v = BeamOps.view(cols, q, m)
        check(lib().qz_beam_deposit(grid.h, C.byref(v), C.byref(box), _dev(bsrc), _stream_ptr(stream)))

    @staticmethod
    def deposit_fx(grid: RadialGrid, cols, q, m, box: Box, fx: ExactSources, bsrc2, stream=None):
        """qz_beam_deposit_fx: adds the beam into exact two-limb sources bsrc2 (2, K, M, 5)."""
        v = BeamOps.view(cols, q, m)
        check(lib().qz_beam_deposit_fx(grid.h, C.byref(v), C.byref(box), fx.h, _dev(bsrc2), _stream_ptr(stream)))

    @staticmethod
    def advance(grid, cols, q, m, box, fld, dt_kick, dt_drift, move, stream=None, pusher: int = 0):
        v = BeamOps.view(cols, q, m, pusher)
        check(lib().qz_beam_advance(grid.h, C.byref(v), C.byref(box), _dev(fld), dt_kick, dt_drift, int(move),
                                    _stream_ptr(stream)))

    @staticmethod
    def push(grid, cols, q, m, box, fld, dt_kick, dt_drift, started: int, stream=None, pusher: int = 0) -> int:
        v = BeamOps.view(cols, q, m, pusher)
        st = C.c_int(started)
        check(lib().qz_beam_push(grid.h, C.byref(v), C.byref(box), _dev(fld), dt_kick, dt_drift, C.byref(st),
                                 _stream_ptr(stream)))
        return st.value

    @staticmethod
    def push_deposit(grid, cols, q, m, box, fld, dt_kick, dt_drift, started: int, bsrc_next, stream=None,
                     pusher: int = 0) -> int:
        v = BeamOps.view(cols, q, m, pusher)
        st = C.c_int(started)
        check(lib().qz_beam_push_deposit(grid.h, C.byref(v), C.byref(box), _dev(fld), dt_kick, dt_drift,
                                         C.byref(st), _dev(bsrc_next), _stream_ptr(stream)))
        return st.value

    @staticmethod
    def deposit_analytic(grid: RadialGrid, b: "_deck.BeamSpec", box: Box, bsrc, stream=None):
        """qz_beam_deposit_analytic: adds an analytic beam's sources to bsrc."""
        a = analytic_beam(b)
        check(lib().qz_beam_deposit_analytic(grid.h, C.byref(a), C.byref(box), _dev(bsrc), _stream_ptr(stream)))

    @staticmethod
    def slice_sums(cols, lo: float, hi: float, nbins: int, out, stream=None):
        """qz_beam_slice_sums: 9 sums per bin of the user xi over [lo, hi) into out (9 * nbins, device)."""
        v = BeamOps.view(cols, -1.0, 1.0)
        check(lib().qz_beam_slice_sums(C.byref(v), float(lo), float(hi), int(nbins), _dev(out), _stream_ptr(stream)))

    @staticmethod
    def sums(cols, gref, xiref, out17, stream=None):
        v = BeamOps.view(cols, -1.0, 1.0)
        check(lib().qz_beam_sums(C.byref(v), gref, xiref, _dev(out17), _stream_ptr(stream)))

    @staticmethod
    def sums_noalloc(cols, gref, xiref, out17, stream=None):
        """qz_beam_sums_noalloc: the same sums with no device allocation (static scratch)."""
        v = BeamOps.view(cols, -1.0, 1.0)
        check(lib().qz_beam_sums_noalloc(C.byref(v), gref, xiref, _dev(out17), _stream_ptr(stream)))


def sample_gaussian(n0, sr, xi0, sxi, gamma0, espread, emit, cut, cx0, cy0, cxs, cys, xp0, yp0, np_, nrot, mirror,
                    seed, xcut) -> Tuple[np.ndarray, float, float]:
    """The reference's gaussian beam generator (std::mt19937_64 + std::normal_distribution), on the host."""
    out = np.zeros((int(np_), 7))
    gref, xiref = np.zeros(1), np.zeros(1)
    n = C.c_int64()
    check(lib().qz_sample_gaussian(n0, sr, xi0, sxi, gamma0, espread, emit, cut, cx0, cy0, cxs, cys, xp0, yp0,
                                   int(np_), int(nrot), int(mirror), C.c_uint64(int(seed)), xcut, _p(out), _p(gref),
                                   _p(xiref), C.byref(n)))
    return out[: n.value], float(gref[0]), float(xiref[0])


def sample_beam(b: "_deck.BeamSpec"):
    """The beam's particles (n, 7), gref, xiref; an analytic beam has none."""
    if b.analytic:
        return np.zeros((0, 7)), 0.0, 0.0
    a = _deck.sampler_args(b)
    a["np_"] = a.pop("np")
    return sample_gaussian(**a)


def slice_table(B: np.ndarray, q: float, lo: float, hi: float) -> np.ndarray:
    """The columns of the reference's slices file (Beam::write_slices_file, src/Beam.cpp:1219-1236) from the
    (nbins, 9) slice sums: xi, charge, x_mean, y_mean, sigma_x, sigma_y, gamma_mean, emit_nx, one row per
    bin with charge (empty bins are left out, as there)."""
    B = np.asarray(B, dtype=np.float64).reshape(-1, 9)
    nb = len(B)
    db = (hi - lo) / nb
    rows = []
    for b in range(nb):
        sw = B[b, 0]
        if sw <= 0:
            continue
        m = B[b] / sw
        xx, yy = m[3] - m[1] * m[1], m[4] - m[2] * m[2]
        pxx, xpx = m[7] - m[6] * m[6], m[8] - m[1] * m[6]
        rows.append([lo + (b + 0.5) * db, q * sw, m[1], m[2], np.sqrt(max(0.0, xx)), np.sqrt(max(0.0, yy)), m[5],
                     np.sqrt(max(0.0, xx * pxx - xpx * xpx))])
    return np.array(rows).reshape(-1, 8)


def write_fields(path: str, spec: "_deck.RunSpec", fld: np.ndarray, diag: np.ndarray, bsrc=None,
                 t: float = 0.0) -> None:
    """qz_write_fields from host arrays: the reference's fields_NNNNNN.bin (version 3) of one sweep."""
    nodes = np.ascontiguousarray(spec.nodes, dtype=np.float64)
    box = Box(xi_min=spec.xi_min, dxi=spec.dxi, K=spec.K, ngp=1 if spec.ngp else 0, modes=spec.modes)
    F = np.ascontiguousarray(fld, dtype=np.float64)
    D = np.ascontiguousarray(diag, dtype=np.float64)
    B = None if bsrc is None else np.ascontiguousarray(bsrc, dtype=np.float64)
    check(lib().qz_write_fields(str(path).encode(), _p(nodes), len(nodes), C.byref(box), float(t), F.ctypes.data,
                                D.ctypes.data, None if B is None else B.ctypes.data, 0))


def analytic_beam(b: "_deck.BeamSpec") -> AnalyticBeam:
    """qz_analytic_beam of an analytic deck beam, in internal coordinates."""
    flat = b.sigma_xi <= 0
    return AnalyticBeam(q=b.q, n0=b.n0, sigma_r=b.sigma_r, xi0=0.0 - b.xi0_user, sigma_xi=0.0 if flat else b.sigma_xi,
                        flattop=1 if flat else 0, length=b.flattop_length,
                        xi_cut=(0.0 - b.xi_cut_head_user) if b.xi_cut_head_user is not None else -1e300,
                        x0=b.x0, y0=b.y0, x_slope=-b.x_slope, y_slope=-b.y_slope, gamma=b.gamma)


# ---------------------------------------------------------------- whole time steps
class Simulation:
    """Simulation::run for constant dt on one GPU (qz_sim): sweeps, moments, fused push + deposit.

    Beams are indexed as in the deck. Analytic beams have no particles: their moment rows are zero and their
    adjoint has no rows; inside qz_sim they are static sources, not beams."""

    def __init__(self, spec: "_deck.RunSpec", beams: Optional[List[Tuple[np.ndarray, float, float]]] = None):
        self.spec = spec
        self.grid = RadialGrid(spec.nodes)
        self.params = sweep_params(spec)
        h = C.c_void_p()
        check(lib().qz_sim_create(self.grid.h, C.byref(self.params), C.byref(h)))
        self.h = h
        self.beam_data = []
        self._cidx = []                 # deck beam -> index of the particle beam in qz_sim (None: analytic)
        for i, b in enumerate(spec.beams):
            if b.analytic:
                a = analytic_beam(b)
                check(lib().qz_sim_add_analytic_beam(self.h, C.byref(a)))
                self.beam_data.append((np.zeros((0, 7)), 0.0, 0.0))
                self._cidx.append(None)
                continue
            parts, gref, xiref = beams[i] if beams is not None else sample_beam(b)
            parts = np.ascontiguousarray(parts, dtype=np.float64)
            self.beam_data.append((parts, gref, xiref))
            check(lib().qz_sim_add_beam(self.h, _p(parts), len(parts), b.q, b.m, 1 if b.rigid else 0, gref, xiref))
            self._cidx.append(sum(c is not None for c in self._cidx))
            if getattr(b, "pusher", 0):
                check(lib().qz_sim_set_beam_pusher(self.h, self._cidx[-1], int(b.pusher)))
        self._pb = [i for i, c in enumerate(self._cidx) if c is not None]   # deck indices of particle beams
        self.fnc = 18 if spec.modes else 6
        self.dnc = 9 if spec.modes else 3

    def _expand(self, mom_c: np.ndarray) -> np.ndarray:
        """moments of the particle beams (steps, npb, 17) -> one row per deck beam (analytic rows zero)"""
        out = np.zeros((mom_c.shape[0], len(self.spec.beams), 17))
        for c, i in enumerate(self._pb):
            out[:, i] = mom_c[:, c]
        return out

    def _c(self, b: int) -> int:
        c = self._cidx[b]
        if c is None:
            raise QZError(1, f"beam {b} is analytic: it has no particles")
        return c

    def run(self, nsteps: int, dt: float, stream=None) -> np.ndarray:
        nb = len(self._pb)
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        check(lib().qz_sim_run(self.h, int(nsteps), float(dt), _p(mom) if nb else None, _stream_ptr(stream)))
        return self._expand(mom[:, :nb, :])

    def set_schedule(self, pipelined: bool = True, sweep_ctas: int = 0, bucket: int = 0, span: int = 0,
                     timeout_s: float = 0.0):
        """qz_sim_set_schedule: pipelined (one launch for the whole run) or step by step."""
        check(lib().qz_sim_set_schedule(self.h, 1 if pipelined else 0, int(sweep_ctas), int(bucket), int(span),
                                        float(timeout_s)))

    def restart(self):
        """qz_sim_restart: the next run starts the beams' leapfrog again (a new run from set beams)."""
        check(lib().qz_sim_restart(self.h))

    def set_adjoint_checkpoint(self, every: int = 0):
        """qz_sim_set_adjoint_checkpoint: slice checkpointing of the pipelined adjoint (0: every
        ceil(sqrt(K))-th slice, 1: every slice, C > 1: every C-th)."""
        check(lib().qz_sim_set_adjoint_checkpoint(self.h, int(every)))

    def set_exact(self, exact: bool = True):
        """qz_sim_set_exact: exact (reproducible) or FP64-reduction beam deposits for m = 0 runs."""
        check(lib().qz_sim_set_exact(self.h, 1 if exact else 0))

    def schedule(self) -> dict:
        """The schedule of the last run (qz_sim_schedule)."""
        info = (C.c_int * 8)()
        check(lib().qz_sim_schedule(self.h, info))
        keys = ("grid", "sweep_ctas", "push_ctas", "ring", "buckets", "bucket", "pipelined", "span")
        return dict(zip(keys, list(info)))

    def times(self) -> dict:
        """GPU ms of the parts of the last pipelined run (qz_sim_times)."""
        t = np.zeros(3)
        check(lib().qz_sim_times(self.h, _p(t)))
        return {"setup_ms": t[0], "kernel_ms": t[1], "finish_ms": t[2]}

    def set_beam(self, b: int, cols, stream=None) -> None:
        """qz_sim_set_beam: beam b's particles from a (7, n) float64 array, numpy (host) or torch (device)."""
        if isinstance(cols, np.ndarray):
            cols = np.ascontiguousarray(cols, dtype=np.float64)
            check(lib().qz_sim_set_beam(self.h, self._c(int(b)), cols.ctypes.data, 0, _stream_ptr(stream)))
        else:
            check(lib().qz_sim_set_beam(self.h, self._c(int(b)), _dev(cols), 1, _stream_ptr(stream)))

    def trace(self, enable: bool = True) -> np.ndarray:
        """Timeline of the last pipelined run (qz_sim_trace): per step (start, end, 16 progress marks, longest
        wait) in ns of GPU clock, and the push workers' 6 totals (tasks, empty scans, lost claims, ns in tasks,
        ns waiting for a task, ns in moments passes); enable turns the recording on for later runs."""
        n = C.c_int()
        check(lib().qz_sim_trace(self.h, 1 if enable else 0, None, 0, C.byref(n)))
        out = (C.c_ulonglong * max(n.value, 1))()
        check(lib().qz_sim_trace(self.h, 1 if enable else 0, out, n.value, C.byref(n)))
        v = np.array(list(out)[: n.value], dtype=np.float64)
        return v[:-6].reshape(-1, 22), v[-6:]

    def run_host(self, nsteps: int, dt: float, cols_host, stream=None) -> np.ndarray:
        """qz_sim_run_host: the particle beams in host memory (list of (7, n) float64 arrays in deck order,
        analytic beams left out, updated in place)."""
        nb = len(self._pb)
        ptrs = (C.c_void_p * max(nb, 1))(*[int(c.ctypes.data) if isinstance(c, np.ndarray) else int(c.data_ptr())
                                           for c in cols_host])
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        check(lib().qz_sim_run_host(self.h, int(nsteps), float(dt), ptrs, _p(mom) if nb else None,
                                    _stream_ptr(stream)))
        return self._expand(mom[:, :nb, :])

    def timing(self, enable: bool = True) -> np.ndarray:
        """qz_sim_timing: the 16 phase-cycle counters of the stand-alone sweeps; enables or disables them."""
        out = (C.c_ulonglong * 16)()
        check(lib().qz_sim_timing(self.h, 1 if enable else 0, out))
        return np.array(list(out), dtype=np.uint64)

    def adjoint(self, nsteps: int, dt: float, lamS, stream=None):
        """qz_sim_adjoint: runs nsteps (step by step, keeping the beams of every step) and the reverse
        pass. lamS (nbeams, 17): the adjoint of the last step's moment sums. Returns (per beam its (n, 7)
        adjoint of the initial particles (x y px py pz xi w), the forward's moment sums, (forward ms,
        reverse ms))."""
        nbd = len(self.spec.beams)
        seeds_d = np.asarray(lamS, dtype=np.float64).reshape(nbd, 17)
        pb = self._pb
        nb = len(pb)
        seeds = np.ascontiguousarray(seeds_d[pb] if nb else np.zeros((1, 17)))
        cols = [np.zeros((7, len(self.beam_data[b][0]))) for b in range(nbd)]
        ptrs = (C.c_void_p * max(nb, 1))(*[int(cols[b].ctypes.data) for b in pb])
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        ms = np.zeros(2)
        check(lib().qz_sim_adjoint(self.h, int(nsteps), float(dt), _p(seeds), ptrs, _p(mom), _p(ms),
                                   _stream_ptr(stream)))
        return [c.T.copy() for c in cols], self._expand(mom[:, :nb, :]), (float(ms[0]), float(ms[1]))

    def adjoint_fn(self, nsteps: int, dt: float, seed_fn, stream=None):
        """qz_sim_adjoint_fn: as adjoint(), with the seed computed after the forward by
        seed_fn(moments ((nsteps+1), nbeams, 17)) -> (nbeams, 17)."""
        nbd = len(self.spec.beams)
        pb = self._pb
        nb = len(pb)
        SEED = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p)
        err = []

        def _cb(mom_p, ns, nbm, out_p, _user):
            try:
                mom = np.ctypeslib.as_array(mom_p, shape=((ns + 1) * nbm * 17,)).reshape(ns + 1, nbm, 17).copy()
                seeds = np.asarray(seed_fn(self._expand(mom)), dtype=np.float64).reshape(nbd, 17)[pb]
                out = np.ctypeslib.as_array(out_p, shape=(nbm * 17,))
                out[:] = seeds.reshape(nbm * 17)
            except Exception as e:                      # a Python error must not unwind through C
                err.append(e)

        cb = SEED(_cb)
        cols = [np.zeros((7, len(self.beam_data[b][0]))) for b in range(nbd)]
        ptrs = (C.c_void_p * max(nb, 1))(*[int(cols[b].ctypes.data) for b in pb])
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        ms = np.zeros(2)
        check(lib().qz_sim_adjoint_fn(self.h, int(nsteps), float(dt), C.cast(cb, C.c_void_p), None, ptrs, _p(mom),
                                      _p(ms), _stream_ptr(stream)))
        if err:
            raise err[0]
        return [c.T.copy() for c in cols], self._expand(mom[:, :nb, :]), (float(ms[0]), float(ms[1]))

    def fields(self):
        K, M = self.spec.K, self.spec.M
        fld = np.zeros(K * M * self.fnc)
        diag = np.zeros(K * M * self.dnc)
        check(lib().qz_sim_fields(self.h, _p(fld), _p(diag)))
        return fld.reshape(K, M, self.fnc), diag.reshape(K, M, self.dnc)

    def beam(self, b: int) -> np.ndarray:
        n = len(self.beam_data[b][0])
        out = np.zeros((n, 7))
        if self._cidx[b] is not None:
            check(lib().qz_sim_beam(self.h, self._cidx[b], _p(out)))
        return out

    def slice_sums(self, b: int, lo: float, hi: float, nbins: int) -> np.ndarray:
        """qz_sim_beam_slice_sums of deck beam b as it stands: (nbins, 9) over bins of the user xi in [lo, hi)."""
        out = np.zeros(9 * int(nbins))
        check(lib().qz_sim_beam_slice_sums(self.h, self._c(int(b)), float(lo), float(hi), int(nbins), _p(out)))
        return out.reshape(int(nbins), 9)

    def write_fields(self, path: str, t: float = 0.0) -> None:
        """qz_sim_write_fields: the field file of the last sweep."""
        check(lib().qz_sim_write_fields(self.h, float(t), str(path).encode()))

    def lost(self) -> int:
        return self.counters()["lost"]

    def counters(self) -> dict:
        """qz_sim_counters: plasma particles removed (of them trapped), deposits with a non-finite
        contribution, pipelined runs that gave up on a wait."""
        c = Counters()
        check(lib().qz_sim_counters(self.h, C.byref(c)))
        return {"lost": int(c.lost), "nonfinite": int(c.nonfinite), "trapped": int(c.trapped), "giveup": int(c.giveup),
                "subslices": int(c.subslices)}

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().qz_sim_destroy(self.h)
            except Exception:
                pass
            self.h = None


# ---------------------------------------------------------------- batched independent runs
class Batch:
    """Many independent runs (a parameter scan) in one persistent launch (qz_batch)."""

    def __init__(self):
        h = C.c_void_p()
        check(lib().qz_batch_create(C.byref(h)))
        self.h = h
        self.specs = []

    def add(self, spec: "_deck.RunSpec", beams: Optional[List[Tuple[np.ndarray, float, float]]] = None) -> int:
        beams = beams if beams is not None else [sample_beam(b) for b in spec.beams]
        nb = len(spec.beams)
        rows = [np.ascontiguousarray(p, dtype=np.float64) for p, _, _ in beams]
        nodes = np.ascontiguousarray(spec.nodes, dtype=np.float64)
        params = sweep_params(spec)
        ptrs = (C.c_void_p * max(nb, 1))(*[r.ctypes.data for r in rows])
        n = (C.c_int64 * max(nb, 1))(*[len(r) for r in rows])
        q = np.array([b.q for b in spec.beams] or [0.0])
        m = np.array([b.m for b in spec.beams] or [1.0])
        rigid = (C.c_int * max(nb, 1))(*[1 if b.rigid else 0 for b in spec.beams])
        gref = np.array([g for _, g, _ in beams] or [0.0])
        xiref = np.array([x for _, _, x in beams] or [0.0])
        idx = C.c_int()
        check(lib().qz_batch_add(self.h, _p(nodes), len(nodes), C.byref(params), nb, ptrs, n, _p(q), _p(m), rigid,
                                 _p(gref), _p(xiref), C.byref(idx)))
        self.specs.append((spec, beams))
        return idx.value

    def run(self, nsteps: int, dt: float, stream=None) -> List[np.ndarray]:
        """Runs every instance; returns per instance its (nsteps+1, nbeams, 17) moment sums."""
        sizes = [(nsteps + 1) * max(1, len(sp.beams)) * 17 for sp, _ in self.specs]
        out = np.zeros(sum(sizes))
        check(lib().qz_batch_run(self.h, int(nsteps), float(dt), _p(out), _stream_ptr(stream)))
        res, off = [], 0
        for (sp, _), sz in zip(self.specs, sizes):
            res.append(out[off:off + sz].reshape(nsteps + 1, max(1, len(sp.beams)), 17)[:, :len(sp.beams)])
            off += sz
        return res

    def info(self) -> dict:
        v = np.zeros(4)
        check(lib().qz_batch_info(self.h, _p(v)))
        return {"instances": int(v[0]), "ctas": int(v[1]), "kernel_ms": float(v[2])}

    def set_tuning(self, index: int, layout: int = -1, cost: float = 0.0) -> None:
        """qz_batch_set_tuning: instance `index`'s shared-memory layout (bits: 1 double-buffered sources,
        2 constants in shared memory, 4 particle copy; -1 keeps it) and queue cost (<= 0 keeps it)."""
        check(lib().qz_batch_set_tuning(self.h, int(index), int(layout), float(cost)))

    def tuning(self, index: int) -> Tuple[int, float]:
        """qz_batch_tuning: (layout bits or -1 for modes = 1, queue cost) of instance `index`."""
        lay, cost = C.c_int(), np.zeros(1)
        check(lib().qz_batch_tuning(self.h, int(index), C.byref(lay), _p(cost)))
        return lay.value, float(cost[0])

    def set_trace(self, enable: bool = True) -> None:
        """qz_batch_set_trace: record the per-instance timeline of the next runs."""
        check(lib().qz_batch_set_trace(self.h, 1 if enable else 0))

    def trace(self) -> np.ndarray:
        """qz_batch_trace: (instances, 5) of the last traced run, in order of addition: CTA, start ms,
        end ms, ms in sweeps, ms in beam phases."""
        n = len(self.specs)
        out = np.zeros((max(n, 1), 5))
        check(lib().qz_batch_trace(self.h, _p(out), n))
        return out[:n]

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().qz_batch_destroy(self.h)
            except Exception:
                pass
            self.h = None
