"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's hot path in plain C (oracle/qz_oracle.c). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may import this module, and
only to check results or to time the reference algorithm on the host cores. The product
(quarz_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libqz_oracle.so")
# the timing build: per-particle loops on all host threads (OpenMP), for the CPU baseline only; the
# parity checks use the serial build, whose summation order is fixed
OMP_LIB_PATH = os.path.join(HERE, "build", "libqz_oracle_omp.so")

THOMAS, PCR, PARTITION = 0, 1, 2
_METHODS = {"auto": THOMAS, "thomas": THOMAS, "pcr": PCR, "partition": PARTITION}


def build(omp: bool = False) -> str:
    subprocess.run(["make", "-s", "-C", HERE] + (["omp"] if omp else []), check=True)
    return OMP_LIB_PATH if omp else LIB_PATH


class _Params(C.Structure):
    _fields_ = [("modes", C.c_int), ("picard", C.c_int), ("ab_order", C.c_int), ("delta_min", C.c_double),
                ("max_qsa", C.c_double), ("xi_min", C.c_double), ("dxi", C.c_double), ("K", C.c_int),
                ("ngp", C.c_int), ("tridiag", C.c_int), ("neutralize", C.c_int), ("smooth_length", C.c_double),
                ("max_cells", C.c_double), ("substep_max", C.c_int)]


class _SpParams(C.Structure):
    _fields_ = [("q", C.c_double), ("m", C.c_double), ("ppc", C.c_int), ("ntheta", C.c_int), ("mobile", C.c_int),
                ("density", C.c_double), ("rmax", C.c_double), ("channel_depth", C.c_double),
                ("channel_radius", C.c_double)]


_lib = None
_use_omp = False


def use_openmp(on: bool = True):
    """Select the OpenMP timing build for every later call (before the first one)."""
    global _use_omp
    if _lib is not None and on != _use_omp:
        raise RuntimeError("oracle library already loaded")
    _use_omp = on


def lib():
    global _lib
    if _lib is None:
        path = OMP_LIB_PATH if _use_omp else LIB_PATH
        if not os.path.exists(path):
            build(_use_omp)
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        L.qzo_sim_create.restype = C.c_void_p
        L.qzo_sim_create.argtypes = [C.POINTER(_Params), dp, C.c_int]
        L.qzo_sim_destroy.argtypes = [C.c_void_p]
        L.qzo_sim_add_species.argtypes = [C.c_void_p, C.POINTER(_SpParams)]
        L.qzo_sim_add_beam.argtypes = [C.c_void_p, dp, C.c_long, C.c_double, C.c_double, C.c_int, C.c_double,
                                       C.c_double]
        L.qzo_sim_step_fields.argtypes = [C.c_void_p, C.c_double]
        L.qzo_sim_push_beams.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.qzo_sim_beam_sums.argtypes = [C.c_void_p, C.c_int, dp]
        L.qzo_sim_beam_get.argtypes = [C.c_void_p, C.c_int, dp]
        L.qzo_sim_beam_count.argtypes = [C.c_void_p, C.c_int]
        L.qzo_sim_beam_count.restype = C.c_long
        for f in ("qzo_sim_fld", "qzo_sim_bsrc", "qzo_sim_diag"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = dp
        L.qzo_sim_lost.argtypes = [C.c_void_p]
        L.qzo_sim_lost.restype = C.c_long
        L.qzo_sim_subslices.argtypes = [C.c_void_p]
        L.qzo_sim_subslices.restype = C.c_long
        L.qzo_sim_plasma_get.argtypes = [C.c_void_p, C.c_int, dp, C.c_int]
        L.qzo_sim_run.argtypes = [C.c_void_p, C.c_int, C.c_double, dp]
        L.qzo_sim_deposit_beams.argtypes = [C.c_void_p]
        L.qzo_sim_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_double, dp, dp, dp]
        L.qzo_sample_gaussian.restype = C.c_long
        L.qzo_sample_gaussian.argtypes = [C.c_double] * 14 + [C.c_long, C.c_int, C.c_int, C.c_uint64, C.c_double,
                                                              dp, dp, dp]
        L.qzo_tridiag.argtypes = [C.c_int, C.c_int, dp, dp, dp, dp, dp]
        L.qzo_filter.argtypes = [dp, C.c_int, C.c_double, C.c_int, dp]
        L.qzo_push.argtypes = [C.c_int, C.c_long, dp, dp, dp, dp, dp]
        L.qzo_slice_sums.argtypes = [dp, C.c_long, C.c_double, C.c_double, C.c_int, dp]
        L.qzo_sim_set_beam_pusher.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.qzo_bessel_i01_scaled.argtypes = [C.c_double, dp, dp]
        L.qzo_sim_add_analytic_beam.argtypes = [C.c_void_p] + [C.c_double] * 5 + [C.c_int] + [C.c_double] * 7
        L.qzo_field_solve.argtypes = [dp, C.c_int, C.c_int, C.c_int, dp, dp, dp, C.c_double, dp]
        L.qzo_operator_rows.argtypes = [dp, C.c_int, C.c_int, dp, dp, dp, dp]
        L.qzo_stencils.argtypes = [dp, C.c_int, dp, dp, dp, dp]
        L.qzo_grid_volumes.argtypes = [dp, C.c_int, dp]
        L.qzo_vay.argtypes = [dp, dp, dp, C.c_double, dp]
        L.qzo_ab_coeffs.argtypes = [C.c_int, dp]
        L.qzo_ab_variable.argtypes = [C.c_int, dp, C.c_double, dp]
        L.qzo_make_uniform.argtypes = [C.c_double, C.c_double, dp, C.c_int]
        L.qzo_make_regions.argtypes = [C.c_double, dp, dp, C.c_int, C.c_double, dp, C.c_int]
        L.qzo_rng_seed.argtypes = [C.c_void_p, C.c_uint64]
        L.qzo_rng_u64.argtypes = [C.c_void_p]
        L.qzo_rng_u64.restype = C.c_uint64
        L.qzo_rng_normal.argtypes = [C.c_void_p]
        L.qzo_rng_normal.restype = C.c_double
        L.qzo_rng_canonical.argtypes = [C.c_void_p]
        L.qzo_rng_canonical.restype = C.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- stand-alone pieces
def tridiag(a, b, c, d, method="thomas"):
    a, b, c, d = map(_c, (a, b, c, d))
    x = np.zeros_like(d)
    lib().qzo_tridiag(_METHODS[method], len(d), _p(a), _p(b), _p(c), _p(d), _p(x))
    return x


def push(kind, u, E, B, eps):
    """The beam pushers of src/Pushers.hpp on rows of momenta: kind 0 vay, 1 boris, 2 hc, 3 imp."""
    u, E, B = (_c(np.atleast_2d(a)) for a in (u, E, B))
    eps = _c(np.broadcast_to(np.asarray(eps, dtype=np.float64), (len(u),)))
    out = np.zeros_like(u)
    if lib().qzo_push(int(kind), len(u), _p(u), _p(E), _p(B), _p(eps), _p(out)) != 0:
        raise ValueError("qzo_push: kind must be 0..3")
    return out


def slice_sums(p7, lo, hi, nbins):
    """Beam::slice_sums of (n, 7) particle rows: (nbins, 9) sums over bins of the user xi in [lo, hi)."""
    p7 = _c(p7)
    out = np.zeros(9 * int(nbins))
    if lib().qzo_slice_sums(_p(p7), len(p7), float(lo), float(hi), int(nbins), _p(out)) != 0:
        raise ValueError("qzo_slice_sums: need nbins >= 1 and hi > lo")
    return out.reshape(int(nbins), 9)


def smooth(nodes, a2, n, f):
    """The radial smoothing filter F_n^{-1} f with a^2 = a2 in every cell (FieldSolver::filter)."""
    nodes, out = _c(nodes), _c(f).copy()
    if lib().qzo_filter(_p(nodes), len(nodes), float(a2), int(n), _p(out)) != 0:
        raise ValueError("qzo_filter failed")
    return out


def bessel_i01_scaled(z):
    """(e^-z I0(z), e^-z I1(z)) by Abramowitz & Stegun 9.8.1-9.8.4."""
    a, b = np.zeros(1), np.zeros(1)
    lib().qzo_bessel_i01_scaled(float(z), _p(a), _p(b))
    return float(a[0]), float(b[0])


def field_solve(nodes, op, rhs, chi=None, wall=None, scale=1.0, method="thomas"):
    nodes, rhs = _c(nodes), _c(rhs)
    f = np.zeros_like(rhs)
    chi_p = _p(_c(chi)) if chi is not None else None
    chi_a = _c(chi) if chi is not None else None
    wall_a = _c(wall) if wall is not None else None
    lib().qzo_field_solve(_p(nodes), len(nodes), {"L0": 0, "L1D": 1, "L1F": 2, "L2D": 3}[op], _METHODS[method],
                          _p(rhs), _p(chi_a) if chi_a is not None else None,
                          _p(wall_a) if wall_a is not None else None, float(scale), _p(f))
    del chi_p
    return f


def operator_rows(nodes, op):
    nodes = _c(nodes)
    M = len(nodes)
    a, b, c = np.zeros(M), np.zeros(M), np.zeros(M)
    fc = np.zeros(1)
    lib().qzo_operator_rows(_p(nodes), M, {"L0": 0, "L1D": 1, "L1F": 2, "L2D": 3}[op], _p(a), _p(b), _p(c), _p(fc))
    return a, b, c, float(fc[0])


def stencils(nodes):
    nodes = _c(nodes)
    M = len(nodes)
    out = [np.zeros(M) for _ in range(4)]
    lib().qzo_stencils(_p(nodes), M, *[_p(o) for o in out])
    return out


def volumes(nodes):
    nodes = _c(nodes)
    V = np.zeros(len(nodes))
    lib().qzo_grid_volumes(_p(nodes), len(nodes), _p(V))
    return V


def vay(u, E, B, eps):
    u, E, B = _c(u), _c(E), _c(B)
    out = np.zeros(3)
    lib().qzo_vay(_p(u), _p(E), _p(B), float(eps), _p(out))
    return out


def ab_coeffs(order):
    c = np.zeros(5)
    lib().qzo_ab_coeffs(order, _p(c))
    return c


def ab_variable(order, t, h):
    t = _c(t)
    c = np.zeros(5)
    lib().qzo_ab_variable(order, _p(t), float(h), _p(c))
    return c


def make_uniform(R, dr):
    out = np.zeros(10_000_000 if False else int(R / dr) + 16)
    n = lib().qzo_make_uniform(float(R), float(dr), _p(out), len(out))
    return out[:n].copy()


def make_regions(R, regions, max_ratio, cap=2_000_000):
    ends = _c([e for e, _ in regions])
    hs = _c([h for _, h in regions])
    out = np.zeros(cap)
    n = lib().qzo_make_regions(float(R), _p(ends), _p(hs), len(regions), float(max_ratio), _p(out), cap)
    if n < 0:
        raise ValueError("make_regions failed")
    return out[:n].copy()


class Rng:
    """The reference's std::mt19937_64 + std::normal_distribution, restated."""

    def __init__(self, seed: int):
        self._buf = C.create_string_buffer(312 * 8 + 32)
        lib().qzo_rng_seed(self._buf, C.c_uint64(seed))

    def u64(self) -> int:
        return int(lib().qzo_rng_u64(self._buf))

    def normal(self) -> float:
        return float(lib().qzo_rng_normal(self._buf))

    def canonical(self) -> float:
        return float(lib().qzo_rng_canonical(self._buf))


def sample_gaussian(n0, sr, xi0, sxi, gamma0, espread, emit, cut, cx0, cy0, cxs, cys, xp0, yp0, np, nrot, mirror,
                    seed, xcut):
    """The reference's gaussian beam generator; returns (particles (n,7) internal xi, gref, xiref)."""
    out = _np.zeros((int(np), 7))
    gref, xiref = _np.zeros(1), _np.zeros(1)
    n = lib().qzo_sample_gaussian(n0, sr, xi0, sxi, gamma0, espread, emit, cut, cx0, cy0, cxs, cys, xp0, yp0,
                                  int(np), int(nrot), int(mirror), C.c_uint64(int(seed)), xcut, _p(out), _p(gref),
                                  _p(xiref))
    if n < 0:
        raise ValueError(f"sample_gaussian failed ({n})")
    return out[:n], float(gref[0]), float(xiref[0])


_np = np


# ---------------------------------------------------------------- whole-deck simulation
class OracleSim:
    """The reference's Simulation (single rank) on a RunSpec from quarz_b200.deck."""

    def __init__(self, spec, beams=None, tridiag=None):
        self.spec = spec
        p = _Params(modes=spec.modes, picard=spec.picard, ab_order=spec.ab_order, delta_min=spec.delta_min,
                    max_qsa=spec.max_qsa, xi_min=spec.xi_min, dxi=spec.dxi, K=spec.K, ngp=1 if spec.ngp else 0,
                    tridiag=_METHODS[tridiag or spec.tridiag], neutralize=1 if spec.neutralize else 0,
                    smooth_length=getattr(spec, "smooth_length", 0.0),
                    max_cells=getattr(spec, "max_cells", 0.0), substep_max=getattr(spec, "substep_max", 64))
        self._nodes = _c(spec.nodes)
        self.h = lib().qzo_sim_create(C.byref(p), _p(self._nodes), len(self._nodes))
        if not self.h:
            raise RuntimeError("qzo_sim_create failed")
        for sp in spec.species:
            sp_p = _SpParams(q=sp.q, m=sp.m, ppc=sp.ppc, ntheta=sp.ntheta, mobile=1 if sp.mobile else 0,
                             density=sp.density, rmax=sp.rmax, channel_depth=sp.channel_depth,
                             channel_radius=sp.channel_radius)
            lib().qzo_sim_add_species(self.h, C.byref(sp_p))
        self.beam_data = []
        for i, b in enumerate(spec.beams):
            if b.analytic:
                self.beam_data.append((np.zeros((0, 7)), 0.0, 0.0))
                xcut = (0.0 - b.xi_cut_head_user) if b.xi_cut_head_user is not None else -1e300
                rc = lib().qzo_sim_add_analytic_beam(self.h, b.q, b.n0, b.sigma_r, 0.0 - b.xi0_user, b.sigma_xi,
                                                     1 if b.sigma_xi <= 0 else 0, b.flattop_length, xcut, b.x0,
                                                     b.y0, -b.x_slope, -b.y_slope, b.gamma)
                if rc != 0:
                    raise ValueError("qzo_sim_add_analytic_beam failed")
                continue
            if beams is not None:
                parts, gref, xiref = beams[i]
            else:
                from quarz_b200.deck import sampler_args
                parts, gref, xiref = sample_gaussian(**sampler_args(b))
            parts = _c(parts)
            self.beam_data.append((parts, gref, xiref))
            lib().qzo_sim_add_beam(self.h, _p(parts), len(parts), b.q, b.m, 1 if b.rigid else 0, gref, xiref)
            lib().qzo_sim_set_beam_pusher(self.h, i, getattr(b, "pusher", 0))
        M, K = spec.M, spec.K
        self.fnc = 18 if spec.modes == 1 else 6
        self.bnc = 15 if spec.modes == 1 else 5
        self.dnc = 9 if spec.modes == 1 else 3

    def __del__(self):
        if getattr(self, "h", None):
            lib().qzo_sim_destroy(self.h)
            self.h = None

    def step_fields(self, t=0.0):
        lib().qzo_sim_step_fields(self.h, float(t))

    def deposit_beams(self):
        lib().qzo_sim_deposit_beams(self.h)

    def push_beams(self, dkick, ddrift):
        lib().qzo_sim_push_beams(self.h, float(dkick), float(ddrift))

    def run(self, nsteps, dt):
        nb = len(self.spec.beams)
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        lib().qzo_sim_run(self.h, int(nsteps), float(dt), _p(mom))
        return mom[:, :nb, :]

    def adjoint(self, nsteps, dt, lamS):
        """Runs nsteps (like run) and then the adjoint: lamS (nbeams, 17) is the adjoint of the last
        step's moment sums. Returns (per beam its (n, 7) adjoint of the initial particles, moments)."""
        nb = len(self.spec.beams)
        counts = [int(lib().qzo_sim_beam_count(self.h, b)) for b in range(nb)]
        lam = np.zeros(7 * sum(counts) + 1)
        mom = np.zeros((nsteps + 1, max(nb, 1), 17))
        seeds = np.ascontiguousarray(np.asarray(lamS, dtype=np.float64).reshape(nb, 17))
        rc = lib().qzo_sim_adjoint(self.h, int(nsteps), float(dt), _p(seeds), _p(lam), _p(mom))
        if rc != 0:
            raise ValueError("qzo_sim_adjoint: deck outside the adjoint's scope (m = 0, linear xi shape, one "
                             "mobile species, fresh beams)")
        out, off = [], 0
        for n in counts:
            out.append(lam[7 * off:7 * (off + n)].reshape(n, 7).copy())
            off += n
        return out, mom[:, :nb, :]

    def _view(self, f, nc):
        ptr = getattr(lib(), f)(self.h)
        n = self.spec.K * self.spec.M * nc
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self.spec.K, self.spec.M, nc).copy()

    def fld(self):
        return self._view("qzo_sim_fld", self.fnc)

    def bsrc(self):
        return self._view("qzo_sim_bsrc", self.bnc)

    def diag(self):
        return self._view("qzo_sim_diag", self.dnc)

    def lost(self):
        return int(lib().qzo_sim_lost(self.h))

    def subslices(self):
        """Sub-slices beyond the regular slices so far (adaptive sub-slicing)."""
        return int(lib().qzo_sim_subslices(self.h))

    def beam(self, b):
        n = lib().qzo_sim_beam_count(self.h, b)
        out = np.zeros((n, 7))
        lib().qzo_sim_beam_get(self.h, b, _p(out))
        return out

    def beam_sums(self, b):
        out = np.zeros(17)
        lib().qzo_sim_beam_sums(self.h, b, _p(out))
        return out

    def plasma(self, sp=0):
        cap = self.spec.M * 64 * 64
        out = np.zeros(6 * cap)
        n = lib().qzo_sim_plasma_get(self.h, sp, _p(out), cap)
        return out[: 6 * n].reshape(6, n)


def from_sums(S, gref, xiref, m1=False):
    """Beam::from_sums (src/Beam.cpp:1157-1192) -> dict of beam diagnostics (user xi convention)."""
    d = {"alive": S[16]}
    sw = S[0]
    if sw <= 0:
        return d
    m = lambda c: S[c + 1] / sw  # noqa: E731
    d["gamma_mean"] = gref + m(0)
    d["gamma_rms"] = np.sqrt(max(0.0, m(1) - m(0) * m(0)))
    d["xi_mean"] = 0.0 - (xiref + m(2))
    d["xi_rms"] = np.sqrt(max(0.0, m(3) - m(2) * m(2)))
    d["r_rms"] = np.sqrt(m(4))
    d["x_mean"], d["y_mean"] = m(5), m(6)
    xx, yy = m(7) - m(5) * m(5), m(8) - m(6) * m(6)
    pxx, pyy = m(11) - m(9) * m(9), m(12) - m(10) * m(10)
    xpx, ypy = m(13) - m(5) * m(9), m(14) - m(6) * m(10)
    if not m1:
        d["x_mean"] = d["y_mean"] = 0.0
        xx = yy = 0.5 * m(4)
        pxx = pyy = 0.5 * (m(11) + m(12))
        xpx = ypy = 0.5 * (m(13) + m(14))
    d["sigma_x"] = np.sqrt(max(0.0, xx))
    d["sigma_y"] = np.sqrt(max(0.0, yy))
    d["emit_nx"] = np.sqrt(max(0.0, xx * pxx - xpx * xpx))
    d["emit_ny"] = np.sqrt(max(0.0, yy * pyy - ypy * ypy))
    d["charge_w"] = sw
    return d
