"""Loading of libqz_b200.so and the ctypes declarations of its C ABI (include/qz_b200.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(HERE, "libqz_b200.so")


class QZError(RuntimeError):
    """An entry point of libqz_b200 returned a non-zero qz_status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"qz_status {code}: {msg}")
        self.code = code


class Species(C.Structure):
    _fields_ = [("q", C.c_double), ("m", C.c_double), ("ppc", C.c_int), ("ntheta", C.c_int), ("mobile", C.c_int),
                ("density", C.c_double), ("rmax", C.c_double), ("channel_depth", C.c_double),
                ("channel_radius", C.c_double)]


class SweepParams(C.Structure):
    _fields_ = [("modes", C.c_int), ("picard", C.c_int), ("ab_order", C.c_int), ("delta_min", C.c_double),
                ("max_qsa", C.c_double), ("xi_min", C.c_double), ("dxi", C.c_double), ("K", C.c_int),
                ("ngp", C.c_int), ("neutralize", C.c_int), ("nspecies", C.c_int), ("species", Species * 4),
                ("smooth_length", C.c_double), ("max_cells_per_step", C.c_double), ("substep_max", C.c_int)]


class Counters(C.Structure):
    _fields_ = [("lost", C.c_ulonglong), ("nonfinite", C.c_ulonglong), ("trapped", C.c_ulonglong),
                ("giveup", C.c_ulonglong), ("subslices", C.c_ulonglong)]


class PlasmaState(C.Structure):
    _fields_ = [("state", C.c_void_p), ("np", C.c_int), ("npad", C.c_int), ("order", C.c_int), ("pushed", C.c_int)]


class BeamView(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("px", C.c_void_p), ("py", C.c_void_p), ("pz", C.c_void_p),
                ("xi", C.c_void_p), ("w", C.c_void_p), ("n", C.c_int64), ("q", C.c_double), ("m", C.c_double),
                ("pusher", C.c_int)]


class Box(C.Structure):
    _fields_ = [("xi_min", C.c_double), ("dxi", C.c_double), ("K", C.c_int), ("ngp", C.c_int), ("modes", C.c_int)]


class AnalyticBeam(C.Structure):
    _fields_ = [("q", C.c_double), ("n0", C.c_double), ("sigma_r", C.c_double), ("xi0", C.c_double),
                ("sigma_xi", C.c_double), ("flattop", C.c_int), ("length", C.c_double), ("xi_cut", C.c_double),
                ("x0", C.c_double), ("y0", C.c_double), ("x_slope", C.c_double), ("y_slope", C.c_double),
                ("gamma", C.c_double)]


_lib = None
_dp = C.POINTER(C.c_double)

# (name, argtypes) of every entry point of include/qz_b200.h
SIGNATURES = {
    "qz_last_error": [],
    "qz_version": [],
    "qz_grid_create": [_dp, C.c_int, C.POINTER(C.c_void_p)],
    "qz_grid_destroy": [C.c_void_p],
    "qz_grid_volumes": [C.c_void_p, _dp],
    "qz_grid_operator": [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp],
    "qz_sweep_create": [C.c_void_p, C.POINTER(SweepParams), C.POINTER(C.c_void_p)],
    "qz_sweep_destroy": [C.c_void_p],
    "qz_sweep_run": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Counters), C.c_void_p],
    "qz_sweep_plasma": [C.c_void_p, _dp, C.c_int, C.POINTER(C.c_int)],
    "qz_sweep_state_shape": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "qz_sweep_run_stage": [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PlasmaState), C.c_void_p, C.c_void_p,
                           C.POINTER(PlasmaState), C.POINTER(Counters), C.c_void_p],
    "qz_sweep_timing": [C.c_void_p, C.c_int, C.POINTER(C.c_ulonglong)],
    "qz_beam_deposit": [C.c_void_p, C.POINTER(BeamView), C.POINTER(Box), C.c_void_p, C.c_void_p],
    "qz_fx_create": [C.c_void_p, C.c_double, C.c_double, C.c_int64, C.POINTER(C.c_void_p)],
    "qz_fx_destroy": [C.c_void_p],
    "qz_beam_deposit_fx": [C.c_void_p, C.POINTER(BeamView), C.POINTER(Box), C.c_void_p, C.c_void_p, C.c_void_p],
    "qz_sweep_set_exact_sources": [C.c_void_p, C.c_void_p],
    "qz_beam_advance": [C.c_void_p, C.POINTER(BeamView), C.POINTER(Box), C.c_void_p, C.c_double, C.c_double,
                        C.c_int, C.c_void_p],
    "qz_beam_push": [C.c_void_p, C.POINTER(BeamView), C.POINTER(Box), C.c_void_p, C.c_double, C.c_double,
                     C.POINTER(C.c_int), C.c_void_p],
    "qz_beam_push_deposit": [C.c_void_p, C.POINTER(BeamView), C.POINTER(Box), C.c_void_p, C.c_double, C.c_double,
                             C.POINTER(C.c_int), C.c_void_p, C.c_void_p],
    "qz_beam_deposit_analytic": [C.c_void_p, C.POINTER(AnalyticBeam), C.POINTER(Box), C.c_void_p, C.c_void_p],
    "qz_beam_slice_sums": [C.POINTER(BeamView), C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p],
    "qz_beam_sums": [C.POINTER(BeamView), C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    "qz_beam_sums_noalloc": [C.POINTER(BeamView), C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    "qz_sample_gaussian": [C.c_double] * 14 + [C.c_int64, C.c_int, C.c_int, C.c_uint64, C.c_double, _dp, _dp, _dp,
                                               C.POINTER(C.c_int64)],
    "qz_sim_create": [C.c_void_p, C.POINTER(SweepParams), C.POINTER(C.c_void_p)],
    "qz_sim_destroy": [C.c_void_p],
    "qz_sim_add_beam": [C.c_void_p, _dp, C.c_int64, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double],
    "qz_sim_add_analytic_beam": [C.c_void_p, C.POINTER(AnalyticBeam)],
    "qz_sim_set_beam_pusher": [C.c_void_p, C.c_int, C.c_int],
    "qz_sim_beam_slice_sums": [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, _dp],
    "qz_write_fields": [C.c_char_p, _dp, C.c_int, C.POINTER(Box), C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.c_int],
    "qz_sim_write_fields": [C.c_void_p, C.c_double, C.c_char_p],
    "qz_sim_run": [C.c_void_p, C.c_int, C.c_double, _dp, C.c_void_p],
    "qz_sim_fields": [C.c_void_p, _dp, _dp],
    "qz_sim_beam": [C.c_void_p, C.c_int, _dp],
    "qz_sim_counters": [C.c_void_p, C.POINTER(Counters)],
    "qz_sim_step_host": [C.c_void_p, C.POINTER(C.c_void_p), C.c_double, C.c_double, C.c_int, _dp, C.c_void_p],
    "qz_sim_restart": [C.c_void_p],
    "qz_sim_set_exact": [C.c_void_p, C.c_int],
    "qz_sim_set_adjoint_checkpoint": [C.c_void_p, C.c_int],
    "qz_sim_set_schedule": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double],
    "qz_sim_schedule": [C.c_void_p, C.POINTER(C.c_int)],
    "qz_sim_times": [C.c_void_p, _dp],
    "qz_sim_set_beam": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p],
    "qz_sim_trace": [C.c_void_p, C.c_int, C.POINTER(C.c_ulonglong), C.c_int, C.POINTER(C.c_int)],
    "qz_sim_run_host": [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_void_p), _dp, C.c_void_p],
    "qz_sim_timing": [C.c_void_p, C.c_int, C.POINTER(C.c_ulonglong)],
    "qz_sim_adjoint_fn": [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p), _dp, _dp,
                          C.c_void_p],
    "qz_sim_adjoint": [C.c_void_p, C.c_int, C.c_double, _dp, C.POINTER(C.c_void_p), _dp, _dp, C.c_void_p],
    "qz_batch_create": [C.POINTER(C.c_void_p)],
    "qz_batch_destroy": [C.c_void_p],
    "qz_batch_add": [C.c_void_p, _dp, C.c_int, C.POINTER(SweepParams), C.c_int, C.POINTER(C.c_void_p),
                     C.POINTER(C.c_int64), _dp, _dp, C.POINTER(C.c_int), _dp, _dp, C.POINTER(C.c_int)],
    "qz_batch_run": [C.c_void_p, C.c_int, C.c_double, _dp, C.c_void_p],
    "qz_batch_info": [C.c_void_p, _dp],
    "qz_batch_set_trace": [C.c_void_p, C.c_int],
    "qz_batch_set_tuning": [C.c_void_p, C.c_int, C.c_int, C.c_double],
    "qz_batch_tuning": [C.c_void_p, C.c_int, C.POINTER(C.c_int), _dp],
    "qz_batch_trace": [C.c_void_p, _dp, C.c_int],
}


def lib():
    """The loaded library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise QZError(-1, f"{library_path} is missing: build it with quarz_b200.build.build()")
        L = C.CDLL(library_path)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_char_p if name in ("qz_last_error", "qz_version") else C.c_int
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != 0:
        raise QZError(code, lib().qz_last_error().decode())
