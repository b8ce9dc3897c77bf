"""quarz_b200 -- B200-native hot path of QUARZ (quasi-static xi sweep + beam push), FP64 CUDA for sm_100a.

The compute lives in libqz_b200.so (built from quarz_b200/csrc by quarz_b200.build). This package is
a thin ctypes layer over its C ABI (include/qz_b200.h) whose objects mirror the reference's C++ call
surface:

    RadialGrid   -> RadialGrid + FieldSolver set-up   (src/RadialGrid.cpp, src/FieldSolver.cpp)
    Sweep        -> Simulation::step_fields slice loop (src/Simulation.cpp:636-795)
    BeamOps      -> Beam::deposit / Beam::push / Beam::sums (src/Beam.cpp)
    Simulation   -> Simulation::run for constant dt    (src/Simulation.cpp:1370-1448)
    Batch        -> many independent Simulation::run in one launch (a parameter scan)

There is no CPU fallback: if the library cannot be loaded every entry point raises.
"""
from __future__ import annotations

from ._lib import QZError, lib, library_path  # noqa: F401
from .api import (Batch, BeamOps, ExactSources, RadialGrid, Simulation, Sweep, analytic_beam, sample_beam,  # noqa: F401
                  sample_gaussian, slice_table, sweep_params, write_fields)

__all__ = ["QZError", "lib", "library_path", "RadialGrid", "Sweep", "BeamOps", "ExactSources", "Simulation", "Batch",
           "sample_gaussian", "sample_beam", "sweep_params", "slice_table", "analytic_beam", "write_fields"]
