"""Mobile ion species (a second, positive mobile plasma species: plasma.species = electrons ions,
ions.charge = 1, ions.mass = 1836; with a positive species the background is not neutralised,
src/Simulation.cpp:124-134): one sweep and whole runs on the GPU against the oracle.

Decks: config 0's blowout cut to xi in [-6, 0] (256 + 256 plasma particles per slice: the register-resident
plasma of the sweep) and the pinched-witness grid cut to xi in [-9, 0] (511 + 511: the plasma state in
global memory). Tolerances as in tests/test_gpu_smoothing.py."""
import pytest

import quarz_b200 as Q
from helpers import CONFIG0
from quarz_b200 import workloads
from test_gpu_smoothing import _one_sweep, _runs_against_oracle

pytestmark = pytest.mark.gpu

IONS = ["plasma.species=electrons ions", "ions.charge=1", "ions.mass=1836", "ions.ppc=1"]


def _blowout_ions():
    return workloads.spec_from_text(CONFIG0, ["xi.min=-6", "driver.nparticles=20000", "time.steps=3"] + IONS)


def _pinched_ions():
    text = workloads.pinched_witness_deck(xi_min=-9.0, driver_np=20000, witness_np=20000, steps=2)
    return workloads.spec_from_text(text, IONS)


def test_ions_deck():
    spec = _blowout_ions()
    assert [s.q for s in spec.species] == [-1.0, 1.0] and not spec.neutralize
    assert all(s.mobile for s in spec.species)


def test_ions_one_sweep_register_plasma():
    _one_sweep(_blowout_ions())


def test_ions_one_sweep_global_plasma():
    _one_sweep(_pinched_ions())


def test_ions_runs_against_oracle():
    _runs_against_oracle(_blowout_ions(), 3)
    _runs_against_oracle(_pinched_ions(), 2)
