"""The reference's printed validation numbers reproduced by the CUDA path (through the C ABI), the
same checks the oracle passes in tests/test_oracle_linear.py and tests/test_oracle_pins.py:

- section 1: the linear wake of a weak driver against its Green's function, uniform and stretched
  grids (four printed digits of each error);
- section 4: the witness energy gain rate of the rigid-driver blowout over 20 steps (0.4477), through
  the pipelined run.
"""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from test_gpu_parity import _gpu_sweep
from test_oracle_linear import LINEAR_DECKS, check_linear
from test_oracle_pins import VAL, _deck

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["uniform", "stretched"])
def test_gpu_linear_wake(name):
    spec = _deck("linear.in", LINEAR_DECKS[name])
    beams = [Q.sample_beam(b) for b in spec.beams]
    _, fld, diag, _, _ = _gpu_sweep(spec, beams)
    check_linear(name, fld, diag, spec)


def test_gpu_gain_full():
    spec = _deck("gain.in")
    beams = [Q.sample_beam(b) for b in spec.beams]
    sim = Q.Simulation(spec, beams=beams)
    sim.set_schedule(True)
    mom = sim.run(spec.steps, spec.dt)
    bi = [b.name for b in spec.beams].index("witness")
    _, gref, xiref = beams[bi]
    t = np.arange(spec.steps + 1) * spec.dt
    g = np.array([O.from_sums(mom[n, bi], gref, xiref)["gamma_mean"] for n in range(spec.steps + 1)])
    assert f"{np.polyfit(t, g, 1)[0]:.4f}" == VAL["gain_full"]
