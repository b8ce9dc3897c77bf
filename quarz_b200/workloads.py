"""Named synthetic workloads (decks) of the benchmark configurations.

All are synthetic: seeded gaussian beams from the reference's generator, uniform cold plasma.
  plain_blowout     uniform 256 cells on r in [0, 6], xi length 12 with dxi 0.01 (1200 slices), ppc 1,
                    driver n_b 5 / sigma_r 0.5 / sigma_xi 1 / gamma 1000 / 0.1 % spread / emit_n 0.05,
                    1e5 particles, dt 10, 10 steps, m = 0
  pinched_witness   512 nodes geometric from 5e-4 at the axis to 0.05 at the wall r = 6 (ratio <= 1.02),
                    xi length 12 with dxi 0.005 (2400 slices), ppc 1; driver as above with 1e6 particles;
                    witness sigma_r 0.02 / sigma_xi 0.1 / 4.5 behind the driver / n_b 20 / gamma 1000 /
                    emit_n 1e-3, 1e6 particles; dt 5, 100 steps, m = 0
  hosing            the pinched-witness grid and box with azimuthal modes m = 0, 1 (Picard 3, 8 azimuths
                    per plasma ring: 4088 particles per slice); driver offset 0.1 in x and tilted 1e-3 in
                    x-xi, witness offset 0.02; 2e6 + 2e6 particles; dt 5, 200 steps
"""
from __future__ import annotations

import numpy as np

from . import deck

PLAIN_BLOWOUT = """
xi.convention = z-t
grid.type = uniform
grid.rmax = 6
grid.dr = 0.0234375
xi.min = -11.99
xi.max = 0
xi.step = 0.01
time.dt = 10
time.steps = 10
plasma.species = electrons
electrons.ppc = 1
beams = driver
driver.n0 = 5
driver.sigma_r = 0.5
driver.sigma_xi = 1
driver.xi0 = -3
driver.gamma = 1000
driver.espread = 0.001
driver.emit_n = 0.05
driver.nparticles = 100000
driver.seed = 1000
"""


def pinched_witness_nodes(n_nodes: int = 512, h0: float = 5e-4, hmax: float = 0.05, R: float = 6.0):
    """Geometric cells h_j = h0 q^j capped at hmax, exactly n_nodes nodes on [0, R]; q by bisection."""
    ncell = n_nodes - 1

    def total(q):
        h, s = h0, 0.0
        for _ in range(ncell):
            s += min(h, hmax)
            h *= q
        return s

    lo, hi = 1.0, 1.02
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if total(mid) < R:
            lo = mid
        else:
            hi = mid
    q = 0.5 * (lo + hi)
    hs, h = [], h0
    for _ in range(ncell):
        hs.append(min(h, hmax))
        h *= q
    nodes = np.concatenate([[0.0], np.cumsum(hs)])
    nodes *= R / nodes[-1]
    nodes[-1] = R
    return nodes, q


def pinched_witness_deck(xi_min: float = -11.995, driver_np: int = 1000000, witness_np: int = 1000000,
                         steps: int = 100) -> str:
    return f"""
xi.convention = z-t
grid.type = file
grid.file = PINCHED_WITNESS_GRID
xi.min = {xi_min}
xi.max = 0
xi.step = 0.005
time.dt = 5
time.steps = {steps}
plasma.species = electrons
electrons.ppc = 1
beams = driver witness
driver.n0 = 5
driver.sigma_r = 0.5
driver.sigma_xi = 1
driver.xi0 = -3
driver.gamma = 1000
driver.espread = 0.001
driver.emit_n = 0.05
driver.nparticles = {driver_np}
driver.seed = 1000
witness.n0 = 20
witness.sigma_r = 0.02
witness.sigma_xi = 0.1
witness.xi0 = -7.5
witness.gamma = 1000
witness.emit_n = 1e-3
witness.nparticles = {witness_np}
witness.seed = 1001
"""


def hosing_deck(xi_min: float = -11.995, driver_np: int = 2000000, witness_np: int = 2000000,
                steps: int = 200) -> str:
    return pinched_witness_deck(xi_min, driver_np, witness_np, steps) + """
modes = 1
solver.picard = 3
electrons.ntheta = 8
driver.x0 = 0.1
driver.x_slope = 1e-3
witness.x0 = 0.02
"""


def spec_from_text(text: str, overrides=()) -> deck.RunSpec:
    """RunSpec of a deck; grid.file = PINCHED_WITNESS_GRID selects the generated 512-node grid."""
    cfg = deck.parse_deck(text, overrides)
    if cfg.get("grid.file") == "PINCHED_WITNESS_GRID":
        cfg.pop("grid.file")
        cfg["grid.type"] = "uniform"
        cfg["grid.rmax"] = "6"
        cfg["grid.dr"] = "1"
        spec = deck.run_spec(cfg)
        spec.nodes = pinched_witness_nodes()[0]
        return spec
    return deck.run_spec(cfg)


def plain_blowout() -> deck.RunSpec:
    return spec_from_text(PLAIN_BLOWOUT)


def pinched_witness(**kw) -> deck.RunSpec:
    return spec_from_text(pinched_witness_deck(**kw))


def hosing(**kw) -> deck.RunSpec:
    return spec_from_text(hosing_deck(**kw))
