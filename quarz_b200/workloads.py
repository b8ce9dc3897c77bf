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
  scan              batched parameter scan: instances with N_r uniform in 128..1024 cells on stretched
                    grids (axis cell log-uniform in [5e-4, 5e-3], geometric to the wall r = 6), xi length
                    uniform in [8, 16] with dxi 0.01, driver n_b log-uniform in [1, 10], witness delay
                    log-uniform in [3, 6] behind the driver centre, witness/driver charge ratio
                    log-uniform in [0.05, 0.3] (set through the witness n_b, pinched-witness shape),
                    5e4 + 5e4 beam particles, dt 5, 20 steps, m = 0
  scan, modes = 1   the same draws with azimuthal modes m = 0, 1 (Picard 3, 4 azimuths per plasma ring,
                    driver offset 0.1 in x) and N_r uniform in 128..1023 cells: the m = 1 sweep keeps one
                    radial row per thread of a CTA of 512 threads, or 1024 above 512 nodes, so M <= 1024
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


def scan_nodes(n_nodes: int, h0: float, R: float = 6.0):
    """Geometric cells h_j = h0 q^j on [0, R] with exactly n_nodes nodes (q by bisection)."""
    ncell = n_nodes - 1
    lo, hi = 1.0, 2.0
    for _ in range(200):
        q = 0.5 * (lo + hi)
        tot = h0 * (q ** ncell - 1.0) / (q - 1.0) if q > 1.0 else h0 * ncell
        if tot < R:
            lo = q
        else:
            hi = q
    q = 0.5 * (lo + hi)
    hs = h0 * q ** np.arange(ncell)
    nodes = np.concatenate([[0.0], np.cumsum(hs)])
    nodes *= R / nodes[-1]
    nodes[-1] = R
    return nodes


def scan_instances(count: int = 512, seed: int = 2024, beam_particles: int = 100000, steps: int = 20,
                   modes: int = 0):
    """The instances of the batched scan, drawn from numpy's PCG64 with `seed` (see the module doc)."""
    rng = np.random.default_rng(seed)
    logu = lambda a, b: float(np.exp(rng.uniform(np.log(a), np.log(b))))  # noqa: E731
    out = []
    for i in range(count):
        ncell = int(rng.integers(128, 1025 if modes == 0 else 1024))
        h0 = logu(5e-4, 5e-3)
        L = float(rng.uniform(8.0, 16.0))
        n0d = logu(1.0, 10.0)
        delay = logu(3.0, 6.0)
        ratio = logu(0.05, 0.3)
        # witness n_b for the charge ratio: Q ~ n_b sigma_r^2 sigma_xi
        n0w = ratio * n0d * (0.5 ** 2 * 1.0) / (0.02 ** 2 * 0.1)
        half = beam_particles // 2
        text = f"""
xi.convention = z-t
grid.type = uniform
grid.rmax = 6
grid.dr = 1
xi.min = {-round(L / 0.01) * 0.01:.2f}
xi.max = 0
xi.step = 0.01
time.dt = 5
time.steps = {steps}
plasma.species = electrons
electrons.ppc = 1
beams = driver witness
driver.n0 = {n0d!r}
driver.sigma_r = 0.5
driver.sigma_xi = 1
driver.xi0 = -3
driver.gamma = 1000
driver.espread = 0.001
driver.emit_n = 0.05
driver.nparticles = {half}
driver.seed = {seed + 2 * i}
witness.n0 = {n0w!r}
witness.sigma_r = 0.02
witness.sigma_xi = 0.1
witness.xi0 = {-3.0 - delay!r}
witness.gamma = 1000
witness.emit_n = 1e-3
witness.nparticles = {beam_particles - half}
witness.seed = {seed + 2 * i + 1}
"""
        if modes == 1:
            text += "modes = 1\nsolver.picard = 3\nelectrons.ntheta = 4\ndriver.x0 = 0.1\n"
        spec = spec_from_text(text)
        spec.nodes = scan_nodes(ncell + 1, h0)
        out.append(spec)
    return out
