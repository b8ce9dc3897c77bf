"""Input decks: the `key = value` format of QUARZ and the derived run set-up.

Only the keys that reach the hot path are interpreted (grid, box, plasma species, particle
beams, pusher / solver options, time stepping). Semantics follow the reference:

  * deck syntax and command-line overrides        src/Config.cpp, src/main.cpp:82-93
  * grid generators (uniform / regions / file)    src/RadialGrid.cpp:14-86
  * box: internal xi = -xi_user, K = lround(L/dxi)+1   src/Simulation.cpp:69-77, src/Types.hpp:30-31
  * species defaults (ppc 4, ntheta 8 with m = 1)  src/PlasmaSpecies.cpp:92-150
  * beam keys of the gaussian generator           src/Beam.cpp:483-570
  * neutralising background when no positive species   src/Simulation.cpp:124-134
  * radial smoothing of the plasma sources (plasma.smooth_length)   src/Simulation.cpp:63-66
  * analytic rigid beams (<beam>.analytic = 1)     src/Beam.cpp:183-203

Keys this module does not know raise ``ValueError`` (the reference's strict unknown-key check,
src/main.cpp:100-116, restricted to the hot-path subset).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# Keys understood here. A deck key outside this set (after expanding <species>/<beam> names)
# is an error, as in the reference.
_GLOBAL_KEYS = {
    "xi.convention", "grid.type", "grid.rmax", "grid.dr", "grid.regions", "grid.max_ratio", "grid.file",
    "xi.min", "xi.max", "xi.step", "time.dt", "time.steps", "time.start", "modes", "solver.picard",
    "solver.tridiag", "pusher.ab_order", "pusher.delta_min", "pusher.max_qsa_factor", "plasma.species",
    "pusher.max_cells_per_step", "pusher.substep_max",
    "plasma.seed", "plasma.neutralize", "plasma.rmax", "plasma.radial", "plasma.channel_depth",
    "plasma.channel_radius", "beams", "beams.xi_shape", "output.dir", "output.every", "pusher.beam",
    "plasma.smooth_length",
}
_SPECIES_KEYS = {"charge", "mass", "mobile", "ppc", "ntheta", "density"}
_BEAM_KEYS = {"n0", "sigma_r", "sigma_xi", "xi0", "gamma", "espread", "emit_n", "cut", "nparticles", "seed",
              "rigid", "charge", "mass", "x0", "y0", "x_slope", "y_slope", "xp0", "yp0", "nsym", "mirror_y",
              "profile", "length", "xi_cut_head", "pusher", "analytic"}


def parse_deck(text: str, overrides: Sequence[str] = ()) -> Dict[str, str]:
    """``key = value`` lines, ``#`` comments; later keys win; overrides are ``key=value`` strings."""
    cfg: Dict[str, str] = {}
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if "=" not in line:
            raise ValueError(f"deck: line without '=': {raw!r}")
        k, v = line.split("=", 1)
        cfg[k.strip()] = v.strip()
    for o in overrides:
        k, v = o.split("=", 1)
        cfg[k.strip()] = v.strip()
    return cfg


def read_deck(path: str, overrides: Sequence[str] = ()) -> Dict[str, str]:
    with open(path) as f:
        return parse_deck(f.read(), overrides)


def _b(v: str) -> bool:
    return v.strip().lower() in ("1", "true", "yes", "on")


# ---------------------------------------------------------------- grid generators
def make_uniform(R: float, dr: float) -> np.ndarray:
    """src/RadialGrid.cpp:139-145"""
    if R <= 0 or dr <= 0:
        raise ValueError("grid: R and dr must be positive")
    n = max(1, int(_lround(R / dr)))
    return np.array([R * float(j) / float(n) for j in range(n + 1)])


def _lround(x: float) -> int:
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def make_regions(R: float, regions: Sequence[Tuple[float, float]], max_ratio: float) -> np.ndarray:
    """src/RadialGrid.cpp:27-71"""
    if not regions:
        raise ValueError("grid: grid.regions is empty")
    if max_ratio < 1.0:
        raise ValueError("grid: grid.max_ratio must be >= 1")
    g = max_ratio - 1.0

    def target(x: float) -> float:
        ht = regions[-1][1]
        for e, h in regions:
            if x < e:
                ht = h
                break
        start = 0.0
        for e, h in regions:
            if start > x and g > 0:
                ht = min(ht, h + g * (start - x))
            if start > x and g == 0:
                ht = min(ht, h)
            start = e
        return ht

    nodes = [0.0]
    x, hprev = 0.0, target(0.0)
    while x < R * (1 - 1e-12):
        ht = target(x + 0.5 * hprev)
        lo, hi = hprev / max_ratio, hprev * max_ratio
        hnew = lo if ht < lo else (hi if hi < ht else ht)
        if len(nodes) == 1:
            hnew = target(0.0)
        x += hnew
        nodes.append(x)
        hprev = hnew
    if len(nodes) >= 3 and (nodes[-1] - R) > (R - nodes[-2]):
        nodes.pop()
    scale = R / nodes[-1]
    out = np.array([v * scale for v in nodes])
    out[-1] = R
    return out


def read_grid_file(path: str) -> np.ndarray:
    vals = []
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if line:
                vals.append(float(line))
    return np.array(vals)


def _pairs(v: str) -> List[Tuple[float, float]]:
    out = []
    for tok in v.replace(",", " ").split():
        a, b = tok.split(":")
        out.append((float(a), float(b)))
    return out


# ---------------------------------------------------------------- run set-up
@dataclass
class SpeciesSpec:
    name: str
    q: float = -1.0
    m: float = 1.0
    mobile: bool = True
    ppc: int = 4
    ntheta: int = 1
    density: float = 1.0
    rmax: float = 1e300
    channel_depth: float = 0.0
    channel_radius: float = 0.0


@dataclass
class BeamSpec:
    name: str
    n0: float = 0.0
    sigma_r: float = 1.0
    sigma_xi: float = 1.0       # > 0 gaussian; flattop uses length
    xi0_user: float = 0.0
    gamma: float = 1.0
    espread: float = 0.0
    emit_n: float = 0.0
    cut: float = 3.0
    nparticles: int = 100000
    seed: int = 12345
    rigid: bool = False
    q: float = -1.0
    m: float = 1.0
    x0: float = 0.0
    y0: float = 0.0
    x_slope: float = 0.0
    y_slope: float = 0.0
    xp0: float = 0.0
    yp0: float = 0.0
    nsym: int = 1
    mirror_y: bool = False
    flattop_length: float = 0.0
    xi_cut_head_user: Optional[float] = None
    analytic: bool = False      # noise-free rigid beam deposited on the grid, no particles
    pusher: int = 0             # <beam>.pusher / pusher.beam: 0 vay, 1 boris, 2 hc, 3 imp (src/Beam.cpp:72-78)


@dataclass
class RunSpec:
    nodes: np.ndarray
    modes: int = 0
    picard: int = 1
    ab_order: int = 3
    delta_min: float = 1e-3
    max_qsa: float = 35.0
    xi_min: float = 0.0          # internal xi of slice 0 (head)
    dxi: float = 0.01
    K: int = 1
    ngp: bool = False
    tridiag: str = "auto"
    neutralize: bool = True
    smooth_length: float = 0.0   # plasma.smooth_length (0: no smoothing)
    max_cells: float = 0.0       # pusher.max_cells_per_step: adaptive sub-slicing (0: off)
    substep_max: int = 64        # pusher.substep_max
    dt: float = 0.0
    steps: int = 0
    species: List[SpeciesSpec] = field(default_factory=list)
    beams: List[BeamSpec] = field(default_factory=list)

    @property
    def M(self) -> int:
        return len(self.nodes)


def run_spec(cfg: Dict[str, str], base_dir: str = ".") -> RunSpec:
    """Interpret a parsed deck (raises ValueError on unknown or unsupported keys)."""
    species_names = cfg.get("plasma.species", "electrons").split() or ["electrons"]
    beam_names = cfg.get("beams", "").split()
    for k in cfg:
        if k in _GLOBAL_KEYS:
            continue
        head, _, tail = k.partition(".")
        if head in species_names and tail in _SPECIES_KEYS:
            continue
        if head in beam_names and tail in _BEAM_KEYS:
            continue
        raise ValueError(f"deck: unknown or unsupported key '{k}'")
    if cfg.get("xi.convention", "z-t") != "z-t":
        raise ValueError("xi.convention: only z-t is supported")

    gtype = cfg.get("grid.type", "uniform")
    if gtype == "uniform":
        nodes = make_uniform(float(cfg["grid.rmax"]), float(cfg["grid.dr"]))
    elif gtype in ("regions", "stretched"):
        nodes = make_regions(float(cfg["grid.rmax"]), _pairs(cfg["grid.regions"]),
                             float(cfg.get("grid.max_ratio", "1.05")))
    elif gtype == "file":
        p = cfg["grid.file"]
        nodes = read_grid_file(p if os.path.isabs(p) else os.path.join(base_dir, p))
    else:
        raise ValueError(f"grid: unknown grid.type '{gtype}'")

    modes = int(cfg.get("modes", "0"))
    if modes not in (0, 1):
        raise ValueError("modes must be 0 or 1")
    xu_max = float(cfg.get("xi.max", "0"))
    xu_min = float(cfg["xi.min"])
    dxi = float(cfg["xi.step"])
    if not (xu_max > xu_min) or not dxi > 0:
        raise ValueError("xi: need xi.min < xi.max and xi.step > 0")
    K = _lround((xu_max - xu_min) / dxi) + 1
    shape = cfg.get("beams.xi_shape", "linear")
    if shape not in ("linear", "ngp"):
        raise ValueError("beams.xi_shape must be linear or ngp")

    spec = RunSpec(
        nodes=np.asarray(nodes, dtype=np.float64),
        modes=modes,
        picard=int(cfg.get("solver.picard", "3" if modes == 1 else "1")),
        ab_order=int(cfg.get("pusher.ab_order", "3")),
        delta_min=float(cfg.get("pusher.delta_min", "1e-3")),
        max_qsa=float(cfg.get("pusher.max_qsa_factor", "35")),
        xi_min=0.0 - xu_max,
        dxi=dxi,
        K=K,
        ngp=(shape == "ngp"),
        tridiag=cfg.get("solver.tridiag", "auto"),
        dt=float(cfg.get("time.dt", "0")),
        steps=int(cfg.get("time.steps", "0")),
    )
    spec.max_cells = float(cfg.get("pusher.max_cells_per_step", "0"))
    spec.substep_max = int(cfg.get("pusher.substep_max", "64"))
    if spec.max_cells < 0 or spec.substep_max < 1:     # src/Simulation.cpp:51-54
        raise ValueError("pusher.max_cells_per_step must be >= 0 and pusher.substep_max >= 1")
    spec.smooth_length = float(cfg.get("plasma.smooth_length", "0"))
    if spec.smooth_length < 0:
        raise ValueError("plasma.smooth_length must be >= 0")
    if not 1 <= spec.ab_order <= 5:
        raise ValueError("pusher.ab_order must be 1..5")

    has_positive = False
    for n in species_names:
        sp = SpeciesSpec(name=n)
        sp.q = float(cfg.get(n + ".charge", "-1"))
        sp.m = float(cfg.get(n + ".mass", "1"))
        sp.mobile = _b(cfg.get(n + ".mobile", "1"))
        sp.ppc = int(cfg.get(n + ".ppc", "4"))
        sp.ntheta = int(cfg.get(n + ".ntheta", "8" if modes == 1 else "1"))
        sp.density = float(cfg.get(n + ".density", "1"))
        sp.rmax = float(cfg.get("plasma.rmax", "1e300"))
        rad = cfg.get("plasma.radial", "uniform")
        if rad == "channel":
            sp.channel_depth = float(cfg["plasma.channel_depth"])
            sp.channel_radius = float(cfg["plasma.channel_radius"])
        elif rad != "uniform":
            raise ValueError(f"plasma.radial '{rad}' is not on this path")
        if sp.ppc < 1:
            raise ValueError(n + ".ppc must be >= 1")
        if modes == 1 and sp.ntheta < 4:
            raise ValueError(n + ".ntheta must be >= 4 with azimuthal mode 1")
        if sp.q > 0:
            has_positive = True
        spec.species.append(sp)
    spec.neutralize = _b(cfg.get("plasma.neutralize", "0" if has_positive else "1"))

    for n in beam_names:
        b = BeamSpec(name=n)
        prof = cfg.get(n + ".profile", "gaussian")
        b.n0 = float(cfg[n + ".n0"])
        b.sigma_r = float(cfg[n + ".sigma_r"])
        if prof == "gaussian":
            b.sigma_xi = float(cfg[n + ".sigma_xi"])
        elif prof == "flattop":
            b.sigma_xi = -1.0
            b.flattop_length = float(cfg[n + ".length"])
        else:
            raise ValueError(f"{n}.profile '{prof}' is not on this path")
        b.xi0_user = float(cfg[n + ".xi0"])
        b.gamma = float(cfg[n + ".gamma"])
        b.espread = float(cfg.get(n + ".espread", "0"))
        b.emit_n = float(cfg.get(n + ".emit_n", "0"))
        b.cut = float(cfg.get(n + ".cut", "3"))
        b.nparticles = int(float(cfg.get(n + ".nparticles", "100000")))
        b.seed = int(cfg.get(n + ".seed", "12345"))
        b.rigid = _b(cfg.get(n + ".rigid", "0"))
        b.analytic = _b(cfg.get(n + ".analytic", "0"))
        if b.analytic:
            b.rigid = True
        b.q = float(cfg.get(n + ".charge", "-1"))
        b.m = float(cfg.get(n + ".mass", "1"))
        b.x0 = float(cfg.get(n + ".x0", "0"))
        b.y0 = float(cfg.get(n + ".y0", "0"))
        b.x_slope = float(cfg.get(n + ".x_slope", "0"))
        b.y_slope = float(cfg.get(n + ".y_slope", "0"))
        b.xp0 = float(cfg.get(n + ".xp0", "0"))
        b.yp0 = float(cfg.get(n + ".yp0", "0"))
        b.nsym = int(cfg.get(n + ".nsym", "1"))
        b.mirror_y = _b(cfg.get(n + ".mirror_y", "0"))
        if n + ".xi_cut_head" in cfg:
            b.xi_cut_head_user = float(cfg[n + ".xi_cut_head"])
        pm = cfg.get(n + ".pusher", cfg.get("pusher.beam", "vay"))
        if pm not in PUSHERS:
            raise ValueError(f"{n}.pusher must be vay|boris|hc|imp (imp_rr, radiation reaction, is not on this path)")
        b.pusher = PUSHERS[pm]
        if modes == 0 and any(v != 0 for v in (b.x0, b.y0, b.x_slope, b.y_slope, b.xp0, b.yp0)):
            raise ValueError(n + ": transverse offsets/tilts need azimuthal mode 1 (modes = 1)")
        spec.beams.append(b)
    return spec


PUSHERS = {"vay": 0, "boris": 1, "hc": 2, "imp": 3}


def sampler_args(b: BeamSpec) -> dict:
    """Arguments of the gaussian generator in internal coordinates (src/Beam.cpp:486-512)."""
    return dict(
        n0=b.n0, sr=b.sigma_r, xi0=0.0 - b.xi0_user,
        sxi=b.sigma_xi if b.sigma_xi > 0 else -b.flattop_length,
        gamma0=b.gamma, espread=b.espread, emit=b.emit_n, cut=b.cut,
        cx0=b.x0, cy0=b.y0, cxs=-b.x_slope, cys=-b.y_slope, xp0=b.xp0, yp0=b.yp0,
        np=b.nparticles, nrot=b.nsym, mirror=1 if b.mirror_y else 0, seed=b.seed,
        xcut=(0.0 - b.xi_cut_head_user) if b.xi_cut_head_user is not None else -1e300,
    )
