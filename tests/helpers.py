"""Shared test helpers: decks of the benchmark configurations (reduced where the oracle must stay
fast), field comparisons, and the reference's derived diagnostics."""
import os

import numpy as np

from quarz_b200 import deck

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

from quarz_b200.workloads import PLAIN_BLOWOUT as CONFIG0  # noqa: E402
from quarz_b200.workloads import pinched_witness_deck as config1_deck  # noqa: E402
from quarz_b200.workloads import pinched_witness_nodes as config1_nodes  # noqa: E402
from quarz_b200.workloads import spec_from_text  # noqa: E402,F401


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt(np.sum(b * b))
    num = np.sqrt(np.sum((a - b) ** 2))
    return num / den if den > 0 else num


def user_xi(spec):
    """xi axis of the field files (user convention, increasing; the head is the last row)."""
    K = spec.K
    return np.array([0.0 - (spec.xi_min + (K - 1 - k) * spec.dxi) for k in range(K)])


def bsum_numbers(spec, fld):
    """The numbers of validation/bsum.py: Ez on the axis at xi = -5, -7, -8, its minimum in (-9.5, -6)
    and (E_r - B_theta)/r at r = 0.5, xi = -6."""
    xi = user_xi(spec)
    ez = fld[::-1, 0, 4]
    r = spec.nodes
    m = (xi > -9.5) & (xi < -6)
    k = int(np.argmin(np.where(m, ez, 1e9)))
    at = lambda x: float(np.interp(x, xi, ez))  # noqa: E731
    ir = int(np.argmin(abs(r - 0.5)))
    wr = (fld[::-1, ir, 0] - fld[::-1, ir, 3]) / r[ir]
    return {"Ez(-5)": at(-5), "Ez(-7)": at(-7), "Ez(-8)": at(-8), "Ezmin": float(ez[k]), "xi_min": float(xi[k]),
            "Wr/r": float(np.interp(-6, xi, wr))}
