"""Gradients of witness energy gain and energy spread with respect to the driver current profile and
the witness delay: the host side of the adjoint run.

The reference has no gradients. The parameterisation follows the adjoint workload of the benchmark:

- The driver current profile is a piecewise-linear function of xi on `nbins` nodes, spread evenly
  over the sampled driver's extent (xi0 +- cut sigma_xi). It starts as the Gaussian exp(-(xi - xi0)^2 /
  (2 sigma_xi^2)) at the nodes. A profile f gives each sampled driver particle the weight
  w_i = w_i^s f(xi_i) / f0(xi_i): the sample's own weight times the profile's ratio to its initial
  piecewise-linear interpolant. So at f = f0 the weights are exactly the sampled ones.
- The witness delay d shifts the witness in xi: internal xi_i = xi_i^s + (d - d0), because the witness
  sits at user xi0 = driver xi0 - d and the library's internal xi is minus the user's.
- The objectives come from the witness's moment sums at the last step (Beam::sums,
  src/Beam.cpp:1133-1155; from_sums, :1157-1192): the mean energy gain <gamma>_T - <gamma>_0, and the
  rms energy spread sqrt(<G^2> - <G>^2) at the last step.

The adjoint run returns dJ/d(initial particle) for a seed dJ/d(last moment sums). This module turns
the seeds and the particle adjoints into the parameter gradients.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import numpy as np

# moment-sum indices (Beam::sums order): 0 sum w, 1 sum w G, 2 sum w G^2 (G = gamma - gref)
_SW, _SG, _SG2 = 0, 1, 2


@dataclass
class DriverProfile:
    """Piecewise-linear current profile on nodes xi_nodes (internal xi, increasing)."""
    xi_nodes: np.ndarray
    f0: np.ndarray

    @classmethod
    def gaussian(cls, xi0_internal: float, sigma_xi: float, cut: float = 3.0, nbins: int = 64) -> "DriverProfile":
        nodes = np.linspace(xi0_internal - cut * sigma_xi, xi0_internal + cut * sigma_xi, nbins)
        return cls(nodes, np.exp(-0.5 * ((nodes - xi0_internal) / sigma_xi) ** 2))

    def hat(self, xi: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """(left node index, weight of the right node) of each xi, clamped to the node span."""
        x = np.clip(np.asarray(xi, dtype=np.float64), self.xi_nodes[0], self.xi_nodes[-1])
        h = self.xi_nodes[1] - self.xi_nodes[0]
        i = np.minimum(((x - self.xi_nodes[0]) / h).astype(np.int64), len(self.xi_nodes) - 2)
        t = (x - self.xi_nodes[i]) / h
        return i, t

    def interp(self, f: np.ndarray, xi: np.ndarray) -> np.ndarray:
        i, t = self.hat(xi)
        return (1.0 - t) * f[i] + t * f[i + 1]


def driver_rows(sample: np.ndarray, prof: DriverProfile, f: np.ndarray) -> np.ndarray:
    """The driver's particle rows (n, 7: x y px py pz xi w) with the weights of profile f."""
    out = np.array(sample, dtype=np.float64, copy=True)
    out[:, 6] = sample[:, 6] * prof.interp(f, sample[:, 5]) / prof.interp(prof.f0, sample[:, 5])
    return out


def witness_rows(sample: np.ndarray, shift: float) -> np.ndarray:
    """The witness rows shifted by `shift` in internal xi (= the change of the delay)."""
    out = np.array(sample, dtype=np.float64, copy=True)
    out[:, 5] += shift
    return out


def _moments(S: np.ndarray) -> Tuple[float, float, float]:
    sw = S[_SW]
    return sw, S[_SG] / sw, S[_SG2] / sw


def gain(S_last: np.ndarray, S_first: np.ndarray, gref: float) -> float:
    return (gref + S_last[_SG] / S_last[_SW]) - (gref + S_first[_SG] / S_first[_SW])


def spread(S_last: np.ndarray) -> float:
    _, m0, m1 = _moments(S_last)
    return float(np.sqrt(max(0.0, m1 - m0 * m0)))


def gain_seed(S_last: np.ndarray) -> np.ndarray:
    """dJ/dS (17) of the gain at the last step (the first step's sums do not depend on the driver
    profile or the witness delay)."""
    d = np.zeros(17)
    d[_SG] = 1.0 / S_last[_SW]
    d[_SW] = -S_last[_SG] / S_last[_SW] ** 2
    return d


def spread_seed(S_last: np.ndarray) -> np.ndarray:
    sw = S_last[_SW]
    J = spread(S_last)
    d = np.zeros(17)
    if J <= 0.0:
        return d
    d[_SG2] = 1.0 / sw
    d[_SG] = -2.0 * S_last[_SG] / sw ** 2
    d[_SW] = -S_last[_SG2] / sw ** 2 + 2.0 * S_last[_SG] ** 2 / sw ** 3
    return d / (2.0 * J)


def profile_gradient(lam_driver: np.ndarray, sample: np.ndarray, prof: DriverProfile) -> np.ndarray:
    """dJ/df (nbins) from the driver particles' adjoint (n, 7): w_i = w_i^s f(xi_i) / f0(xi_i)."""
    i, t = prof.hat(sample[:, 5])
    c = lam_driver[:, 6] * sample[:, 6] / prof.interp(prof.f0, sample[:, 5])
    g = np.zeros(len(prof.xi_nodes))
    np.add.at(g, i, c * (1.0 - t))
    np.add.at(g, i + 1, c * t)
    return g


def delay_gradient(lam_witness: np.ndarray) -> float:
    """dJ/d(delay) from the witness particles' adjoint (n, 7): internal xi moves by +1 per unit."""
    return float(np.sum(lam_witness[:, 5]))


# ---------------------------------------------------------------------------- torch interface
def _objective_and_gradient(spec, samples, prof: DriverProfile, f: np.ndarray, shift: float, which: str,
                            stream=None):
    """One forward run with the driver profile f and the witness shifted by `shift`, then the adjoint
    (qz_sim_adjoint): (J, dJ/df (nbins), dJ/d(delay)). samples: [(rows, gref, xiref)] of driver and witness
    as sampled (the profile and shift are applied here)."""
    from .api import Simulation

    (ds, dg, dx), (ws, wg, wx) = samples[0], samples[1]
    beams = [(driver_rows(ds, prof, f), dg, dx), (witness_rows(ws, shift), wg, wx)] + list(samples[2:])
    if which not in ("gain", "spread"):
        raise ValueError("which must be 'gain' or 'spread'")
    sim = Simulation(spec, beams=beams)
    out = {}

    def seed_fn(mom):                     # the linearisation at this run's last moment sums
        S_last, S_first = mom[-1, 1], mom[0, 1]
        out["J"] = gain(S_last, S_first, wg) if which == "gain" else spread(S_last)
        seeds = np.zeros((len(beams), 17))
        seeds[1] = gain_seed(S_last) if which == "gain" else spread_seed(S_last)
        return seeds

    lam, _, _ = sim.adjoint_fn(spec.steps, spec.dt, seed_fn, stream=stream)
    J = out["J"]
    # lam is dJ/d(rows as run); w_i = w_i^s f(xi_i) / f0(xi_i) is linear in f with the sampled xi
    return J, profile_gradient(lam[0], ds, prof), delay_gradient(lam[1])


class WitnessObjective:
    """Witness energy gain or energy spread of a run as a differentiable function of the driver profile
    (torch tensor of nbins nodal values) and the witness delay change (0-d tensor), for torch.autograd.

        obj = WitnessObjective(spec, samples, prof, "gain")
        J = obj(f, d)          # f: (64,) float64, d: () float64, both may require grad
        J.backward()           # f.grad, d.grad from one adjoint run

    The forward computes J and its gradient together (one adjoint run: its forward gives J and the
    seed), and the backward scales the stored gradient by the incoming one."""

    def __init__(self, spec, samples, prof: DriverProfile, which: str = "gain"):
        self.spec, self.samples, self.prof, self.which = spec, samples, prof, which

    def __call__(self, f, delay):
        import torch

        obj = self

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, f_t, d_t):
                J, gf, gd = _objective_and_gradient(obj.spec, obj.samples, obj.prof,
                                                    f_t.detach().cpu().numpy().astype(np.float64),
                                                    float(d_t.detach().cpu()), obj.which)
                ctx.save_for_backward(torch.as_tensor(gf, dtype=torch.float64, device=f_t.device),
                                      torch.as_tensor(gd, dtype=torch.float64, device=d_t.device))
                return torch.as_tensor(J, dtype=torch.float64, device=f_t.device)

            @staticmethod
            def backward(ctx, g):
                gf, gd = ctx.saved_tensors
                return g * gf, g * gd

        return _Fn.apply(f, delay)
