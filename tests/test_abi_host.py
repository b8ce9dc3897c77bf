"""Host-side checks without a GPU: the C ABI library loads and exports every declared entry point,
the beam generator of the library (std::mt19937_64 + std::normal_distribution) equals the oracle's
restatement bit for bit, and the deck / grid set-up follows the reference."""
import os
import re

import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import ROOT_DIR, spec_from_text
from quarz_b200 import deck, workloads


def _declared():
    text = open(os.path.join(ROOT_DIR, "include", "qz_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:qz_status|const char\*)\s+(qz_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) >= 20
    L = Q.lib()
    for n in names:
        assert hasattr(L, n), n
    # and the Python binding declares each of them
    from quarz_b200._lib import SIGNATURES
    assert sorted(SIGNATURES) == names


def test_error_reporting_without_device():
    # invalid arguments are rejected on the host, with a message, before any device work
    with pytest.raises(Q.QZError) as e:
        Q.RadialGrid([0.0, 1.0])
    assert "at least 2 cells" in str(e.value)
    with pytest.raises(Q.QZError) as e:
        Q.RadialGrid([0.0, 2.0, 1.0])
    assert "increasing" in str(e.value)


@pytest.mark.parametrize("wl", ["plain_blowout", "pinched_witness"])
def test_library_sampler_equals_oracle(wl):
    spec = workloads.plain_blowout() if wl == "plain_blowout" else workloads.pinched_witness(
        driver_np=20000, witness_np=20000)
    for b in spec.beams:
        a = deck.sampler_args(b)
        po, go, xo = O.sample_gaussian(**a)
        pq, gq, xq = Q.sample_beam(b)
        assert np.array_equal(po, pq) and go == gq and xo == xq


def test_sampler_offsets_and_symmetry_copies():
    b = deck.BeamSpec(name="d", n0=2, sigma_r=0.3, sigma_xi=0.5, xi0_user=-2, gamma=500, espread=0.01, emit_n=0.1,
                      nparticles=4000, seed=7, x0=0.1, x_slope=1e-3, nsym=4, mirror_y=True)
    po, go, xo = O.sample_gaussian(**deck.sampler_args(b))
    pq, gq, xq = Q.sample_beam(b)
    assert np.array_equal(po, pq) and go == gq and xo == xq


def test_grid_generators_match_oracle():
    for R, regs, mr in ((8.0, [(0.5, 0.0025), (2.5, 0.01), (8.0, 0.05)], 1.05), (4.0, [(0.3, 0.002), (4, 0.02)], 1.05),
                        (3.0, [(0.2, 0.002), (3.0, 0.05)], 1.08)):
        assert np.array_equal(deck.make_regions(R, regs, mr), O.make_regions(R, regs, mr))
    assert np.array_equal(deck.make_uniform(6.0, 6 / 256), O.make_uniform(6.0, 6 / 256))


def test_deck_rejects_unknown_keys_and_unsupported_paths():
    base = workloads.PLAIN_BLOWOUT
    with pytest.raises(ValueError):
        deck.run_spec(deck.parse_deck(base, ["laser.a0=1"]))
    with pytest.raises(ValueError):
        deck.run_spec(deck.parse_deck(base, ["pusher.beam=imp_rr"]))    # radiation reaction is not on this path
    assert deck.run_spec(deck.parse_deck(base, ["pusher.beam=boris"])).beams[0].pusher == 1
    assert deck.run_spec(deck.parse_deck(base, ["pusher.beam=boris", "driver.pusher=hc"])).beams[0].pusher == 2
    with pytest.raises(ValueError):
        deck.run_spec(deck.parse_deck(base, ["driver.x0=0.1"]))   # offsets need modes = 1


def test_workload_sizes():
    s0 = workloads.plain_blowout()
    assert (s0.M, s0.K, s0.species[0].ppc) == (257, 1200, 1)
    s1 = workloads.pinched_witness(driver_np=10, witness_np=10)
    h = np.diff(s1.nodes)
    assert (s1.M, s1.K) == (512, 2400)
    assert abs(h[0] - 5e-4) < 1e-12 and abs(h.max() - 0.05) < 1e-12 and (h[1:] / h[:-1]).max() <= 1.02
    assert s1.nodes[-1] == 6.0
