"""The field file of one sweep (qz_write_fields: Simulation::write_fields, src/Simulation.cpp:878-993, the
fields_NNNNNN.bin version 3 that the reference's tools/quarz_read.py reads), written from the oracle's
host arrays and read back with a reader of the documented layout: header, radial nodes, the user xi axis
(increasing, the head of the box last), the component names in the reference's order, and every value
bit for bit, for modes 0 and 1. Host arrays only: no GPU."""
import numpy as np
import pytest

import oracle as O
import quarz_b200 as Q
from helpers import CONFIG0, spec_from_text
from quarz_b200 import workloads


def read_fields(path):
    """the version-3 layout: int32 {3, M, K, mode1}, float64 t, r[M], xi[K], int32 ncomp, ncomp x {name[16], data[K][M]}"""
    with open(path, "rb") as f:
        ver, M, K, m1 = np.fromfile(f, dtype=np.int32, count=4)
        t = np.fromfile(f, dtype=np.float64, count=1)[0]
        r = np.fromfile(f, dtype=np.float64, count=M)
        xi = np.fromfile(f, dtype=np.float64, count=K)
        nc = np.fromfile(f, dtype=np.int32, count=1)[0]
        out = {"version": int(ver), "t": t, "r": r, "xi": xi, "mode1": bool(m1), "names": []}
        for _ in range(nc):
            name = f.read(16).split(b"\0")[0].decode()
            out["names"].append(name)
            out[name] = np.fromfile(f, dtype=np.float64, count=M * K).reshape(K, M)
        assert f.read(1) == b""
    return out


M0 = ["psi", "ez", "er", "eth", "br", "bth", "bz", "ne", "ni", "rhob"]
M1 = [n + s for n in ("psi", "ez", "bz", "ne", "ni", "rhob") for s in ("_c", "_s")] + \
     ["er_c", "er_s", "eth_c", "eth_s", "br_c", "br_s", "bth_c", "bth_s"]


@pytest.mark.parametrize("modes", [0, 1])
def test_field_file_layout_and_values(tmp_path, modes):
    if modes == 0:
        spec = spec_from_text(CONFIG0, ["xi.min=-4", "driver.nparticles=2000"])
    else:
        spec = workloads.spec_from_text(workloads.hosing_deck(xi_min=-2.0, driver_np=2000, witness_np=2000, steps=1),
                                        ["xi.step=0.02"])
    sim = O.OracleSim(spec)
    sim.step_fields(0.0)
    F, D, B = sim.fld(), sim.diag(), sim.bsrc()
    path = tmp_path / "fields_000000.bin"
    Q.write_fields(path, spec, F, D, B, t=12.5)
    got = read_fields(path)
    K, M = spec.K, spec.M
    assert (got["version"], got["mode1"], got["t"]) == (3, modes == 1, 12.5)
    np.testing.assert_array_equal(got["r"], spec.nodes)
    np.testing.assert_array_equal(got["xi"], [0.0 - (spec.xi_min + (K - 1 - k) * spec.dxi) for k in range(K)])
    assert np.all(np.diff(got["xi"]) > 0)
    assert got["names"] == M0 + (M1 if modes else [])
    rows = slice(None, None, -1)                      # file row K-1-k holds slice k
    want = {"psi": D[..., 0], "ez": F[..., 4], "er": F[..., 0], "eth": F[..., 1], "br": F[..., 2], "bth": F[..., 3],
            "bz": F[..., 5], "ne": D[..., 1], "ni": D[..., 2], "rhob": B[..., 4]}
    if modes:
        want.update({"psi_c": 2 * D[..., 3], "psi_s": -2 * D[..., 4], "ez_c": 2 * F[..., 14], "ez_s": -2 * F[..., 15],
                     "bz_c": 2 * F[..., 16], "bz_s": -2 * F[..., 17], "ne_c": 2 * D[..., 5], "ne_s": -2 * D[..., 6],
                     "ni_c": 2 * D[..., 7], "ni_s": -2 * D[..., 8], "rhob_c": 2 * B[..., 13], "rhob_s": -2 * B[..., 14],
                     "er_c": F[..., 6] + F[..., 8], "er_s": F[..., 7] - F[..., 9], "eth_c": F[..., 7] + F[..., 9],
                     "eth_s": F[..., 8] - F[..., 6], "br_c": F[..., 10] + F[..., 12], "br_s": F[..., 11] - F[..., 13],
                     "bth_c": F[..., 11] + F[..., 13], "bth_s": F[..., 12] - F[..., 10]})
    for n, w in want.items():
        np.testing.assert_array_equal(got[n], w[rows], err_msg=n)
    assert np.any(got["rhob"] != 0) and np.any(got["psi"] != 0)
