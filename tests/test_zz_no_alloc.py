"""qz_beam_sums_noalloc (the moment sums with their scratch in static device memory) against
qz_beam_sums on the same particles, two calls in a row each, through the C ABI.

Both entry points run the same two reduction kernels in the same order, so the sums agree to
rounding; the test allows 1e-13 relative per sum. An empty beam (n = 0) must give 17 zeros. A fresh
process that calls only the allocation-free entry point must see the device's free memory and
torch's allocator counters unchanged across its calls. This file is collected last so that it also
runs after every other GPU test has used the device."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import quarz_b200 as Q
from quarz_b200._lib import BeamView, check, lib

pytestmark = pytest.mark.gpu

TOL = 1e-13
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _beam(torch, n, seed):
    rng = np.random.default_rng(seed)
    cols = np.stack([
        rng.normal(0, 0.3, n), rng.normal(0, 0.3, n),            # x y
        rng.normal(0, 0.5, n), rng.normal(0, 0.5, n),            # px py
        rng.normal(1000, 1.0, n), rng.normal(3, 1, n),           # pz xi
        np.where(rng.random(n) < 0.05, 0.0, rng.uniform(0.5, 1.5, n)),   # w, some removed particles
    ])
    return torch.from_numpy(np.ascontiguousarray(cols)).cuda().contiguous()


@pytest.mark.parametrize("n", [0, 1000, 200_000])
def test_noalloc_sums_equal_allocating_sums(n):
    import torch

    assert torch.cuda.is_available(), "CUDA device required"
    cols = _beam(torch, n, 11 + n)
    gref, xiref = 1000.0, 3.0
    got = []
    for _ in range(2):
        ref = torch.full((17,), np.nan, dtype=torch.float64, device="cuda")
        out = torch.full((17,), np.nan, dtype=torch.float64, device="cuda")
        Q.BeamOps.sums(cols, gref, xiref, ref)
        Q.BeamOps.sums_noalloc(cols, gref, xiref, out)
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.all(np.abs(o - r) <= TOL * np.maximum(np.abs(r), 1e-300)), (o, r)
        got.append(o)
    assert np.array_equal(got[0], got[1])
    assert got[0][16] == np.count_nonzero(cols[6].cpu().numpy())
    if n == 0:
        assert np.array_equal(got[0], np.zeros(17))


_PROBE = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import quarz_b200 as Q
torch.cuda.set_device(0)
rng = np.random.default_rng(5)
n = 300000
cols = torch.from_numpy(np.ascontiguousarray(np.stack([rng.normal(0, 0.3, n), rng.normal(0, 0.3, n),
    rng.normal(0, 0.5, n), rng.normal(0, 0.5, n), rng.normal(1000, 1, n), rng.normal(3, 1, n),
    rng.uniform(0.5, 1.5, n)]))).cuda().contiguous()
outs = [torch.zeros(17, dtype=torch.float64, device="cuda") for _ in range(20)]
Q.BeamOps.sums_noalloc(cols, 1000.0, 3.0, outs[0])       # the first call loads the module and does the set-up
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
st0 = torch.cuda.memory_stats()
for o in outs[1:]:
    Q.BeamOps.sums_noalloc(cols, 1000.0, 3.0, o)
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
st1 = torch.cuda.memory_stats()
same = all(torch.equal(outs[0], o) for o in outs[1:])
print(json.dumps({"free0": free0, "free1": free1, "same": same,
                  "torch_allocs": [st0.get("allocation.all.allocated", 0), st1.get("allocation.all.allocated", 0)],
                  "torch_reserved": [st0.get("reserved_bytes.all.current", 0), st1.get("reserved_bytes.all.current", 0)]}))
"""


def test_noalloc_sums_allocate_nothing_in_a_fresh_process():
    out = subprocess.run([sys.executable, "-c", _PROBE, ROOT], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["same"]
    assert r["free0"] == r["free1"], r
    assert r["torch_allocs"][0] == r["torch_allocs"][1], r
    assert r["torch_reserved"][0] == r["torch_reserved"][1], r


def test_noalloc_sums_argument_errors():
    with pytest.raises(Q.QZError):
        check(lib().qz_beam_sums_noalloc(None, 0.0, 0.0, None, None))
    v = BeamView()
    v.n = -1
    out = C.c_void_p(1)
    with pytest.raises(Q.QZError) as e:
        check(lib().qz_beam_sums_noalloc(C.byref(v), 0.0, 0.0, out, None))
    assert "negative" in str(e.value)
