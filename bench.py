#!/usr/bin/env python
"""Benchmark of the QUARZ hot path on B200: one time step of the pinched-witness workload.

Workload (quarz_b200.workloads.pinched_witness): m = 0, 512 stretched radial nodes (5e-4 -> 0.05),
2400 xi slices (dxi 0.005), ppc 1 cold plasma (511 rings per slice), driver 1e6 + witness 1e6 beam
particles, dt 5. One step = one quasi-static sweep (2400 slice solves) + the Vay push of both beams
with the next step's beam deposit fused in.

Metric: slice-solves/s = K * steps / time (whole job: summed over GPUs; each GPU runs an independent
replica of the workload -- the sweep is sequential in xi, so there is no data-path collective).
Also reported: beam pushes/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "slice-solves/s"
UNIT = "slice-solves/s"
WORKLOAD = "pinched_witness"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            P = json.load(f)
        return float(P["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _config(spec, nb_total, extra=None):
    c = {"workload": WORKLOAD, "modes": spec.modes, "radial_nodes": spec.M, "xi_slices": spec.K,
         "dxi": spec.dxi, "plasma_ppc": spec.species[0].ppc, "plasma_particles_per_slice": spec.M - 1,
         "beam_particles": nb_total, "ab_order": spec.ab_order, "dt": spec.dt,
         "l2": "inputs larger than L2: beam 112 MB + field store 59 MB + beam sources 49 MB per step",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """NVML samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        names = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4,
                 "hw_power_brake_slowdown": 0x80}
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            self._stop.wait(0.01)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv:
            self.t.join()

    def result(self):
        import statistics

        med = statistics.median(self.samples) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def run_b200(args, rank, world, local_rank):
    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200 import workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec = workloads.pinched_witness()
    beams = [Q.sample_beam(b) for b in spec.beams]
    K, M = spec.K, spec.M
    grid = Q.RadialGrid(spec.nodes)
    sweep = Q.Sweep(grid, Q.sweep_params(spec))
    f64 = dict(dtype=torch.float64, device=dev)
    fld = torch.zeros(K * M * 6, **f64)
    diag = torch.zeros(K * M * 3, **f64)
    bsrc = [torch.zeros(K * M * 5, **f64), torch.zeros(K * M * 5, **f64)]
    cols = [torch.from_numpy(np.ascontiguousarray(p.T)).to(dev).contiguous() for p, _, _ in beams]
    nb_total = sum(len(p) for p, _, _ in beams)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    stream = torch.cuda.Stream(device=dev)
    started = [0] * len(beams)
    state = {"cur": 0}
    dt = spec.dt

    def step(ev=None):
        cur, nxt = state["cur"], 1 - state["cur"]
        if ev is not None:
            ev[0].record(stream)
        sweep.run_async(bsrc[cur], fld, diag, stream=stream)
        if ev is not None:
            ev[1].record(stream)
        bsrc[nxt].zero_()
        if ev is not None:
            ev[2].record(stream)
        for i, b in enumerate(spec.beams):
            started[i] = Q.BeamOps.push_deposit(grid, cols[i], b.q, b.m, box, fld, dt, dt, started[i], bsrc[nxt],
                                                stream=stream)
        if ev is not None:
            ev[3].record(stream)
        state["cur"] = nxt

    with torch.cuda.stream(stream):
        for i, b in enumerate(spec.beams):
            Q.BeamOps.deposit(grid, cols[i], b.q, b.m, box, bsrc[0], stream=stream)
        for _ in range(args.warmup):
            step()
    # the first push includes the leapfrog start-up kick; all timed steps are regular ones
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize(dev)
        with torch.cuda.stream(stream):
            t0.record(stream)
            for s in range(args.steps):
                step(evs[s])
            t1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1)
    sweep_ms = [e[0].elapsed_time(e[1]) for e in evs]
    push_ms = [e[2].elapsed_time(e[3]) for e in evs]
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    launches_per_step = 1 + len(spec.beams)   # sweep kernel + fused push/deposit per beam
    # end-to-end through the host-buffer call of the C ABI (qz_sim_step_host)
    e2e = run_e2e(args, spec, beams, dev) if args.e2e_steps > 0 else None
    out = {
        "ms": ms, "sweep_ms": sweep_ms, "push_ms": push_ms, "clocks": clk.result(), "spec": spec,
        "nb_total": nb_total, "launches": launches_per_step * args.steps, "e2e": e2e,
    }
    return out


def run_e2e(args, spec, beams, dev):
    import ctypes as C

    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200._lib import check, lib

    sim = Q.Simulation(spec, beams=beams)
    host = [torch.from_numpy(np.ascontiguousarray(p.T)).contiguous().pin_memory() for p, _, _ in beams]
    ptrs = (C.c_void_p * len(host))(*[h.data_ptr() for h in host])
    mom = np.zeros((len(beams), 17))
    stream = torch.cuda.Stream(device=dev)
    sp = C.c_void_p(stream.cuda_stream)
    dt = spec.dt

    def one():
        check(lib().qz_sim_step_host(sim.h, ptrs, dt, dt, 1, mom.ctypes.data_as(C.POINTER(C.c_double)), sp))

    for _ in range(2):
        one()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        one()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.e2e_steps
    nbytes = sum(7 * 8 * len(p) for p, _, _ in beams)
    return {"ms_per_step": ms, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 17 * 8 * len(beams)}


def oracle_step_rate(steps, warmup, spec=None):
    """The CPU oracle (serial restatement of the reference path) on the same workload: slice-solves/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from quarz_b200 import workloads

    O.build()
    spec = spec or workloads.pinched_witness()
    sim = O.OracleSim(spec)
    dt = spec.dt
    sim.step_fields(0.0)
    sim.push_beams(dt, dt)     # start-up + first push outside the timing
    for _ in range(max(0, warmup - 1)):
        sim.step_fields(0.0)
        sim.push_beams(dt, dt)
    t = time.perf_counter()
    for _ in range(steps):
        sim.step_fields(0.0)
        sim.push_beams(dt, dt)
    el = time.perf_counter() - t
    return spec.K * steps / el, el, spec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-steps", type=int, default=10, help="oracle steps of the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        rate, el, spec = oracle_step_rate(args.steps, args.warmup)
        nb = sum(b.nparticles for b in spec.beams)
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": _config(spec, nb),
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                                 "sample": f"{args.steps} full time steps of the workload (sweep + beam push) "
                                           f"after {args.warmup} warm-up steps, serial oracle"},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch

        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    r = run_b200(args, rank, world, local_rank)
    spec = r["spec"]
    K = spec.K
    ms_step = r["ms"] / args.steps
    value = world * K * args.steps / (r["ms"] * 1e-3)
    # roofline of the dominant kernel (the sweep): algorithmic HBM bytes per slice =
    # beam-source row read (5 M doubles) + field row and diagnostics written ((6 + 3) M doubles)
    sweep_ms = sorted(r["sweep_ms"])[len(r["sweep_ms"]) // 2]
    bytes_sweep = K * spec.M * (5 + 6 + 3) * 8
    hbm, peak_kind = _peaks()
    achieved = bytes_sweep / (sweep_ms * 1e-3) / 1e9
    push_ms = sorted(r["push_ms"])[len(r["push_ms"]) // 2]
    nbt = r["nb_total"]
    bytes_push = nbt * (7 * 8 + 7 * 8) + K * spec.M * (6 + 5) * 8   # particles read+written, fld read, bsrc write
    push_gbs = bytes_push / (push_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": _config(spec, nbt),
        "beam_pushes_per_s": world * nbt / (push_ms * 1e-3),
        "sweep_ms": sweep_ms, "per_slice_us": 1e3 * sweep_ms / K, "push_deposit_ms": push_ms,
        "roofline": {"bound": "hbm", "kernel": "sweep_m0_kernel", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": None,
                     "note": "one CTA on one SM, latency-bound chain of 5 barrier phases per slice; "
                             "algorithmic bytes = K*M*(5+6+3)*8 per sweep"},
        "roofline_beam": {"bound": "hbm", "kernel": "beam_push_kernel<deposit>", "achieved": push_gbs, "peak": hbm,
                          "unit": "GB/s", "frac": push_gbs / hbm, "peak_kind": peak_kind},
        "clocks": r["clocks"], "gpu_launches": r["launches"],
    }
    if r["e2e"]:
        e = r["e2e"]
        line["e2e"] = {"value": world * K / (e["ms_per_step"] * 1e-3), "unit": UNIT,
                       "h2d_bytes_per_step": e["h2d_bytes_per_step"], "d2h_bytes_per_step": e["d2h_bytes_per_step"],
                       "ms_per_step": e["ms_per_step"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, el, _ = oracle_step_rate(args.cpu_steps, 1, spec)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{args.cpu_steps} full time steps of the same workload (sweep + beam push), "
                                          f"serial oracle, {el:.1f} s"}
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
