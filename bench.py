#!/usr/bin/env python
"""Benchmark of the QUARZ hot path on B200: the pinched-witness run.

Workload (quarz_b200.workloads.pinched_witness): m = 0, 512 stretched radial nodes (5e-4 -> 0.05),
2400 xi slices (dxi 0.005), ppc 1 cold plasma (511 rings per slice), driver 1e6 + witness 1e6 beam
particles, dt 5, 100 time steps. One bench step = the whole run as Simulation::run does it: 101
quasi-static sweeps (2400 slice solves each), the moment sums of every step, and 100 Vay pushes of
both beams with the next step's deposit, through the library's public call (qz_sim_run), starting
every time from the same initial beams (resident in HBM).

Metric: slice-solves/s = K * (time steps + 1) / time (whole job: summed over GPUs; each GPU runs an
independent replica -- the sweep is sequential in xi, so there is no data-path collective). Also
reported: beam pushes/s.

Other workloads (not the headline; their lines are recorded beside it):
  --workload hosing   the same run with azimuthal modes 0 and 1 (8 azimuths per ring, Picard 3),
                      offset / tilted driver, 2e6 + 2e6 particles, 200 steps
  --workload scan     512 independent runs of 20 steps (a parameter scan) in one launch: runs/s, with
                      the plain loop over single runs (step by step, and pipelined) timed on a sample
  --workload scan_m1  the same scan with azimuthal modes 0 and 1 (128..1023 cells; above 512 nodes the
                      m = 1 instances run in a second launch of 1024-thread CTAs)
  --workload adjoint  the gradient of witness energy gain and spread with respect to a 64-bin driver
                      profile and the witness delay, pinched witness over 50 steps: adjoint / forward time
  --workload stages   the xi-pipelined run over the ranks (one slab of the box per GPU, the reference's
                      multi-rank mode), pinched witness with the ngp xi shape, 20 steps
  --smooth A          the pinched-witness or hosing run with plasma.smooth_length = A (the radial
                      smoothing of the plasma sources; 0.005 in the reference's validation section 14)

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload ...] [--smooth A]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "slice-solves/s"
UNIT = "slice-solves/s"
WORKLOAD = "pinched_witness"
# our kernels per run, per beam: iota + cell keys + reorder + group starts + step-0 deposit; per run:
# the pipelined kernel + the moment reduction (the radix sort's own kernels are library code)
OWN_LAUNCHES_PER_BEAM = 5
OWN_LAUNCHES_PER_RUN = 2


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            P = json.load(f)
        return float(P["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _library_source():
    """The source hash the loaded library was built from (qz_version: '... src <hash>')."""
    import quarz_b200 as Q

    v = Q.lib().qz_version()
    v = v.decode() if isinstance(v, bytes) else str(v)
    m = re.search(r"src ([0-9a-f]+|unknown)", v)
    return m.group(1) if m else "unknown"


def _traffic_ratio():
    """DRAM bytes per algorithmic byte of the pipelined kernel, from the ncu capture of a shorter run of
    the same workload summarised in profiles/ (traffic grows with the steps like the algorithmic bytes),
    and the library source hash that capture measured. Returns (ratio or None, measured hash or None)."""
    path = os.path.join(ROOT, "profiles", "pipeline_kernel_pinched_witness.md")
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        return None, None
    m = re.search(r"dram_bytes_per_algorithmic_byte:\s*([0-9.eE+]+)", text)
    h = re.search(r"library source:\s*([0-9a-f]+)", text)
    return (float(m.group(1)) if m else None), (h.group(1) if h else None)


def _config(spec, nb_total, steps, extra=None, workload=WORKLOAD):
    c = {"workload": workload, "modes": spec.modes, "radial_nodes": spec.M, "xi_slices": spec.K,
         "dxi": spec.dxi, "plasma_ppc": spec.species[0].ppc, "plasma_particles_per_slice": spec.M - 1,
         "beam_particles": nb_total, "ab_order": spec.ab_order, "dt": spec.dt, "time_steps_per_run": steps,
         "l2": "inputs larger than L2: beams 112 MB + a field store of 59 MB and beam sources of 49 MB per step "
               "in flight (rings of one slot per step)",
         "parallelism": "replicas"}
    if getattr(spec, "smooth_length", 0.0):
        c["smooth_length"] = spec.smooth_length
    if extra:
        c.update(extra)
    return c


def algorithmic_bytes(spec, nb_total, steps):
    """HBM bytes a run must move at least: per sweep the beam sources read (5 doubles per node and
    slice) and the fields + diagnostics written (6 + 3); per push step every particle read and written
    (7 doubles each way), the field store read once (6) and the next beam sources written once (5)."""
    km = spec.K * spec.M
    sweep = km * (5 + 6 + 3) * 8
    push = nb_total * 7 * 8 * 2 + km * (6 + 5) * 8
    return (steps + 1) * sweep + steps * push


# FP64 operations of the reference algorithm, counted from the cited reference lines (per plasma particle
# per slice; per radial node per slice; per beam particle per time step). m = 0:
#   plasma particle: deposit (src/PlasmaSpecies.cpp:409-478) 47 + S deposit with its field gather
#   (:508-559) 102 + AB3 push with its gather (:561-668) 110 + two cell lookups / weights 24 + the 12
#   deposit additions of the warp sums = 295;
#   radial node: 5 Thomas solves x 8 (psi, E_z, B_z, B_r, B_theta; src/Tridiag.cpp:111-125) + source
#   combination, stencils, W+, the B+ right-hand sides and the slice store (src/Simulation.cpp:408-633)
#   60 = 100;
#   beam particle: bilinear gather of 6 components 36 + Vay (src/Pushers.hpp:36-68) 60 + drift and
#   weights 24 + the linear deposit of 5 components on 4 points (src/Beam.cpp:725-785) 60 = 180.
# m = 1 (8 azimuths, 27 solves, Picard 3; gathers of 18 components, deposits of 15):
#   plasma particle 470, radial node 400, beam particle 330.
FLOPS = {0: (295, 100, 180), 1: (470, 400, 330)}


def run_flops(spec, nb_total, steps):
    """FP64 operations of a run: (steps + 1) sweeps of K slices and `steps` pushes of every beam particle."""
    fp, fm, fb = FLOPS[spec.modes]
    npl = (spec.M - 1) * (spec.species[0].ntheta if spec.modes == 1 else 1) * spec.species[0].ppc
    return (steps + 1) * spec.K * (npl * fp + spec.M * fm) + steps * nb_total * fb


# Latency floor of one m = 0 slice on one SM (cycles): its dependent chain. Per slice the sweep runs 5
# block scans (psi / E_z / B_z forward and backward, the B+ pivot scan and its two substitutions share
# one pass each way) and 4 further barriers. A block scan is a 5-level warp-shuffle scan (shuffle ~24 +
# FP64 FMA ~8 cycles per level), two shared-memory round trips (~60), the scan of the 16 warp carries
# (~130) and its barrier (~45): ~400 cycles. A plasma particle's chain per slice (push, cell lookup by
# a 9-level binary search in shared memory, two divides of ~68 cycles, the S and plasma deposits with
# their warp sums) is ~2,000 cycles. Barrier and divide costs are the ones measured on this part with
# clock64 counters; the shuffle and FMA latencies are those of the CUDA documentation's latency tables.
SLICE_FLOOR_CYCLES = {"block_scans": 5 * 400, "barriers": 4 * 45, "particle_chain": 2000}


def fp64_gemm_tflops(dev, n=8192, reps=3):
    """Measured FP64 peak: cuBLAS DGEMM (torch.matmul, float64, n^3) on this GPU, best of reps."""
    import torch

    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def sweep_latency(spec, beams, dev, sim, steps_traced):
    """Per-slice latency of the sweep: stand-alone (one qz_sweep_run of the initial beams' sources, on one
    SM) and inside the pipelined run (from the run trace: the time sweep n takes from its first to its
    last slice, median over the steps), in us; the stand-alone sweep's phase cycles per slice."""
    import numpy as np
    import torch

    import quarz_b200 as Q

    grid = Q.RadialGrid(spec.nodes)
    sw = Q.Sweep(grid, Q.sweep_params(spec))
    K, M = spec.K, spec.M
    f64 = dict(dtype=torch.float64, device=dev)
    m1 = spec.modes == 1                    # (B_NC, F_NC, D_NC) = (15, 18, 9) with mode 1, else (5, 6, 3)
    bsrc = torch.zeros(K * M * (15 if m1 else 5), **f64)
    fld = torch.zeros(K * M * (18 if m1 else 6), **f64)
    diag = torch.zeros(K * M * (9 if m1 else 3), **f64)
    box = Q.BeamOps.box(spec.xi_min, spec.dxi, K, spec.ngp, spec.modes)
    for b, (parts, _, _) in zip(spec.beams, beams):
        cols = torch.from_numpy(np.ascontiguousarray(parts.T)).to(dev).contiguous()
        Q.BeamOps.deposit(grid, cols, b.q, b.m, box, bsrc)
    sw.run(bsrc, fld, diag)
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sw.run_async(bsrc, fld, diag)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    alone = 1e3 * min(ms) / K
    sw.timing(True)
    sw.run(bsrc, fld, diag)
    cyc = sw.timing(False).astype(np.float64) / K
    del sw, bsrc, fld, diag
    sim.trace(True)
    sim.run(steps_traced, spec.dt)
    per, _ = sim.trace(False)
    pace = float(np.median((per[:, 1] - per[:, 0]) / K)) * 1e-3
    return {"sweep_us_per_slice_standalone": alone, "sweep_us_per_slice_in_pipeline": pace,
            "standalone_phase_cycles_per_slice": {"psi_ez_bz": float(cyc[1]), "s_deposit": float(cyc[2]),
                                                  "bplus": float(cyc[3]), "store_push_deposit": float(cyc[4])}}


class ClockSampler:
    """NVML samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.mem_used_max = 0
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
                self.mem_used_max = max(self.mem_used_max, int(nv.nvmlDeviceGetMemoryInfo(self.h).used))
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


def _workload(args):
    from quarz_b200 import workloads

    spec = workloads.hosing() if args.workload == "hosing" else workloads.pinched_witness()
    if args.time_steps:
        spec.steps = args.time_steps
    if args.smooth:
        spec.smooth_length = args.smooth
    return spec


def run_b200(args, rank, world, local_rank):
    import numpy as np
    import torch

    import quarz_b200 as Q

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec = _workload(args)
    T = spec.steps
    beams = [Q.sample_beam(b) for b in spec.beams]
    nb_total = sum(len(p) for p, _, _ in beams)
    sim = Q.Simulation(spec, beams=beams)
    init = [torch.from_numpy(np.ascontiguousarray(p.T)).to(dev).contiguous() for p, _, _ in beams]
    stream = torch.cuda.Stream(device=dev)
    kernel_ms, moments = [], []

    def one():
        for b in range(len(init)):
            sim.set_beam(b, init[b], stream=stream)
        moments.append(sim.run(T, spec.dt, stream=stream))
        kernel_ms.append(sim.times()["kernel_ms"])

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    kernel_ms.clear()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize(dev)
        t0.record(stream)
        for _ in range(args.steps):
            one()
        t1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    sched = sim.schedule()
    e2e = run_e2e(args, spec, beams, sim, dev) if args.e2e_steps > 0 else None
    launches = (OWN_LAUNCHES_PER_BEAM * len(beams) + OWN_LAUNCHES_PER_RUN) * args.steps
    return {"ms": ms, "kernel_ms": kernel_ms, "clocks": clk.result(), "spec": spec, "nb_total": nb_total,
            "launches": launches, "e2e": e2e, "schedule": sched, "beams": beams, "sim": sim, "dev": dev,
            "init": init}


def run_e2e(args, spec, beams, sim, dev):
    """The same run through the host-buffer call (qz_sim_run_host): the beams are copied in from pinned
    host memory and back out every run, inside the timed region."""
    import numpy as np
    import torch

    host = [torch.from_numpy(np.ascontiguousarray(p.T)).contiguous().pin_memory() for p, _, _ in beams]
    init = [h.clone() for h in host]
    stream = torch.cuda.Stream(device=dev)
    ms = []
    for i in range(1 + args.e2e_steps):
        for h, h0 in zip(host, init):
            h.copy_(h0)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.run_host(spec.steps, spec.dt, host, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i > 0:                                   # the first call is a warm-up
            ms.append(e0.elapsed_time(e1))
    nbytes = sum(7 * 8 * len(p) for p, _, _ in beams)
    return {"ms_per_run": sum(ms) / len(ms), "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes + 17 * 8 * len(beams) * (spec.steps + 1)}


def run_hosing_extra(dev, steps=2, warmup=1, cpu_steps=1):
    """The hosing run (modes 0 and 1, 2e6 + 2e6 particles, 200 steps) through qz_sim_run: slice-solves/s
    on the device, and the oracle on the host threads for the same unit."""
    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200 import workloads

    spec = workloads.hosing()
    T = spec.steps
    beams = [Q.sample_beam(b) for b in spec.beams]
    sim = Q.Simulation(spec, beams=beams)
    init = [torch.from_numpy(np.ascontiguousarray(p.T)).to(dev).contiguous() for p, _, _ in beams]
    ms = []
    for it in range(warmup + steps):
        for b in range(len(init)):
            sim.set_beam(b, init[b])
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.run(T, spec.dt)
        e1.record()
        torch.cuda.synchronize(dev)
        if it >= warmup:
            ms.append(e0.elapsed_time(e1))
    del sim, init
    torch.cuda.empty_cache()
    nb = sum(len(p) for p, _, _ in beams)
    per = sum(ms) / len(ms)
    out = {"metric": METRIC, "value": spec.K * (T + 1) / (per * 1e-3), "unit": UNIT, "ms_per_run": per,
           "runs_timed": steps, "config": _config(spec, nb, T, None, "hosing"),
           "beam_pushes_per_s": nb * T / (per * 1e-3)}
    rate, el = oracle_rate(cpu_steps, 0, spec)
    out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": oracle_rate.threads, "kind": "port",
                           "sample": f"{cpu_steps} full time step(s) of the hosing run (sweep + moment sums + push "
                                     f"of 4e6 particles), oracle on {oracle_rate.threads} host threads, {el:.1f} s"}
    return out


def run_stages(args, rank, world, local_rank):
    """The xi-pipelined run (quarz_b200.stages): the pinched-witness deck with the ngp xi shape, the box cut
    into one slab per rank; slice-solves/s of the whole job, timed on the device (max over ranks)."""
    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200 import stages, workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec = workloads.spec_from_text(workloads.pinched_witness_deck(steps=args.time_steps or 20),
                                    ["beams.xi_shape=ngp"])
    T = spec.steps
    beams = [Q.sample_beam(b) for b in spec.beams]
    ms = []
    for it in range(args.warmup + args.steps):
        run = stages.Stages(spec, world, beams, ranks=[rank], device=dev)
        if world > 1:
            st = run.stages[0]
            np_, npad, order = st.sweep.state_shape()
            run.channel = stages.DistChannel(dev, len(beams), (6 + 5 * order, npad), spec.M)
            run.local = False
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run.run(T, spec.dt)
        e1.record()
        torch.cuda.synchronize(dev)
        if it >= args.warmup:
            ms.append(e0.elapsed_time(e1))
        del run
    t = float(np.median(ms))
    if world > 1:
        tt = torch.tensor([t], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    nb = sum(len(p) for p, _, _ in beams)
    return {"metric": METRIC, "value": spec.K * (T + 1) / (t * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(spec, nb, T, {"xi_shape": "ngp", "parallelism": f"xi-pipelined over {world} slab(s)"},
                              "stages"),
            "gpu_launches": None}


def run_scan(args, rank, world, local_rank):
    """The batched scan: 512 runs of 20 steps in one launch (qz_batch), runs/s; beside it the plain loop
    over single runs on 6 sampled instances (step by step and pipelined)."""
    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200 import workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from quarz_b200 import scan

    modes = 1 if args.workload == "scan_m1" else 0
    # 512 instances per GPU, the whole scan split over the ranks by estimated cost
    all_specs = workloads.scan_instances(512 * world, seed=2024, modes=modes)
    all_beams = [[Q.sample_beam(b) for b in s.beams] for s in all_specs]
    costs = [scan.instance_cost(s, sum(len(p) for p, _, _ in bm)) for s, bm in zip(all_specs, all_beams)]
    mine = scan.partition(costs, world)[rank]
    specs, beams = [all_specs[i] for i in mine], [all_beams[i] for i in mine]
    batch = Q.Batch()
    for s_, b_ in zip(specs, beams):
        batch.add(s_, b_)
    T, dt = specs[0].steps, specs[0].dt
    for _ in range(args.warmup):
        batch.run(T, dt)
    # the built-in layouts and queue order, then the autotuner's (its calibration batch is set-up work,
    # outside the timed region, reported beside the line)
    batch.run(T, dt)
    untuned_ms = batch.info()["kernel_ms"]
    from quarz_b200 import tune

    t0 = time.time()
    tuning = tune.calibrate(specs, beams, dt)
    tune.apply(batch, specs, beams, T, tuning)
    calib_s = time.time() - t0
    batch.run(T, dt)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    kms, last = [], None
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            last = batch.run(T, dt)   # (the beams restart from where the previous batch left them)
            kms.append(batch.info()["kernel_ms"])
    ms = sum(kms)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    # the final gather of per-instance results (last-step moment sums), outside the timed region
    gathered = scan.run_sharded(all_specs, all_beams, lambda s, b: last, device=dev)
    done = int(np.count_nonzero(np.abs(gathered).sum(axis=(1, 2))))
    loop = {}
    idx = np.linspace(0, len(specs) - 1, 6).astype(int)
    for name, pipelined in (("step_by_step", False), ("pipelined", True)):
        tt = 0.0
        for i in idx:
            sim = Q.Simulation(specs[i], beams=beams[i])
            sim.set_schedule(pipelined)
            sim.run(T, dt)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            sim2 = Q.Simulation(specs[i], beams=beams[i])
            sim2.set_schedule(pipelined)
            torch.cuda.synchronize(dev)
            e0.record()
            sim2.run(T, dt)
            e1.record()
            torch.cuda.synchronize(dev)
            tt += e0.elapsed_time(e1)
        loop[name] = 1e3 * len(idx) / tt
    value = len(all_specs) * args.steps / (ms * 1e-3)
    return {"metric": "runs/s", "value": value, "unit": "runs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "modes": modes, "instances": len(all_specs),
                       "instances_with_results": done, "time_steps_per_run": T,
                       "beam_particles_per_run": 100000, "radial_nodes": "129..1025" if modes == 0 else "129..1024",
                       "xi_slices": "801..1601",
                       "parallelism": "a CTA per instance, one launch per batch; instances split over GPUs by cost"},
            "loop_runs_per_s": loop, "speedup_vs_step_by_step_loop": value / world / loop["step_by_step"],
            "speedup_vs_pipelined_loop": value / world / loop["pipelined"],
            "autotuner": {"untuned_runs_per_s": len(specs) / (untuned_ms * 1e-3), "calibration_s": calib_s,
                          "layouts": {"/".join(map(str, k)): v for k, v in sorted(tuning.layouts.items())},
                          "classes": "modes/filter/plasma in global memory/M div 128",
                          "layout_bits": "1 double-buffered sources, 2 constants in shared memory, 4 particle copy"},
            "clocks": clk.result(), "gpu_launches": args.steps}


def run_adjoint(args, rank, world, local_rank):
    """One bench step = one gradient (qz_sim_adjoint: forward keeping the beams of every step, then the
    reverse pass) of the witness energy gain with respect to the 64 driver-profile bins and the witness
    delay, on the pinched-witness run over 50 steps; the forward it is compared with is the same run
    through qz_sim_run (pipelined), both timed on the device."""
    import numpy as np
    import torch

    import quarz_b200 as Q
    from quarz_b200 import adjoint as A
    from quarz_b200 import workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec = workloads.pinched_witness(steps=args.time_steps or 50)
    T, dt = spec.steps, spec.dt
    beams = [Q.sample_beam(b) for b in spec.beams]
    drv = spec.beams[0]
    prof = A.DriverProfile.gaussian(-drv.xi0_user, drv.sigma_xi, drv.cut, 64)
    sim = Q.Simulation(spec, beams=beams)
    init = [torch.from_numpy(np.ascontiguousarray(p.T)).to(dev).contiguous() for p, _, _ in beams]
    fwd, mom = [], None
    for it in range(args.warmup + args.steps):
        for b in range(len(init)):
            sim.set_beam(b, init[b])
        mom = sim.run(T, dt)
        if it >= args.warmup:
            fwd.append(sim.times()["kernel_ms"])
    seeds = np.zeros((len(beams), 17))
    seeds[1] = A.gain_seed(mom[-1, 1])
    adj, split, grads = [], [], None
    # one simulation for every gradient, its beams reset before each (as for the forward runs above), so
    # that its rings are allocated once and not inside a timed forward; the first gradient is a warm-up
    s2 = Q.Simulation(spec, beams=beams)
    with ClockSampler(local_rank) as clk:
        for it in range(max(1, args.steps) + 1):
            for b in range(len(init)):
                s2.set_beam(b, init[b])
            s2.restart()
            lam, _, ms = s2.adjoint(T, dt, seeds)
            if it:
                adj.append(ms[0] + ms[1])
                split.append(ms)
    del s2
    grads = (A.profile_gradient(lam[0], beams[0][0], prof), A.delay_gradient(lam[1]))
    f_ms, a_ms = float(np.median(fwd)), float(np.median(adj))
    nbt = sum(len(p) for p, _, _ in beams)
    return {"metric": "adjoint/forward time ratio", "value": a_ms / f_ms, "unit": "x", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": a_ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(spec, nbt, T, {"objective": "witness mean energy gain",
                                             "parameters": "64 driver-profile bins + witness delay",
                                             "adjoint": "pipelined forward recording the beams of every step, "
                                                        "the plasma state at every ceil(sqrt(K))-th slice and the "
                                                        "W+ field of every slice, then the pipelined reverse pass "
                                                        "(reverse sweeps that push each segment again from its "
                                                        "checkpoint, beam adjoint tasks)"},
                              "adjoint"),
            "forward_ms": f_ms, "adjoint_ms": a_ms,
            "adjoint_split_ms": {"forward_keeping_beams": float(np.median([m[0] for m in split])),
                                 "reverse": float(np.median([m[1] for m in split]))},
            "gradient_norm_profile": float(np.linalg.norm(grads[0])), "gradient_delay": grads[1],
            "peak_device_bytes": clk.mem_used_max,
            "peak_device_bytes_note": "NVML memory used on the device during the gradients (the whole process: "
                                      "the forward run's own buffers and torch's cache included)",
            "clocks": clk.result(),
            # per gradient: the forward run's own kernels (per beam: iota, cell keys, reorder, group starts,
            # step-0 deposit; the pipeline, the moment reduction), the reverse pass's (bucket cells, running
            # maximum, per beam the seed and the reorder back; the reverse pipeline)
            "gpu_launches": args.steps * (OWN_LAUNCHES_PER_BEAM * len(beams) + OWN_LAUNCHES_PER_RUN + 3 + 2 * len(beams))}


def _oracle_openmp():
    """The oracle's timing build (per-particle loops on all host threads) and its thread count; the
    serial build and 1 thread when the timing build cannot be made."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    try:
        O.build(omp=True)
        O.use_openmp(True)
        threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or (os.cpu_count() or 1)
    except Exception:
        O.build()
        threads = 1
    return O, threads


def oracle_rate(time_steps, warmup, spec):
    """The CPU oracle (restatement of the reference path) on the same workload, on all host threads:
    slice-solves/s over time_steps full time steps (sweep + moment sums + push), after warm-up steps."""
    O, threads = _oracle_openmp()
    oracle_rate.threads = threads
    sim = O.OracleSim(spec)
    dt = spec.dt
    sim.step_fields(0.0)
    sim.push_beams(dt, dt)     # start-up + first push outside the timing
    for _ in range(max(0, warmup - 1)):
        sim.step_fields(0.0)
        sim.push_beams(dt, dt)
    t = time.perf_counter()
    for _ in range(time_steps):
        sim.step_fields(0.0)
        for b in range(len(spec.beams)):
            sim.beam_sums(b)
        sim.push_beams(dt, dt)
    el = time.perf_counter() - t
    return spec.K * time_steps / el, el


def oracle_scan_rate(time_steps, warmup, modes=0):
    """The CPU oracle on the scan: one full time step (sweep + moment sums + push) of each of
    `time_steps` instances sampled across the 512, after warm-up steps of the first; a run of T steps
    costs T + 1 sweeps, so runs/s = 1 / ((T + 1) x the mean time of a step)."""
    import numpy as np

    from quarz_b200 import workloads

    O, threads = _oracle_openmp()
    oracle_scan_rate.threads = threads
    specs = workloads.scan_instances(512, seed=2024, modes=modes)
    idx = np.linspace(0, len(specs) - 1, max(1, time_steps)).astype(int)
    sim = O.OracleSim(specs[idx[0]])
    for _ in range(warmup):
        sim.step_fields(0.0)
        sim.push_beams(specs[idx[0]].dt, specs[idx[0]].dt)
    el = 0.0
    for i in idx[:time_steps]:
        spec = specs[i]
        sim = O.OracleSim(spec)
        t = time.perf_counter()
        sim.step_fields(0.0)
        for b in range(len(spec.beams)):
            sim.beam_sums(b)
        sim.push_beams(spec.dt, spec.dt)
        el += time.perf_counter() - t
    T = specs[0].steps
    return 1.0 / ((T + 1) * el / max(1, time_steps)), el


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5, help="timed runs (each: the workload's time steps)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--e2e-steps", type=int, default=3, help="timed runs through the host-buffer call")
    ap.add_argument("--cpu-steps", type=int, default=10, help="oracle time steps of the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: no latency roofline, FP64 rate or hosing / scan / adjoint lines")
    ap.add_argument("--time-steps", type=int, default=0, help="time steps per run (default: the workload's)")
    ap.add_argument("--workload", choices=["pinched_witness", "hosing", "scan", "scan_m1", "adjoint", "stages"],
                    default="pinched_witness")
    ap.add_argument("--smooth", type=float, default=0.0,
                    help="plasma.smooth_length of the pinched-witness / hosing run (0: none, the headline)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload in ("scan", "scan_m1"):
            rate, el = oracle_scan_rate(args.steps, args.warmup, 1 if args.workload == "scan_m1" else 0)
            line = {"impl": "reference", "metric": "runs/s", "value": rate, "unit": "runs/s", "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "config": {"workload": args.workload, "instances": 512, "time_steps_per_run": 20,
                                                    "beam_particles_per_run": 100000},
                    "cpu_baseline": {"value": rate, "unit": "runs/s", "cores": oracle_scan_rate.threads, "kind": "port",
                                     "sample": f"one full time step of each of {args.steps} instances sampled "
                                               f"across the scan, oracle on {oracle_scan_rate.threads} host "
                                               f"threads; a run = 21 such steps"},
                    "e2e": {"value": rate, "unit": "runs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line))
            return
        spec = _workload(args)
        # each bench step is one full time step of the oracle (a bounded sample of the run)
        rate, el = oracle_rate(args.steps, args.warmup, spec)
        nb = sum(b.nparticles for b in spec.beams)
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": _config(spec, nb, spec.steps, None, args.workload),
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": oracle_rate.threads, "kind": "port",
                                 "sample": f"{args.steps} full time steps of the workload (sweep + moment sums + "
                                           f"beam push) after {args.warmup} warm-up steps, oracle on "
                                           f"{oracle_rate.threads} host threads"},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import datetime

        import torch

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload == "adjoint":
        line = run_adjoint(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line))
        return
    if args.workload == "stages":
        line = run_stages(args, rank, world, local_rank)
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(line))
        return
    if args.workload in ("scan", "scan_m1"):
        line = run_scan(args, rank, world, local_rank)
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            rate, el = oracle_scan_rate(args.cpu_steps, 1, 1 if args.workload == "scan_m1" else 0)
            line["cpu_baseline"] = {"value": rate, "unit": "runs/s", "cores": oracle_scan_rate.threads,
                                    "kind": "port",
                                    "sample": f"one full time step of each of {args.cpu_steps} instances sampled "
                                              f"across the scan, oracle on {oracle_scan_rate.threads} host threads, "
                                              f"{el:.1f} s; a run = 21 such steps"}
        if rank == 0:
            print(json.dumps(line))
        return
    r = run_b200(args, rank, world, local_rank)
    spec = r["spec"]
    K, T = spec.K, spec.steps
    nbt = r["nb_total"]
    ms_step = r["ms"] / args.steps
    value = world * K * (T + 1) * args.steps / (r["ms"] * 1e-3)
    # roofline of the dominant kernel (the pipelined run: one launch per bench step)
    kms = sorted(r["kernel_ms"])[len(r["kernel_ms"]) // 2]
    alg = algorithmic_bytes(spec, nbt, T)
    hbm, peak_kind = _peaks()
    achieved = alg / (kms * 1e-3) / 1e9
    ratio, measured_src = _traffic_ratio()
    lib_src = _library_source()
    fresh = ratio is not None and measured_src == lib_src
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": _config(spec, nbt, T, {"schedule": r["schedule"]}, args.workload),
        "beam_pushes_per_s": world * nbt * T * args.steps / (r["ms"] * 1e-3),
        "kernel_ms_per_run": kms, "per_sweep_ms": kms / (T + 1),
        "roofline": {"bound": "hbm", "kernel": "pipeline_kernel", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": ratio * alg if fresh else None,
                     "traffic_source": (f"ncu capture of this library build (src {lib_src}), scaled by steps"
                                        if fresh else
                                        f"stale: the ncu capture measured src {measured_src}, this library is "
                                        f"src {lib_src}"),
                     "algorithmic_bytes": alg,
                     "note": "one launch per run; its floor is one sweep's dependent chain (K slices, one SM) "
                             "plus the step-to-step stagger, not HBM: the latency and fp64 entries measure it"},
        "clocks": r["clocks"], "gpu_launches": r["launches"],
    }
    if r["e2e"]:
        e = r["e2e"]
        line["e2e"] = {"value": world * K * (T + 1) / (e["ms_per_run"] * 1e-3), "unit": UNIT,
                       "h2d_bytes_per_step": e["h2d_bytes_per_step"], "d2h_bytes_per_step": e["d2h_bytes_per_step"],
                       "ms_per_step": e["ms_per_run"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, el = oracle_rate(args.cpu_steps, 1, spec)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": oracle_rate.threads, "kind": "port",
                                "sample": f"{args.cpu_steps} full time steps of the same workload (sweep + moment "
                                          f"sums + beam push), oracle on {oracle_rate.threads} host threads, "
                                          f"{el:.1f} s"}
    if rank == 0 and world == 1 and not args.no_extras and args.workload == WORKLOAD and not args.smooth:
        line.update(extras(args, r, line))
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def extras(args, r, line):
    """Measurements beside the headline (one GPU, default run): the sweep's latency roofline and FP64
    rate, and the other configurations' lines (hosing, the batched scan, the adjoint), each bounded to
    a few runs."""
    import types

    import torch

    spec, dev = r["spec"], r["dev"]
    T = spec.steps
    out = {}
    lat = sweep_latency(spec, r["beams"], dev, r["sim"], T)
    sm_mhz = (r["clocks"] or {}).get("sm_mhz") or 1965.0
    floor_cyc = sum(SLICE_FLOOR_CYCLES.values())
    floor_us = floor_cyc / sm_mhz
    lat.update({"floor_us_per_slice": floor_us, "floor_cycles_per_slice": floor_cyc,
                "floor_model": "per slice: 5 block scans x ~400 cycles (5 warp-shuffle levels, two shared-memory "
                               "round trips, the scan of 16 warp carries, one barrier) + 4 barriers x 45 cycles + one "
                               "plasma particle's dependent chain ~2,000 cycles, at the median SM clock under load",
                "frac_standalone": floor_us / lat["sweep_us_per_slice_standalone"],
                "frac_in_pipeline": floor_us / lat["sweep_us_per_slice_in_pipeline"]})
    # the cost of exact deposits: the same run with FP64 reductions for the beam deposits
    sim = r["sim"]
    sim.set_exact(False)
    fms = []
    for it in range(4):
        for b in range(len(r["init"])):
            sim.set_beam(b, r["init"][b])
        sim.run(T, spec.dt)
        if it:
            fms.append(sim.times()["kernel_ms"])
    sim.set_exact(True)
    fk = sorted(fms)[len(fms) // 2]
    out["fp64_beam_deposits"] = {"kernel_ms_per_run": fk, "value": spec.K * (T + 1) / (fk * 1e-3), "unit": UNIT,
                                 "note": "the headline run with qz_sim_set_exact(0): FP64 reductions for the beam "
                                         "deposits (run-to-run last-bit differences) instead of exact integer sums"}
    del r["sim"], sim
    torch.cuda.empty_cache()
    line["roofline"]["latency"] = lat
    kms = line["kernel_ms_per_run"]
    fl = run_flops(spec, r["nb_total"], T)
    peak64 = fp64_gemm_tflops(dev)
    sweeps = r["schedule"].get("sweep_ctas") or 1
    achieved = fl / (kms * 1e-3) / 1e12
    line["roofline"]["fp64"] = {
        "flops_per_run": fl, "achieved_tflops": achieved, "peak_tflops": peak64,
        "peak_kind": "measured here: cuBLAS DGEMM (torch.matmul float64 8192^3, best of 3); MEASURED_PEAKS.json "
                     "has no FP64 figure", "frac": achieved / peak64,
        "sweep_sms": sweeps, "frac_of_sweep_sms": achieved / (peak64 * sweeps / 148.0),
        "flops_model": "per plasma particle per slice 295, per radial node per slice 100, per beam particle per "
                       "step 180 (m = 0; counted from the reference lines the kernels restate)"}
    out["hosing"] = run_hosing_extra(dev)
    sub = types.SimpleNamespace(workload="scan", steps=1, warmup=1, time_steps=0)
    sc = run_scan(sub, 0, 1, dev.index or 0)
    rate, el = oracle_scan_rate(4, 0, 0)
    sc["cpu_baseline"] = {"value": rate, "unit": "runs/s", "cores": oracle_scan_rate.threads, "kind": "port",
                          "sample": f"one full time step of each of 4 instances sampled across the scan, oracle on "
                                    f"{oracle_scan_rate.threads} host threads, {el:.1f} s; a run = 21 such steps"}
    sc["speedup_vs_pipelined_loop"] = sc["value"] / sc["loop_runs_per_s"]["pipelined"]
    out["scan"] = {k: sc[k] for k in ("metric", "value", "unit", "ms_per_step", "config", "loop_runs_per_s",
                                      "speedup_vs_step_by_step_loop", "speedup_vs_pipelined_loop", "autotuner",
                                      "cpu_baseline")}
    torch.cuda.empty_cache()
    sub = types.SimpleNamespace(workload="adjoint", steps=2, warmup=1, time_steps=50)
    ad = run_adjoint(sub, 0, 1, dev.index or 0)
    out["adjoint"] = {k: ad[k] for k in ("metric", "value", "unit", "forward_ms", "adjoint_ms", "adjoint_split_ms",
                                         "config") if k in ad}
    if "peak_device_bytes" in ad:
        out["adjoint"]["peak_device_bytes"] = ad["peak_device_bytes"]
    return out


if __name__ == "__main__":
    main()
