"""Benchmark of the ARS(2,2,2) IMEX step: FP64 zone-updates/s.

Workload: Orszag-Tang vortex, 4096^2 periodic on [0, 2pi)^2, FP64, gamma = 5/3, eta = 1e-4, CFL 0.4
(dt = 0.9 * min(0.4 * h / s_max, h^2 / (4 eta)), chosen on the device every step). One step is one
full IMEX step (2 explicit stages, 2 implicit CG solves, finalize). One zone-update is one cell
advanced by one step. The state (805 MB) exceeds the 126 MB L2, so no flush is needed between steps.

Lines printed (rank 0, one JSON line):
  default             value = device-resident throughput; e2e = through the C ABI with the state
                      copied host->device and back every step; roofline of the dominant kernel;
                      cpu_baseline = the reference's own IMEX step (compiled here) on 1 host core.
  --impl reference    the reference's CPU implementation (oracle/_ref, compiled from the
                      reference's headers) on the same workload, a bounded sample per step, as
                      independent single-threaded replicas on the host's cores (the reference has
                      no threads of its own); value = all replicas' zone-updates/s.
The default line also carries "batched": 64 independent periodic runs of seeded sizes from
{256, 384, 512, 768, 1024}^2 (random smooth states, eta log-uniform in [1e-4, 1e-2], CFL dt per
instance), stepped as one batch (one launch per stage, CUDA graph, autotuned decomposition) and,
for comparison, as the plain per-instance loop (one context per instance, each run in turn on one
stream; and, as a second figure, the same loop with one mhd_step call per step and instance, the
reference driver's call pattern), all timed with CUDA events; and "adjoint": the differentiable form on a 1024^2 smooth
state (4 random Fourier modes, velocity amplitude 0.05, Az amplitude 0.1, rho = p = 1), eta = 5e-3,
100 fixed steps of dt = 1e-3, checkpoint every 10 steps, loss = 1/2 |rho(T) - rho_target|^2 with the
target from the forward solver at eta = 4e-3: forward and backward device times per step (the
backward recomputes each segment's explicit stages from its checkpoint) and central-difference
checks of dL/deta and of the derivative along a smooth perturbation of Az; and "snapshot": the
headline run for 100 steps with a snapshot file in the reference's format (941 MB at 4096^2) written
every 50 steps by the asynchronous writer, against the same steps without files.
Multi-GPU: replicas only (independent simulations per rank, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 zone-updates/s per IMEX step"
UNIT = "zone-updates/s"
N_GRID = 4096
ETA = 1e-4
COURANT = 0.4
WORKLOAD = "orszag_tang_4096x4096_eta1e-4_cfl0.4"

# Algorithmic bytes per zone of each kernel (compulsory-traffic model of the reference algorithm):
# stage 1 reads U^n (48), writes the accumulator (48), the predictor (48) and the solve's
# right-hand side (8) = 152; each CG iteration reads and writes x, r, p = 48; stage 2 reads U1*
# (48), E1 (8), the accumulator (48), writes U2* (48) and the right-hand side (8) = 160; finalize
# reads B2* (16), E2 (8), hydro for the CFL (32), writes B^{n+1} (16) = 72.
# Per step: 384 + 48 * (k1 + k2) bytes per zone.
ALG_BYTES = {"stage1": 152.0, "stage2": 160.0, "finalize": 72.0, "cg_per_iter": 48.0}
KERNELS = ("stage1", "cg1", "stage2", "cg2", "finalize")


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs. The sampler is
    running (first sample received) before the region starts and takes one more sample after it
    ends, so the reported samples bracket the region even when it is shorter than the interval."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []  # (wall time, csv line)
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.time() + 10.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *a):
        self.t1 = time.time()
        if self.proc is not None:
            deadline = time.time() + 2.0
            while time.time() < deadline and self.proc.poll() is None and \
                    not any(t >= self.t1 for t, _ in self.lines):
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples inside the region, plus the last one before and the first one after it
        inside = [ln for t, ln in self.lines if self.t0 <= t <= self.t1]
        before = [ln for t, ln in self.lines if t < self.t0][-1:]
        after = [ln for t, ln in self.lines if t > self.t1][:1]
        for ln in before + inside + after:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "samples_inside_region": len(inside)}


def make_state(n):
    import magnetohydrodynamics_simulator_b200 as m

    dx = m.problems.grid_spacing(n)
    return m.problems.orszag_tang(n, n, dx, dx), dx


def cpu_reference_step_rate(n, steps, warmup=0):
    """Time `steps` steps of the reference's own driver loop (oracle/_ref: CFL_condition_checker,
    generate_A_matrix + compute when dt changes -- every step here -- and IMEX) at n^2, after
    `warmup` untimed steps; returns (zone-updates/s, seconds). Building the initial state is
    outside the timed region."""
    from oracle.oracle import Reference, reference_available

    if not reference_available():
        return None
    state, dx = make_state(n)
    ref = Reference(n, n, dx, dx, ETA)
    ref.set_state(state)
    if warmup:
        ref.run(warmup)
    t0 = time.perf_counter()
    ref.run(steps)
    sec = time.perf_counter() - t0
    return n * n * steps / sec, sec


# Host memory of one reference simulation (grids, workspace, reconstruction, sparse matrix),
# measured at 512^2: about 1.1 kB per zone.
REF_BYTES_PER_ZONE = 1200


def max_over_ranks(dist, value, device="cpu"):
    """The largest of every rank's value: multi-rank times are the slowest rank's."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _reference_replica(core, n, steps, warmup, conn):
    """One reference simulation in its own process, pinned to one host core."""
    try:
        if core is not None:
            os.sched_setaffinity(0, {core})
        conn.send(cpu_reference_step_rate(n, steps, warmup))
    except Exception as e:  # reported, not raised: the parent decides
        conn.send(repr(e))
    conn.close()


def reference_replicas(n, steps, warmup, procs):
    """`procs` independent reference simulations at once, one per host core (the reference is
    single-threaded, so replicas are how it uses the host's cores). Returns the whole-job
    zone-updates/s (procs * n^2 * steps / the slowest replica's time) and that time."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    cores = sorted(os.sched_getaffinity(0))
    jobs = []
    for k in range(procs):
        a, b = ctx.Pipe(duplex=False)
        p = ctx.Process(target=_reference_replica, args=(cores[k % len(cores)], n, steps, warmup, b))
        p.start()
        jobs.append((p, a))
    results = []
    for p, a in jobs:
        try:
            results.append(a.recv())
        except EOFError:  # the process died without an answer (killed, out of memory, ...)
            p.join()
            results.append(f"replica process ended without a result (exit code {p.exitcode})")
        p.join()
    bad = [r for r in results if not isinstance(r, tuple)]
    if bad:
        raise RuntimeError(f"reference replica failed: {bad[0]}")
    sec = max(r[1] for r in results)
    return procs * n * n * steps / sec, sec


def run_reference_arm(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from oracle.oracle import reference_available

    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmhdref.so was not built "
                          "(the reference sources were absent when __graft_entry__.build() ran)"}))
        return 0
    # Each step is a bounded sample of the workload: one IMEX step of the same Orszag-Tang
    # problem on the largest grid (<= 4096^2) whose K + 1 steps fit in ~60 s of one core (sized
    # from a timed 512^2 probe step), run as independent replicas on as many host cores as the
    # host memory holds.
    probe_rate, _ = cpu_reference_step_rate(512, 1)
    budget = 60.0
    n = 4096
    while n > 256 and (args.steps + 1) * n * n / probe_rate > budget:
        n //= 2
    try:
        import psutil

        avail = psutil.virtual_memory().available
    except Exception:
        avail = 8 << 30
    cores = len(os.sched_getaffinity(0))
    procs = max(1, min(cores, int(0.5 * avail // (REF_BYTES_PER_ZONE * n * n))))
    warm = min(args.warmup, 1)
    rate, sec = reference_replicas(n, args.steps, warm, procs)
    sample = (f"{args.steps} steps of the reference driver loop (its own CFL dt, matrix rebuilt "
              f"each step, IMEX) on the Orszag-Tang problem at {n}x{n}, eta 1e-4, after "
              f"{warm} untimed step, in each of {procs} concurrent single-threaded replicas pinned "
              f"to {procs} of the host's {cores} cores (slowest replica's time); reference headers "
              f"compiled -O3 -ffast-math")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "grid": [N_GRID, N_GRID], "sampled_grid": [n, n],
                   "eta": ETA, "cfl": COURANT, "parallelism": f"replicas{args.gpus}"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_gpu_arm(args):
    import torch

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        from datetime import timedelta

        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    import magnetohydrodynamics_simulator_b200 as m

    n = args.grid
    state, dx = make_state(n)
    # wall-clock limit of one implicit solve (a profiler replaying the persistent solver can
    # lower it so that no replay pass can wait long)
    cg_timeout = float(os.environ.get("MHD_B200_CG_TIMEOUT_S", "30"))
    ctx = m.Context(n, n, dx, dx, ETA, courant=COURANT, cg_timeout_s=cg_timeout)
    ctx.set_state(state)
    stream = torch.cuda.ExternalStream(ctx.stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- warm-up
    for _ in range(args.warmup):
        ctx.step(0.0)
    ctx.synchronize()

    # ---- timed region: K steps, device-resident inputs, CFL dt on the device
    ctx.lib.mhd_set_kernel_timing(ctx.h, 1)
    sum0 = ctx.cg_products_sum()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            ctx.step(0.0)
        stop.record(stream)
        stop.synchronize()
    barrier()
    status = ctx.synchronize_status()
    ms = start.elapsed_time(stop)
    sum1 = ctx.cg_products_sum()
    divb_after = ctx.divb()  # |div B| of the state the timed steps left (outside the timing)
    import ctypes

    kt = (ctypes.c_double * 5)()
    ksteps = ctypes.c_longlong()
    ctx.lib.mhd_kernel_times(ctx.h, kt, ctypes.byref(ksteps))
    ctx.lib.mhd_set_kernel_timing(ctx.h, 0)
    prods = ctx.last_cg_products()
    ms_max = max_over_ranks(dist, ms, "cuda")
    zones = float(n) * n
    value = world * zones * args.steps / (ms_max * 1e-3)

    # ---- end to end through the C ABI with host buffers: every step uploads its input state from
    # pinned host memory and reads its result back. Pipelined form (mhd_set_state_async /
    # mhd_get_state_async): in quarter planes on two copy streams, so one step's read-back overlaps
    # the next step's upload; the timed region ends when the last read-back is in host memory.
    pinned = [torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy() for _ in range(6)]
    ctx.get_state_into(pinned)
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        ctx.set_state_async(pinned)
        ctx.step(0.0)
        ctx.get_state_async(pinned)
    ctx.transfers_wait()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(dist, e0.elapsed_time(e1), "cuda")
    e2e_value = world * zones * e2e_steps / (e2e_ms * 1e-3)
    # the same with the synchronous calls (mhd_set_state, mhd_step, mhd_get_state per step)
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(e2e_steps):
        ctx.set_state(pinned)
        ctx.step(0.0)
        ctx.get_state_into(pinned)
    s1.record(stream)
    s1.synchronize()
    e2e_sync_ms = max_over_ranks(dist, s0.elapsed_time(s1), "cuda")
    status2 = ctx.synchronize_status()
    # both transfer modes are public calls; a host link that does not overlap its two directions
    # gains nothing from the pipelined one, so the line reports the faster mode of this box
    e2e_modes = {
        "pipelined": {"value": e2e_value, "ms_per_step": e2e_ms / e2e_steps,
                      "how": "mhd_set_state_async + mhd_step + mhd_get_state_async per step from pinned "
                             "host planes (read-back and next upload overlap piece by piece)"},
        "synchronous": {"value": world * zones * e2e_steps / (e2e_sync_ms * 1e-3),
                        "ms_per_step": e2e_sync_ms / e2e_steps,
                        "how": "mhd_set_state + mhd_step + mhd_get_state per step from pinned host planes"},
    }
    e2e_mode = max(e2e_modes, key=lambda k: e2e_modes[k]["value"])
    e2e = {"value": e2e_modes[e2e_mode]["value"], "unit": UNIT, "h2d_bytes_per_step": int(6 * zones * 8),
           "d2h_bytes_per_step": int(6 * zones * 8), "steps": e2e_steps, "mode": e2e_mode,
           "how": e2e_modes[e2e_mode]["how"], "modes": e2e_modes}

    # ---- roofline of the dominant kernel (per-kernel CUDA events over the timed region)
    peak, peak_kind = load_peaks()
    ksum = dict(zip(KERNELS, list(kt)))
    steps_rec = max(1, ksteps.value)
    # mean products of each solve over the timed steps (device-side running sums read around it)
    k1 = (sum1[0] - sum0[0]) / args.steps
    k2 = (sum1[1] - sum0[1]) / args.steps
    per_kernel = {}
    for name in KERNELS:
        avg_ms = ksum[name] / steps_rec
        if name == "cg1":
            alg = ALG_BYTES["cg_per_iter"] * k1
        elif name == "cg2":
            alg = ALG_BYTES["cg_per_iter"] * k2
        else:
            alg = ALG_BYTES[name]
        gbs = alg * zones / (avg_ms * 1e-3) / 1e9
        per_kernel[name] = {"ms": avg_ms, "alg_bytes_per_zone": alg, "achieved_gbs": gbs,
                            "frac": gbs / peak}
    # the solver kernel (k_cg_sweep) runs twice per step: its share of the step is both launches
    solver_ms = per_kernel["cg1"]["ms"] + per_kernel["cg2"]["ms"]
    solver_gbs = ALG_BYTES["cg_per_iter"] * (k1 + k2) * zones / (solver_ms * 1e-3) / 1e9
    step_kernels_ms = sum(per_kernel[k]["ms"] for k in KERNELS)
    shares = {"k_stage_sweep<1>": per_kernel["stage1"]["ms"] / step_kernels_ms,
              "k_cg_sweep": solver_ms / step_kernels_ms,
              "k_stage_sweep<2>": per_kernel["stage2"]["ms"] / step_kernels_ms,
              "k_finalize_sweep": per_kernel["finalize"]["ms"] / step_kernels_ms}
    longest = max(KERNELS, key=lambda k: per_kernel[k]["ms"])
    # per kernel function: (per-launch algorithmic bytes, mean launch ms, launches per step, key of
    # its measured DRAM bytes per zone and per unit, units per launch)
    funcs = {
        "k_stage_sweep<1>": (ALG_BYTES["stage1"] * zones, per_kernel["stage1"]["ms"], 1, "stage1", 1),
        "k_cg_sweep": (ALG_BYTES["cg_per_iter"] * (k1 + k2) / 2 * zones, solver_ms / 2, 2, "cg", (k1 + k2) / 2),
        "k_stage_sweep<2>": (ALG_BYTES["stage2"] * zones, per_kernel["stage2"]["ms"], 1, "stage2", 1),
        "k_finalize_sweep": (ALG_BYTES["finalize"] * zones, per_kernel["finalize"]["ms"], 1, "finalize", 1),
    }
    dominant = max(funcs, key=lambda f: shares[f])  # the largest share of the step's time
    tr = {}
    tr_path = os.path.join(ROOT, "profiles", "dram_bytes_per_zone.json")
    if os.path.exists(tr_path):
        try:
            with open(tr_path) as f:
                tr = json.load(f)
        except Exception:
            tr = {}

    def traffic_of(name):
        _, _, _, key, units = funcs[name]
        if key not in tr:
            return None
        return tr[key]["bytes_per_zone_per_unit"] * units * zones

    # FP64-pipe bound of each kernel from its ncu-counted FP64 thread instructions per zone: B200
    # issues 64 per SM and clock (148 SMs at the 1965 MHz maximum SM clock)
    fi = {}
    fi_path = os.path.join(ROOT, "profiles", "fp64_inst_per_zone.json")
    if os.path.exists(fi_path):
        try:
            with open(fi_path) as f:
                fi = json.load(f)
        except Exception:
            fi = {}

    def fp64_of(name, ms, alg):
        _, _, _, key, units = funcs[name]
        if key not in fi:
            return None
        inst = fi[key]["fp64_thread_inst_per_zone_per_unit"] * units * zones
        rate_peak = fi.get("fp64_thread_inst_per_sm_per_clock", 64) * 148 * 1965e6
        t_fp64 = inst / rate_peak
        t_hbm = alg / (peak * 1e9)
        return {"thread_inst_per_launch": inst, "achieved_inst_per_s": inst / (ms * 1e-3),
                "peak_inst_per_s": rate_peak, "frac": t_fp64 / (ms * 1e-3),
                "flops_per_launch": fi[key]["flops_per_zone_per_unit"] * units * zones,
                "binding_roofline": "fp64" if t_fp64 > t_hbm else "hbm",
                "hbm_frac_at_fp64_peak": min(1.0, t_hbm / t_fp64)}

    def figures(name):
        alg, ms, launches, _, _ = funcs[name]
        gbs = alg / (ms * 1e-3) / 1e9
        return {"kernel": name, "launches_per_step": launches, "share_of_step": shares[name],
                "alg_bytes_per_launch": alg, "ms_per_launch": ms, "achieved": gbs, "frac": gbs / peak,
                "traffic": traffic_of(name), "fp64_pipe": fp64_of(name, ms, alg)}

    dom = figures(dominant)
    longest_name = {"stage1": "k_stage_sweep<1>", "cg1": "k_cg_sweep", "stage2": "k_stage_sweep<2>",
                    "cg2": "k_cg_sweep", "finalize": "k_finalize_sweep"}[longest]
    step_alg = (384.0 + 48.0 * (k1 + k2)) * zones
    step_ms = ms_max / args.steps
    roofline = {
        "bound": "hbm", "kernel": dominant,
        "achieved": dom["achieved"], "peak": peak, "unit": "GB/s", "frac": dom["frac"],
        "traffic": dom["traffic"], "peak_source": peak_kind,
        "kernel_is": "the kernel with the largest share of the step's time (per launch: its "
                     "algorithmic bytes over its mean launch time)",
        "longest_launch": figures(longest_name),
        "per_function": {f: figures(f) for f in funcs},
        "shares": shares,
        "step": {"alg_bytes_per_zone": 384.0 + 48.0 * (k1 + k2),
                 "achieved": step_alg / (step_ms * 1e-3) / 1e9,
                 "frac": step_alg / (step_ms * 1e-3) / 1e9 / peak},
        "kernels": per_kernel,
    }

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = headline_parity(ctx, state, n, dx)
    if parity is not None:
        parity["divb_after_timed_steps"] = {"steps": args.warmup + args.steps, "rms": divb_after[0],
                                            "max": divb_after[1]}
    clk = clocks.summary()
    batched = None
    if not args.no_batch:
        batched = measure_batched(torch, m, args.batch_steps)
        # the single context's solver on the headline grid, per zone and matrix product
        batched["solver_work"]["single_context_ps_per_zone_product"] = (
            solver_ms * 1e9 / (zones * (k1 + k2)))
    adjoint = None
    if not args.no_adjoint:
        adjoint = measure_adjoint(torch, m)
    snapshot = None
    if not args.no_snapshot and rank == 0:
        snapshot = measure_snapshots(torch, m, ctx)
    decomposed = None
    if not args.no_decomposed and rank == 0:
        decomposed = measure_decomposed(torch, m)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if n == N_GRID else f"orszag_tang_{n}x{n}_eta1e-4_cfl0.4",
                   "grid": [n, n], "eta": ETA, "cfl": COURANT,
                   "parallelism": f"replicas{world}", "l2": "inputs exceed L2 (805 MB state)",
                   "cg_products_last_step": list(prods),
                   "cg_products_mean_per_step": [k1, k2]},
        "e2e": e2e,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clk,
        "gpu_launches": args.steps * ctx.launches_per_step,
        "status": [status, status2],
        "batched": batched,
        "adjoint": adjoint,
        "snapshot": snapshot,
        "decomposed": decomposed,
    }
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def headline_parity(ctx, state, n, dx):
    """One step of the headline problem from its initial state, on the GPU (the context, dt = its
    CFL step) and in the reference's own code (oracle/_ref, the reference driver loop given the
    same dt: CFL evaluation, matrix build, IMEX), compared field by field. The reference step is
    timed too: it is the CPU baseline (1 host core; the reference is single-threaded). Returns
    (cpu_baseline, parity)."""
    from oracle.oracle import Reference, reference_available, rel_linf

    if not reference_available():
        return None, None
    ctx.set_state(state)
    dt = ctx.cfl_dt()
    ctx.step(dt)
    st = ctx.synchronize_status()
    got = ctx.get_state()
    g_rms, g_max = ctx.divb()
    prods = ctx.last_cg_products()
    ref = Reference(n, n, dx, dx, ETA)
    ref.set_state(state)
    t0 = time.perf_counter()
    ref.cfl_dt()
    _, rprods = ref.run(1, dts=np.array([dt]))
    sec = time.perf_counter() - t0
    want = ref.get_state()
    r_rms, r_max = ref.divb()
    names = ("rho", "mx", "my", "E", "bxf", "byf")
    errs = {k: rel_linf(g, w) for k, g, w in zip(names, got, want)}
    del ref
    cpu = {"value": n * n / sec, "unit": UNIT, "cores": 1, "kind": "reference",
           "sample": f"1 step of the reference driver loop (CFL evaluation, matrix build, IMEX) on "
                     f"the {n}x{n} Orszag-Tang initial state with the GPU's dt; reference headers "
                     f"compiled -O3 -ffast-math, single thread, {sec:.1f} s"}
    parity = {"what": f"one step from the {n}x{n} Orszag-Tang initial state, dt = {dt!r} (the GPU's "
                      f"CFL 0.4 step), GPU against the reference's own IMEX (oracle/_ref)",
              "rel_linf_per_field": errs, "max_rel_linf": max(errs.values()), "bar": 1e-10,
              "divb_max": {"gpu": g_max, "reference": r_max}, "divb_rms": {"gpu": g_rms, "reference": r_rms},
              "cg_products": {"gpu": list(prods), "reference": [int(x) for x in rprods[0]]},
              "status": st}
    return cpu, parity


BATCH_WORKLOAD = "mixed64_sizes256-1024_seed2024_eta1e-4..1e-2_cfl0.5"


def measure_snapshots(torch, m, ctx, steps=100, every=50):
    """Snapshot files in the reference's format (mhd_snapshot_write) every `every` steps of the
    headline run, against the same steps without them: device time of the steps on the context's
    stream, and wall time until the files are on disk. One snapshot is written first, so that the
    writer's buffers exist before the timed region. Files go to a temporary directory. At 4096^2 a
    file is 941 MB, a few tenths of a second of disk writing: the interval leaves the disk time to
    keep up (a shorter one makes the writer's two slots, and so the stepping, wait for the disk)."""
    import tempfile

    stream = torch.cuda.ExternalStream(ctx.stream)
    nchunks = max(1, steps // every)

    def timed(folder):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for k in range(nchunks):
            ctx.run(every, record=False)
            if folder:
                ctx.snapshot_write(os.path.join(folder, f"snapshot_{k:06d}.dat"), 2, every, 0.0)
        e1.record(stream)
        e1.synchronize()
        if folder:
            ctx.snapshot_wait()
        return e0.elapsed_time(e1), time.perf_counter() - t0

    with tempfile.TemporaryDirectory() as folder:
        ctx.snapshot_write(os.path.join(folder, "warmup.dat"), 2, every, 0.0)
        ctx.snapshot_wait()
        plain_ms, _ = timed(None)
        snap_ms, wall_s = timed(folder)
    nbytes = ctx.snapshot_bytes(2)
    return {
        "what": f"{nchunks} snapshot files (ng = 2) written every {every} steps while stepping",
        "bytes_per_snapshot": nbytes,
        "ms_per_step_plain": plain_ms / (nchunks * every),
        "ms_per_step_with_snapshots": snap_ms / (nchunks * every),
        "files_on_disk_s": wall_s,
        "file_write_GBps": nchunks * nbytes / wall_s / 1e9,
    }


def measure_decomposed(torch, m, n=4096, P=2, Q=2, steps=3):
    """The domain decomposition on one GPU: Orszag-Tang n^2 split P x Q, subdomains exchanging
    their rings by device kernels (the ranks of a multi-GPU run emulated in one process),
    against a single context on the same steps; wall time per step and the largest per-field
    difference. Three forms of the solve: the single-sweep solver with its decisions on the device
    (the default: each iteration one replayed CUDA graph, the host polling a control block one
    iteration behind), the two-sweep solve with decisions on the device, and the same with every
    product's sums read back by the host (these two must agree bit for bit)."""
    from magnetohydrodynamics_simulator_b200.decomposed import (DecomposedRun, GpuSubdomain,
                                                                LocalTransport, Partition)

    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    part = Partition(n, n, P, Q)
    start, dts, runs = None, None, {}
    forms = {"sweep_device": (True, "sweep"), "two_sweep_device": (True, "two_sweep"),
             "two_sweep_host": (False, "two_sweep")}
    for mode, (device, form) in forms.items():
        subs = [GpuSubdomain(*part.shape(i), dx, dx, ETA) for i in range(part.count)]
        run = DecomposedRun(part, LocalTransport(part, subs), dx, dx, ETA, courant=COURANT,
                            device_decisions=device, cg_form=form)
        run.set_state(ic)
        run.step()  # warm-up
        if start is None:
            start = run.get_state()
        else:
            run.set_state(start)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        got_dts, prods = [], []
        for k in range(steps):
            dt, kk = run.step(0.0 if dts is None else dts[k])
            got_dts.append(dt)
            prods.append(kk)
        torch.cuda.synchronize()
        runs[mode] = dict(ms=1e3 * (time.perf_counter() - t0) / steps, prods=prods, state=run.get_state(),
                          divb=run.divb()[1], status=run.status)
        dts = dts or got_dts
        run.close()
        for sd in subs:
            sd.close()
    ctx = m.Context(n, n, dx, dx, ETA, courant=COURANT)
    ctx.set_state(start)
    ctx.step(dts[0])  # warm-up of the single context, then the same steps again from the start
    ctx.set_state(start)
    ctx.synchronize()
    t1 = time.perf_counter()
    for dt in dts:
        ctx.step(dt)
    ctx.synchronize()
    single = time.perf_counter() - t1
    want = ctx.get_state()

    def err(mode):
        return max(float(np.max(np.abs(g - w)) / max(float(np.max(np.abs(w))), 1.0))
                   for g, w in zip(runs[mode]["state"], want))

    a, b = runs["two_sweep_device"], runs["two_sweep_host"]
    same = all(np.array_equal(x, y) for x, y in zip(a["state"], b["state"])) and a["prods"] == b["prods"]
    out = {"what": f"Orszag-Tang {n}x{n} split {P}x{Q} on one GPU (rings by device kernels), "
                   f"{steps} CFL steps, against a single context stepped with the same dts",
           "ms_per_step_decomposed": runs["sweep_device"]["ms"],
           "ms_per_step_two_sweep_device_decisions": a["ms"],
           "ms_per_step_two_sweep_host_decisions": b["ms"],
           "ms_per_step_single_context": 1e3 * single / steps,
           "cg_products": runs["sweep_device"]["prods"],
           "max_rel_linf_vs_single": err("sweep_device"),
           "max_rel_linf_vs_single_two_sweep": err("two_sweep_device"),
           "two_sweep_device_and_host_decisions_bit_identical": bool(same),
           "divb_max": runs["sweep_device"]["divb"], "status": runs["sweep_device"]["status"],
           "note": "wall time; the default form: the single context's single-sweep solver on every "
                   "subdomain, one CUDA graph per iteration, the host polling the solve's control "
                   "block one iteration behind"}
    ctx.close()
    return out


def measure_batched(torch, m, steps):
    """Batched stepping of the mixed-size batch vs the plain per-instance loop (same inputs,
    same steps, CFL dt per instance). Returns the "batched" object of the JSON line."""
    specs = m.problems.mixed_batch(64)
    insts, ics = [], []
    for n_i, eta_i, seed_i in specs:
        fields, dx_i = m.problems.random_instance(n_i, seed_i)
        insts.append(dict(nx=n_i, ny=n_i, dx=dx_i, dy=dx_i, eta=eta_i))
        ics.append(fields)
    zones = float(sum(s["nx"] * s["ny"] for s in insts))

    b = m.Batch(insts)
    for i, f in enumerate(ics):
        b.set_state(i, f)
    tuning = b.autotune()
    # the work of the solves in the tuning step: one step of the chosen decomposition from the same
    # initial states gives every instance's products (the states are set again before timing)
    b.step()
    b.synchronize()
    prods0 = b.last_cg_products()
    zone_products = float(sum(s["nx"] * s["ny"] * int(p[0] + p[1]) for s, p in zip(insts, prods0)))
    bstream = torch.cuda.ExternalStream(b.stream)
    b.run(4, record=False)  # warm-up (graph capture path included)
    for i, f in enumerate(ics):
        b.set_state(i, f)
    b.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(bstream)
    b.run(steps, record=False)
    e1.record(bstream)
    e1.synchronize()
    batch_ms = e0.elapsed_time(e1)
    worst, _ = b.synchronize_status()
    launches = b.launches_per_step
    b.close()

    # plain loop: one context per instance on one shared stream, each advanced `steps` steps in turn
    shared = torch.cuda.Stream()
    ctxs = []
    for s, f in zip(insts, ics):
        c = m.Context(s["nx"], s["ny"], s["dx"], s["dy"], s["eta"], stream=shared.cuda_stream)
        c.set_state(f)
        c.run(4, record=False)  # warm-up
        c.set_state(f)
        ctxs.append(c)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(shared)
    for c in ctxs:
        c.run(steps, record=False)
    p1.record(shared)
    p1.synchronize()
    plain_ms = p0.elapsed_time(p1)
    # the same loop in the drop-in call pattern: one mhd_step per step and instance (CFL dt on the
    # device), as the reference's driver calls IMEX once per step, without graph capture
    for c, f in zip(ctxs, ics):
        c.set_state(f)
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(shared)
    for c in ctxs:
        for _ in range(steps):
            c.step(0.0)
    q1.record(shared)
    q1.synchronize()
    step_calls_ms = q0.elapsed_time(q1)
    for c in ctxs:
        c.close()
    return {
        "workload": BATCH_WORKLOAD, "instances": len(insts), "steps": steps,
        "zones_per_step": int(zones), "value": zones * steps / (batch_ms * 1e-3), "unit": UNIT,
        "ms_per_step": batch_ms / steps, "launches_per_step": launches,
        "tuning": {k: tuning[k] for k in ("stage_rows", "cg_rows", "cg_order")},
        "tuning_step_ms": {"explicit_kernels": tuning["stage_ms"], "implicit_solves": tuning["cg_ms"],
                           "note": "device time of one autotuning step of the chosen decomposition"},
        "solver_work": {"zone_products": zone_products,
                        "mean_products_per_solve": zone_products / (2.0 * zones),
                        "ps_per_zone_product": tuning["cg_ms"] * 1e9 / zone_products,
                        "note": "the tuning step's solves: every instance's matrix products times "
                                "its zones; converged instances drop out of the lockstep"},
        "plain_loop": {"value": zones * steps / (plain_ms * 1e-3), "unit": UNIT,
                       "ms_per_step": plain_ms / steps,
                       "how": "one context per instance on one stream, run(steps) in turn (CUDA graph, "
                              "dt and matrix rule on the device)"},
        "speedup_vs_plain_loop": plain_ms / batch_ms,
        "plain_loop_step_calls": {
            "value": zones * steps / (step_calls_ms * 1e-3), "unit": UNIT,
            "ms_per_step": step_calls_ms / steps, "speedup_of_batch": step_calls_ms / batch_ms,
            "how": "the same contexts, one mhd_step (CFL dt on the device) per step and instance, "
                   "instances in turn, no graph capture: the reference driver's call pattern"},
        "status": worst,
    }


ADJ_WORKLOAD = "adjoint_1024x1024_4modes_v0.05_az0.1_eta5e-3_dt1e-3_100steps_ckpt10"


def measure_adjoint(torch, m, n=1024, nsteps=100, every=10, dt=1e-3, eta=5e-3):
    """Forward / backward device time of the differentiable trajectory and a gradient check."""
    from magnetohydrodynamics_simulator_b200.autograd import state_from_potential, trajectory

    dev = "cuda"
    dx = 2 * np.pi / n
    rng = np.random.default_rng(5)
    x = np.arange(n) * dx
    X, Y = np.meshgrid(x, x)

    def modes(amp, shift):
        f = np.zeros((n, n))
        for _ in range(4):
            kx, ky = rng.integers(-4, 5, size=2)
            f += amp * rng.uniform(0.5, 1.0) * np.sin(kx * (X + shift) + ky * (Y + shift) + rng.uniform(0, 2 * np.pi))
        return torch.tensor(f, device=dev)

    vx, vy = modes(0.05, dx / 2), modes(0.05, dx / 2)
    az0, daz = modes(0.1, 0.0), modes(0.1, 0.0)
    one = torch.ones(n, n, dtype=torch.float64, device=dev)
    adj = m.Adjoint(n, n, dx, dx, eta, dt, nsteps, checkpoint_every=every)
    astream = torch.cuda.ExternalStream(adj.stream)

    def u0_of(az):
        return state_from_potential(az, one, vx, vy, one, dx, dx).contiguous()

    def loss(az, eta_v, target):
        uT = trajectory(u0_of(az), torch.tensor(eta_v, dtype=torch.float64, device=dev), adj)
        return 0.5 * ((uT[0] - target) ** 2).sum()

    with torch.no_grad():
        target = trajectory(u0_of(az0), torch.tensor(0.8 * eta, dtype=torch.float64, device=dev), adj)[0].clone()
    # warm-up forward + backward
    az = az0.clone().requires_grad_(True)
    loss(az, eta, target).backward()
    # timed: device time of the library calls, events on the library's stream
    u0 = u0_of(az0)
    uT = torch.empty_like(u0)
    gT = torch.randn_like(u0)
    g0 = torch.empty_like(u0)
    ptr = lambda t: [t[k].data_ptr() for k in range(6)]  # noqa: E731
    adj.set_eta(eta)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(astream)
    adj.forward(ptr(u0), ptr(uT))
    ev[1].record(astream)
    adj.backward(ptr(gT), ptr(g0))
    ev[2].record(astream)
    ev[2].synchronize()
    fwd_ms, bwd_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    # gradients through torch.autograd vs central differences of the forward solver, taken on the
    # final state (difference of two trajectories, contracted afterwards)
    az = az0.clone().requires_grad_(True)
    eta_t = torch.tensor(eta, dtype=torch.float64, device=dev, requires_grad=True)
    uTg = trajectory(u0_of(az), eta_t, adj)
    L0 = 0.5 * ((uTg[0] - target) ** 2).sum()
    L0.backward()
    g_eta, g_dir_loss = float(eta_t.grad), float((az.grad * daz).sum())
    w = torch.randn(target.shape, generator=torch.Generator(device=dev).manual_seed(3),
                    dtype=torch.float64, device=dev)
    az = az0.clone().requires_grad_(True)
    e0 = torch.tensor(eta, dtype=torch.float64, device=dev)
    (trajectory(u0_of(az), e0, adj)[0] * w).sum().backward()
    g_dir = float((az.grad * daz).sum())
    with torch.no_grad():
        h = 1e-3 * eta
        rp, rm = trajectory(u0_of(az0), e0 + h, adj)[0], trajectory(u0_of(az0), e0 - h, adj)[0]
        fd_eta = float((((rp - rm) / (2 * h)) * ((rp + rm) / 2 - target)).sum())
        s_ = 3e-7
        rp = trajectory(u0_of(az0 + s_ * daz), e0, adj)[0]
        rm = trajectory(u0_of(az0 - s_ * daz), e0, adj)[0]
        fd_dir = float((((rp - rm) / (2 * s_)) * w).sum())
        fd_dir_loss = float((((rp - rm) / (2 * s_)) * ((rp + rm) / 2 - target)).sum())
        # the same difference at half the step, and their Richardson combination (4 D(s/2) - D(s)) / 3,
        # which removes an O(s^2) error term where the scheme is smooth
        rp2 = trajectory(u0_of(az0 + 0.5 * s_ * daz), e0, adj)[0]
        rm2 = trajectory(u0_of(az0 - 0.5 * s_ * daz), e0, adj)[0]
        fd_dir_half = float((((rp2 - rm2) / s_) * w).sum())
        fd_dir_rich = (4.0 * fd_dir_half - fd_dir) / 3.0
    f_launch, a_launch = adj.launch_counts()
    mem_default = adj.device_bytes
    adj.close()
    # the memory-bounded mode: one segment's solutions kept, each segment re-solved backwards
    adj2 = m.Adjoint(n, n, dx, dx, eta, dt, nsteps, checkpoint_every=every, recompute_solves=True)
    a2stream = torch.cuda.ExternalStream(adj2.stream)
    g0b = torch.empty_like(u0)
    adj2.set_eta(eta)
    torch.cuda.synchronize()
    ev2 = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev2[0].record(a2stream)
    adj2.forward(ptr(u0), ptr(uT))
    ev2[1].record(a2stream)
    adj2.backward(ptr(gT), ptr(g0b))
    ev2[2].record(a2stream)
    ev2[2].synchronize()
    rec_fwd_ms, rec_bwd_ms = ev2[0].elapsed_time(ev2[1]), ev2[1].elapsed_time(ev2[2])
    mem_recompute = adj2.device_bytes
    same = bool(torch.equal(g0, g0b))
    adj2.close()
    return {
        "workload": ADJ_WORKLOAD, "grid": [n, n], "steps": nsteps, "checkpoint_every": every,
        "forward_ms_per_step": fwd_ms / nsteps, "backward_ms_per_step": bwd_ms / nsteps,
        "adjoint_over_forward": bwd_ms / fwd_ms,
        "backward_includes": "recomputation of each segment's explicit stages from its checkpoint "
                             "(the implicit solutions of every step are kept by the forward pass)",
        "launches_per_step": {"forward": f_launch, "backward": a_launch},
        "device_bytes": mem_default,
        "recompute_solves": {"device_bytes": mem_recompute,
                             "forward_ms_per_step": rec_fwd_ms / nsteps,
                             "backward_ms_per_step": rec_bwd_ms / nsteps,
                             "adjoint_over_forward": rec_bwd_ms / rec_fwd_ms,
                             "gradient_bit_identical": same},
        "gradient_check": {
            "method": "central differences of the final state (two trajectories), contracted after",
            "d_eta": {"loss": "1/2|rho(T) - rho_target|^2", "adjoint": g_eta,
                      "central_difference": fd_eta, "step": 1e-3 * eta,
                      "rel_err": abs(g_eta - fd_eta) / abs(fd_eta)},
            "d_az_direction": {"loss": "<w, rho(T)>, w ~ N(0,1)", "adjoint": g_dir,
                               "central_difference": fd_dir, "step": 3e-7,
                               "rel_err": abs(g_dir - fd_dir) / abs(fd_dir),
                               "central_difference_half_step": fd_dir_half,
                               "rel_err_half_step": abs(g_dir - fd_dir_half) / abs(fd_dir_half),
                               "richardson": fd_dir_rich,
                               "rel_err_richardson": abs(g_dir - fd_dir_rich) / abs(fd_dir_rich)},
            "d_az_direction_density_loss": {"loss": "1/2|rho(T) - rho_target|^2", "adjoint": g_dir_loss,
                                            "central_difference": fd_dir_loss, "step": 3e-7,
                                            "rel_err": abs(g_dir_loss - fd_dir_loss) / abs(fd_dir_loss)},
        },
    }


def run_profile_case(args):
    """Small fixed cases for profilers (nothing is timed or printed as a result):
    batched  the mixed 64-instance batch of the "batched" section, two CFL steps at the
             decomposition the autotuner picks for it (stage rows 192, tail 32, solver tiles of a
             height chosen phase by phase), no autotuning;
    adjoint  the 1024^2 state of the "adjoint" section, one 10-step trajectory (one checkpoint
             segment): forward, then backward;
    snapshot the Orszag-Tang state at 2048^2 (201 MB, above the L2), one step, then one snapshot
             packed on the device and copied to the host (mhd_snapshot_pack, 235 MB);
    decomposed  Orszag-Tang 2048^2 split 2 x 2 on one GPU (the default single-sweep solve with
             device decisions), one warm-up step and two CFL steps;
    step     the Orszag-Tang state at 2048^2 (201 MB, above the L2), two CFL steps of a single
             context (the headline workload's kernels at a quarter of its zones)."""
    import torch

    import magnetohydrodynamics_simulator_b200 as m

    torch.cuda.set_device(0)
    if args.profile_case == "step":
        n = 2048
        state, dx = make_state(n)
        ctx = m.Context(n, n, dx, dx, ETA, courant=COURANT)
        ctx.set_state(state)
        for _ in range(2):
            ctx.step(0.0)
        st = ctx.synchronize_status()
        ctx.close()
        return 0 if st == 0 else 1
    if args.profile_case == "decomposed":
        from magnetohydrodynamics_simulator_b200.decomposed import (DecomposedRun, GpuSubdomain,
                                                                    LocalTransport, Partition)

        n = 2048
        state, dx = make_state(n)
        part = Partition(n, n, 2, 2)
        subs = [GpuSubdomain(*part.shape(i), dx, dx, ETA) for i in range(part.count)]
        run = DecomposedRun(part, LocalTransport(part, subs), dx, dx, ETA, courant=COURANT)
        run.set_state(state)
        for _ in range(3):
            run.step()
        torch.cuda.synchronize()
        ok = run.status == "ok"
        run.close()
        for sd in subs:
            sd.close()
        return 0 if ok else 1
    if args.profile_case == "snapshot":
        n = 2048
        state, dx = make_state(n)
        ctx = m.Context(n, n, dx, dx, ETA, courant=COURANT)
        ctx.set_state(state)
        ctx.step(0.0)
        buf = ctx.snapshot_pack(2, 50, 1e-3)
        st = ctx.synchronize_status()
        ctx.close()
        return 0 if st == 0 and buf.size > 0 else 1
    if args.profile_case == "batched":
        specs, ics = [], []
        for n, e, seed in m.problems.mixed_batch(64):
            fields, h = m.problems.random_instance(n, seed)
            specs.append(dict(nx=n, ny=n, dx=h, dy=h, eta=e))
            ics.append(fields)
        b = m.Batch(specs)
        for i, f in enumerate(ics):
            b.set_state(i, f)
        b.set_tuning(192, 0, 1, 32)  # what the autotuner picks for this batch
        for _ in range(2):
            b.step()
        worst, _ = b.synchronize_status()
        b.close()
        return 0 if worst == 0 else 1
    from magnetohydrodynamics_simulator_b200.autograd import state_from_potential

    n, nsteps = 1024, 10
    dx = 2 * np.pi / n
    rng = np.random.default_rng(5)
    X, Y = np.meshgrid(np.arange(n) * dx, np.arange(n) * dx)

    def modes(amp, shift):
        f = np.zeros((n, n))
        for _ in range(4):
            kx, ky = rng.integers(-4, 5, size=2)
            f += amp * rng.uniform(0.5, 1.0) * np.sin(kx * (X + shift) + ky * (Y + shift) + rng.uniform(0, 2 * np.pi))
        return torch.tensor(f, device="cuda")

    vx, vy, az = modes(0.05, dx / 2), modes(0.05, dx / 2), modes(0.1, 0.0)
    one = torch.ones(n, n, dtype=torch.float64, device="cuda")
    u0 = state_from_potential(az, one, vx, vy, one, dx, dx).contiguous()
    adj = m.Adjoint(n, n, dx, dx, 5e-3, 1e-3, nsteps, checkpoint_every=nsteps)
    uT, g0, gT = torch.empty_like(u0), torch.empty_like(u0), torch.randn_like(u0)
    ptr = lambda t: [t[k].data_ptr() for k in range(6)]  # noqa: E731
    torch.cuda.synchronize()
    adj.forward(ptr(u0), ptr(uT))
    adj.backward(ptr(gT), ptr(g0))
    torch.cuda.synchronize()
    adj.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=N_GRID)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-snapshot", action="store_true")
    ap.add_argument("--no-decomposed", action="store_true")
    ap.add_argument("--profile-case", choices=("batched", "adjoint", "snapshot", "decomposed", "step"), default=None,
                    help="run a small fixed case for a profiler and exit (no measurement)")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
