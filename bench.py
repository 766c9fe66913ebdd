#!/usr/bin/env python
"""Benchmark of the Euler hot path: 3-D 256^3 Taylor-Green SSP-RK3 member-steps/s.

Workload (config "TG-3D 256^3"): u = (sin x cos y cos z, -cos x sin y cos z, 0)
sampled at x_i = 2 pi i / N, N = 256 (padded M = 384), SmoothCutoff viscosity
eps = 0.05 (eps_N = 0.05/N, k0 = 2 pi sqrt(N)), SSP-RK3, C = 0.2.  A step is
one SSP-RK3 step (three right-hand sides) of every member of the batch.

  value   batched FP32-bulk member-steps/s, state resident in HBM, timed with
          CUDA events over K steps (max over ranks); every step reads inputs
          larger than L2 (126 MB), so no flush is needed.
  e2e     the same metric through the public API with host buffers: each
          step copies the batch's state host->device from pinned memory,
          steps it (Simulation.steps) and copies the new state back; three
          batched Simulations on their own streams take steps in turn, so
          copies overlap transforms.
  fp64_*  the plain FP64 form, one member, same workload.

``--impl reference`` times the CPU restatement of the reference's path (the
oracle; the reference itself cannot be built here) on the host cores.
Multi-GPU: replicas only (ensemble members are independent; weak scaling).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D 256^3 Euler member-steps/s, batched FP32 vs plain FP64 at L2<=1e-5; p99 latency"
UNIT = "member-steps/s"
VISC_CFG = {"type": "Smooth Cutoff", "eps": 0.05}
C_CFL = 0.2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="tg3d256",
                    choices=["tg3d256", "tg2d64", "tg3d-accuracy", "dsl-ensemble", "fbm512", "serving",
                             "dft-gemm-stage", "exchange", "dsl-classes"],
                    help="tg3d256 is the headline; the others are the remaining workloads, one JSON line each")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of Poisson arrivals")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: arrivals per second")
    ap.add_argument("--dry-run", action="store_true",
                    help="launch and rank bookkeeping only (gloo, no GPU): each rank reports in, rank 0 "
                         "prints how many ranks took part")
    ap.add_argument("--cpu-budget", type=float, default=150.0,
                    help="--impl reference: seconds of timed whole SSP-RK3 steps at most")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_key, table=None):
    """DRAM bytes per launch of a kernel from the committed ncu summary, or
    None; with `table`, that sub-table's entry for the kernel instead."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(table, {}).get(kernel_key) if table else d.get(kernel_key)
    except Exception:
        return None


class CpuStepper:
    """Whole SSP-RK3 steps of one member with the oracle (FP64, scipy.fft on
    `cores` threads): the CPU restatement of the reference's path.  The
    oracle evaluates a 3-D right-hand side whole (dudt) or slab by slab
    (dudt_slabs, the same arithmetic in a cache-friendlier order); the first
    right-hand side times both and the faster one is used, so the baseline is
    not held back by the evaluation order."""

    def __init__(self, n, cores):
        from oracle import euler_oracle as ora
        self.ora = ora
        ora.set_workers(cores)
        g = ora.Grid(3, n)
        self.eq = ora.IncompressibleEuler(g, ora.make_viscosity(VISC_CFG, g))
        self.ts = ora.SSP_RK3(self.eq)
        self.u = ora.initialize(ora.taylor_green_workload(3, n))
        t0 = time.perf_counter()
        self.eq.dudt(self.u)
        t1 = time.perf_counter()
        self.eq.dudt_slabs(self.u)
        t2 = time.perf_counter()
        self.eq.slabs = (t2 - t1) < (t1 - t0)
        self.form = "slab by slab" if self.eq.slabs else "whole arrays"
        self.cap = self.ora.math.inf if self.eq.visc() == 0 else \
            C_CFL * 2.0 / (self.eq.visc() * (self.ora.PI * n) ** 2)

    def step(self):
        """One timed SSP-RK3 step; returns its seconds."""
        t0 = time.perf_counter()
        self.ts.integrate(0.0, self.cap, C_CFL, self.u)
        return time.perf_counter() - t0


def cpu_sample(n, cores):
    """One whole SSP-RK3 step of one 3-D member with the oracle; returns
    (seconds, member-steps in the sample, stepper)."""
    st = CpuStepper(n, cores)
    return st.step(), 1.0, st


def run_reference(args, rank, world):
    """The reference arm: the oracle (the reference itself cannot be built
    here) on all host cores, whole SSP-RK3 steps of one 256^3 member.  The
    steps reported are the steps actually timed: at most --steps, and no
    more than fit in --cpu-budget seconds (at least one)."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    t_start = time.perf_counter()
    st = CpuStepper(args.n, cores)
    st.step()  # warm-up step (plans, page faults); one is enough on the CPU
    samples = []
    while len(samples) < max(1, args.steps):
        samples.append(st.step())
        if sum(samples) + statistics.mean(samples) > args.cpu_budget:
            break
    per_member_step = statistics.mean(samples)
    value = 1.0 / per_member_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": len(samples), "warmup": 1, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": per_member_step * 1e3, "timed_s": sum(samples),
        "run_s": time.perf_counter() - t_start,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"TG-3D {args.n}^3, M={3 * args.n // 2}, SmoothCutoff eps=0.05, SSP-RK3, C=0.2",
                   "members": 1, "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{len(samples)} whole SSP-RK3 steps (3 right-hand sides each) of one "
                                   f"{args.n}^3 member, FP64 numpy/scipy.fft restatement of the reference CPU "
                                   f"path ({st.form}), after one warm-up step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    import azeban_b200 as az
    from azeban_b200 import _lib
    from azeban_b200 import init as azinit

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from azeban_b200 import replicas

    barrier = replicas.barrier

    def max_over_ranks(x):
        return replicas.max_over_ranks(x)

    N, B, K, W = args.n, args.batch, args.steps, args.warmup
    g = az.Grid(3, N)
    visc = az.make_viscosity(VISC_CFG, g)
    stream = torch.cuda.current_stream()

    # ---- FP32-bulk batched form (the headline) ---------------------------
    u0_32 = azinit.taylor_green(3, N, "f32")
    batch_u = u0_32.unsqueeze(0).repeat(B, 1, 1, 1, 1).contiguous()
    eq32 = az.IncompressibleEuler(g, visc, "f32", batch=B)
    ts32 = az.SSP_RK3(eq32)
    sim32 = az.Simulation(g, C_CFL, ts32, batch_u)
    sim32.steps(W)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    evs[0].record(stream)
    for i in range(K):
        sim32.steps(1)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(K)]
    total_ms = max_over_ranks(evs[0].elapsed_time(evs[K]))
    value = replicas.aggregate_rate(B * K, world, total_ms)
    ms_per_step = total_ms / K
    sorted_ms = sorted(step_ms)
    p50 = sorted_ms[len(sorted_ms) // 2]
    p99 = sorted_ms[min(len(sorted_ms) - 1, math.ceil(0.99 * len(sorted_ms)) - 1)]

    # ---- live per-pass roofline over K more steps --------------------------
    _lib.lib.az_profile_enable(1)
    sim32.steps(K)
    torch.cuda.synchronize()
    _lib.lib.az_profile_enable(0)
    import ctypes as ct
    ms = (ct.c_double * 5)()
    by = (ct.c_double * 5)()
    nl = (ct.c_longlong * 5)()
    _lib.check(_lib.lib.az_profile_read(ms, by, nl, 5))
    pass_names = ["inv_x_pad", "inv_y_pad", "z_product", "fwd_y_trunc", "fwd_x_epilogue"]
    # The product pass kernel: k_zfused (bit 2 of its tuned variant), k_zpass (bit 1) or k_rows_product.
    zv = ct.c_int()
    _lib.check(_lib.lib.az_tune_get(1, g.N_phys_pad, 1, ct.byref(zv)))
    product_kernel = "k_zfused" if zv.value & 4 else "k_zpass" if zv.value & 2 else "k_rows_product"
    kernel_keys = ["k_cols_pad_inv_x", "k_cols_pad_inv_y", product_kernel,
                   "k_cols_trunc_fwd", "k_fwd_epilogue"]
    peak, peak_kind = measured_peak_hbm()
    passes = {}
    for i, nm in enumerate(pass_names):
        if nl[i]:
            avg_ms = ms[i] / nl[i]
            passes[nm] = {"launches": nl[i], "avg_ms": avg_ms, "bytes_per_launch": by[i] / nl[i],
                          "gbs": by[i] / nl[i] / (avg_ms * 1e-3) / 1e9,
                          "share": ms[i] / max(sum(ms), 1e-30)}
    dom = max(range(5), key=lambda i: ms[i])
    dom_bytes = by[dom] / max(nl[dom], 1)
    dom_ms = ms[dom] / max(nl[dom], 1)
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = ncu_traffic(kernel_keys[dom])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": pass_names[dom],
                "shared_pipe_pct": ncu_traffic(kernel_keys[dom], "_shared_pipe_pct"),
                "peak_source": peak_kind, "passes": passes,
                "step_bytes_model_gb": sum(by) / K / 1e9,
                "step_gbs_model": sum(by) / K / (ms_per_step * 1e-3) / 1e9}

    # ---- plain FP64 form, one member ----------------------------------------
    fp64 = None
    if not args.no_fp64:
        u0_64 = azinit.taylor_green(3, N, "f64")
        eq64 = az.IncompressibleEuler(g, visc, "f64")
        sim64 = az.Simulation(g, C_CFL, az.SSP_RK3(eq64), u0_64)
        sim64.steps(W)
        K64 = max(3, K // 2)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim64.steps(K64)
        e1.record(stream)
        torch.cuda.synchronize()
        t64 = max_over_ranks(e0.elapsed_time(e1))
        fp64 = {"member_steps_per_s": world * K64 / (t64 / 1e3), "ms_per_step": t64 / K64, "steps": K64}
        del sim64, eq64

    # ---- accuracy: FP32 bulk vs FP64 (one member) ---------------------------
    # Times are in azeban units (domain [0,1)^3, k = 2 pi n): t = 1/(2 pi) is
    # t = 1 of the same arrays read on [0,2 pi)^3.  "floor" is FP64 started
    # from the FP32-rounded initial state: how far rounding the initial data
    # alone drifts by then (the flow's own sensitivity).
    accuracy = None
    if not args.no_accuracy:
        def l2(a, b):
            return float(torch.linalg.vector_norm(a.to(torch.complex128) - b) / torch.linalg.vector_norm(b))

        u64 = azinit.taylor_green(3, N, "f64")
        u32 = azinit.taylor_green(3, N, "f32")
        sims = {
            "fp32": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, visc, "f32")), u32),
            "fp64": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, visc, "f64")), u64),
            "fp64_rounded_init": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, visc, "f64")),
                                               u32.to(torch.complex128).contiguous()),
        }
        accuracy = {}
        for t in (1.0 / (2 * math.pi), 1.0):
            for s_ in sims.values():
                s_.simulate_until(t)
            ref = sims["fp64"].u()
            accuracy[f"t={t:.6g}"] = {
                "l2_rel_fp32_vs_fp64": l2(sims["fp32"].u(), ref),
                "l2_rel_floor_fp64_rounded_init": l2(sims["fp64_rounded_init"].u(), ref),
                "steps_fp32": sims["fp32"].state()[1][0], "steps_fp64": sims["fp64"].state()[1][0]}
        del sims

    # ---- end to end through the public API with host buffers ---------------
    # A step is the host->device copy of the batch's state from pinned memory,
    # one SSP-RK3 step of the batch (Simulation.steps, no host sync) and the
    # device->host copy of the new state.  NBUF batched Simulations take steps
    # in turn: their steps run in order on one compute stream (no two steps
    # share the SMs), while a copy-in stream fills the next batch's state and
    # a copy-out stream drains the previous one, chained by events.  The host
    # link bounds it: 0.81 GB each way per step of 4 members take 16.2 ms
    # when both directions run at once and 18.1-18.8 ms per step pipelined
    # without any transform (measured for 2 to 6 buffers), against 17.4 ms
    # of transforms; with both, 19.9-20.4 ms per step.  Three buffers: a
    # batch's copy-in waits for its own previous copy-out.
    e2e = None
    if not args.no_e2e:
        NBUF = 3
        host_in = batch_u.cpu().pin_memory()
        host_out = [torch.empty_like(host_in).pin_memory() for _ in range(NBUF)]
        s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        esims = [az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, visc, "f32", B)), batch_u)
                 for _ in range(NBUF)]
        out_done = [None] * NBUF
        torch.cuda.synchronize()

        def e2e_steps(n, start_evt=None):
            if start_evt is not None:
                for sb in (s_in, s_comp, s_out):
                    sb.wait_event(start_evt)
            for k in range(n):
                j = k % NBUF
                u_dev = esims[j].u()
                if out_done[j] is not None:
                    s_in.wait_event(out_done[j])
                with torch.cuda.stream(s_in):
                    u_dev.copy_(host_in, non_blocking=True)
                in_done = torch.cuda.Event()
                in_done.record(s_in)
                s_comp.wait_event(in_done)
                esims[j].steps(1, stream=s_comp)
                comp_done = torch.cuda.Event()
                comp_done.record(s_comp)
                s_out.wait_event(comp_done)
                with torch.cuda.stream(s_out):
                    host_out[j].copy_(u_dev, non_blocking=True)
                out_done[j] = torch.cuda.Event()
                out_done[j].record(s_out)
            for sb in (s_in, s_comp, s_out):
                ev = torch.cuda.Event()
                ev.record(sb)
                stream.wait_event(ev)

        e2e_steps(max(NBUF, W))
        torch.cuda.synchronize()
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        e2e_steps(K, a0)
        a1.record(stream)
        torch.cuda.synchronize()
        te = max_over_ranks(a0.elapsed_time(a1))
        nbytes = host_in.numel() * host_in.element_size()
        e2e = {"value": world * B * K / (te / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes,
               "form": f"{NBUF} batched Simulations ({B} members each) taking steps in turn on one compute stream, "
                       "copies in and out on two copy streams"}
        del esims

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        sec, msteps, cst = cpu_sample(N, cores)
        cpu = {"value": msteps / sec, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"one whole SSP-RK3 step of one {N}^3 member, FP64 numpy/scipy.fft restatement of "
                         f"the reference CPU path ({cst.form}), {sec:.1f} s"}

    launches_per_step = 1 + 3 * 5 + 1 + 1
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"TG-3D {N}^3 batched FP32 bulk, M={3 * N // 2}, SmoothCutoff eps=0.05, "
                                   f"SSP-RK3, C=0.2", "members_per_gpu": B, "N": N, "M": 3 * N // 2,
                       "precision": "fp32 bulk, fp64 CFL", "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}"},
            "p50_step_ms": p50, "p99_step_ms": p99,
            "fp64": fp64,
            "fp32_over_fp64": (value / world) / fp64["member_steps_per_s"] * world if fp64 else None,
            # The same precision on both sides: the plain FP64 GPU form against
            # the FP64 CPU restatement, one member each.
            "like_for_like_fp64": ({"gpu_member_steps_per_s": fp64["member_steps_per_s"] / world,
                                    "cpu_member_steps_per_s": cpu["value"],
                                    "gpu_over_cpu": fp64["member_steps_per_s"] / world / cpu["value"]}
                                   if fp64 and cpu else None),
            "accuracy": accuracy,
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches_per_step * K,
        }
        if fp64:
            line["fp32_over_fp64"] = (value / world) / (fp64["member_steps_per_s"] / world)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _ev():
    import torch
    return torch.cuda.Event(enable_timing=True)


def run_tg2d64(args):
    """Taylor-Green 2-D 64^2 FP64 to t = 1 (the reference's CPU-runnable
    configuration): GPU time to solution, the oracle's time on the host cores,
    and their agreement."""
    import torch

    import azeban_b200 as az
    from azeban_b200 import init as azinit
    from oracle import euler_oracle as ora
    g = az.Grid(2, 64)
    sim = az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, az.make_viscosity(VISC_CFG, g))),
                        azinit.taylor_green(2, 64, "f64"))
    torch.cuda.synchronize()
    e0, e1 = _ev(), _ev()
    e0.record()
    sim.simulate_until(1.0)
    e1.record()
    torch.cuda.synchronize()
    gpu_ms = e0.elapsed_time(e1)
    og = ora.Grid(2, 64)
    ora.set_workers(os.cpu_count() or 1)
    t0 = time.perf_counter()
    osim = ora.Simulation(og, C_CFL, ora.SSP_RK3(ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFG, og))),
                          ora.initialize(ora.taylor_green_workload(2, 64)))
    osim.simulate_until(1.0)
    cpu_s = time.perf_counter() - t0
    steps = sim.state()[1][0]
    print(json.dumps({"workload": "TG-2D 64^2 FP64 to t=1", "steps": steps, "oracle_steps": len(osim.dts),
                      "gpu_ms_to_solution": gpu_ms, "cpu_oracle_s_to_solution": cpu_s,
                      "cpu_cores": os.cpu_count(),
                      "l2_rel_gpu_vs_oracle": ora.rel_l2(sim.u().cpu().numpy(), osim.u_)}), flush=True)


def _until_rounding_state(sim, group, t):
    """simulate_until(t) of a one-member FP64 simulation, with its state
    rounded to FP32 after every step (the rounding any FP32 state storage
    injects once per step)."""
    import torch
    group.set_end(t)
    while sim.state()[0][0] < t:
        group.steps(1)
        u = sim.u()
        u.copy_(u.to(torch.complex64).to(torch.complex128))


def run_tg3d_accuracy(args):
    """Taylor-Green 3-D at 128^3 and 256^3, FP64 and FP32 bulk: relative L2 of
    FP32 vs FP64 at 10 output times over [0, 1/(2 pi)] (t in [0, 1] on
    [0, 2 pi)^3) and at azeban t = 1, beside two floors: FP64 started from
    the FP32-rounded initial state (the flow's sensitivity to one rounding at
    t = 0), and FP64 with its state rounded to FP32 after every step (the
    rounding a FP32 state stores into every step, without any FP32
    arithmetic)."""
    import torch

    import azeban_b200 as az
    from azeban_b200 import init as azinit
    out = []
    for N in (128, 256):
        g = az.Grid(3, N)
        v = az.make_viscosity(VISC_CFG, g)
        u64 = azinit.taylor_green(3, N, "f64")
        u32 = azinit.taylor_green(3, N, "f32")
        sims = {"fp32": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f32")), u32),
                "fp64": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f64")), u64),
                "floor": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f64")),
                                       u32.to(torch.complex128).contiguous()),
                "storage": az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f64")),
                                         u32.to(torch.complex128).contiguous())}
        storage_group = az.Group([sims["storage"]])
        times = [(i + 1) / (10 * 2 * math.pi) for i in range(10)] + [1.0]
        rows = []
        busy_ms = {"fp32": 0.0, "fp64": 0.0}
        for t in times:
            for name, s_ in sims.items():
                e0, e1 = _ev(), _ev()
                e0.record()
                if name == "storage":
                    _until_rounding_state(s_, storage_group, t)
                else:
                    s_.simulate_until(t)
                e1.record()
                torch.cuda.synchronize()
                if name in busy_ms:
                    busy_ms[name] += e0.elapsed_time(e1)
            ref = sims["fp64"].u()
            nrm = torch.linalg.vector_norm(ref)
            rows.append({"t": t, "l2_fp32_vs_fp64": float(torch.linalg.vector_norm(sims["fp32"].u().to(torch.complex128) - ref) / nrm),
                         "floor": float(torch.linalg.vector_norm(sims["floor"].u() - ref) / nrm),
                         "floor_state_rounded_each_step": float(torch.linalg.vector_norm(sims["storage"].u() - ref) / nrm)})
        # one member each, stepped to t = 1 (azeban units) through simulate_until
        rate = {}
        for name, ms in busy_ms.items():
            steps = sims[name].state()[1][0]
            rate[name] = {"steps": steps, "ms_per_step": ms / steps, "member_steps_per_s": steps / (ms / 1e3)}
        out.append({"N": N, "outputs": rows, "throughput_one_member": rate})
        del sims, storage_group
    print(json.dumps({"workload": "TG-3D accuracy FP32 bulk vs FP64", "results": out}), flush=True)


def run_dsl_classes(args):
    """Each class of the DSL-2D ensemble alone (FP32 bulk, at its ensemble
    batch size): 20 timed Simulation.steps(1) calls after 3 warm-up steps, and
    the per-pass times from the library's per-pass CUDA events.  Model bytes
    per member-step (fused axis-pass model, 2-D): 22 N Nh + 30 M Nh complex
    elements."""
    import ctypes as ct

    import numpy as np
    import torch

    import azeban_b200 as az
    from azeban_b200 import _lib
    from azeban_b200 import init as azinit
    rng = np.random.default_rng(2024)
    rows = []
    for N, B in [(128, 256), (256, 192), (512, 64)]:
        g = az.Grid(2, N)
        M, Nh = g.N_phys_pad, N // 2 + 1
        eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFG, g), "f32", batch=B)
        u0 = azinit.double_shear_layer(N, math.pi / 15, 0.05, rng.uniform(0, 2 * math.pi, B), "f32")
        sim = az.Simulation(g, C_CFL, az.SSP_RK3(eq), u0)
        sim.steps(3)
        torch.cuda.synchronize()
        e0, e1 = _ev(), _ev()
        e0.record()
        for _ in range(20):
            sim.steps(1)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 20
        _lib.check(_lib.lib.az_profile_enable(1))
        sim.steps(5)
        torch.cuda.synchronize()
        _lib.check(_lib.lib.az_profile_enable(0))
        t = (ct.c_double * 5)()
        by = (ct.c_double * 5)()
        nl = (ct.c_longlong * 5)()
        _lib.check(_lib.lib.az_profile_read(t, by, nl, 5))
        model = (22 * N * Nh + 30 * M * Nh) * 8.0
        passes = {}
        for i, name in ((0, "inv_x_pad"), (2, "product"), (4, "epilogue")):
            if nl[i]:
                passes[name] = {"us": 1e3 * t[i] / nl[i], "gbs": by[i] / nl[i] / (t[i] / nl[i] * 1e6)}
        rows.append({"N": N, "batch": B, "ms_per_step": ms, "member_steps_per_s": B / (ms / 1e3),
                     "model_gbs": B * model / (ms / 1e3) / 1e9, "passes": passes})
        del sim, eq
    print(json.dumps({"workload": "DSL-2D classes each alone, FP32 bulk, ensemble batch sizes", "results": rows}),
          flush=True)


def run_dsl_ensemble(args):
    """2-D double-shear-layer ensemble, 512 members of mixed resolution in one
    group (128^2 x256, 256^2 x192, 512^2 x64; each step a captured graph per
    unfinished class, the classes on concurrent streams), FP32 bulk, phases
    phi ~ U[0, 2 pi) from a seed, to t = 1/(2 pi) (t = 1 on [0, 2 pi)^2)."""
    import numpy as np
    import torch

    import azeban_b200 as az
    from azeban_b200 import init as azinit
    classes = [(128, 256), (256, 192), (512, 64)]
    rng = np.random.default_rng(2024)
    sims, keep, first = [], [], {}
    for N, B in classes:
        g = az.Grid(2, N)
        eq = az.IncompressibleEuler(g, az.make_viscosity(VISC_CFG, g), "f32", batch=B)
        ts = az.SSP_RK3(eq)
        phases = rng.uniform(0, 2 * math.pi, B)
        u0 = azinit.double_shear_layer(N, math.pi / 15, 0.05, phases, "f32")
        sims.append(az.Simulation(g, C_CFL, ts, u0))
        keep += [eq, ts]
        first[N] = (phases[0], u0[0].clone())
    group = az.Group(sims)
    t_end = 1.0 / (2 * math.pi)
    torch.cuda.synchronize()
    e0, e1 = _ev(), _ev()
    e0.record()
    group.simulate_until(t_end)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    msteps = sum(sum(s.state()[1]) for s in sims)
    errs = {}
    for (N, B), sim in zip(classes, sims):
        g = az.Grid(2, N)
        ph, _ = first[N]
        u64 = azinit.double_shear_layer(N, math.pi / 15, 0.05, [ph], "f64")[0]
        ref = az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, az.make_viscosity(VISC_CFG, g), "f64")), u64)
        ref.simulate_until(t_end)
        r = ref.u()
        errs[f"{N}^2"] = float(torch.linalg.vector_norm(sim.u()[0].to(torch.complex128) - r) / torch.linalg.vector_norm(r))
    print(json.dumps({"workload": "DSL-2D ensemble 512 members (128^2 x256, 256^2 x192, 512^2 x64) FP32, one group, a graph per unfinished class per step",
                      "t_end": t_end, "wall_ms": ms, "member_steps": msteps,
                      "member_steps_per_s": msteps / (ms / 1e3), "l2_member0_vs_fp64": errs}), flush=True)


def run_fbm512(args):
    """3-D 512^3 (768^3 padded) fractional Brownian field, H = 0.75, FP32 bulk,
    50 steps: per-pass HBM GB/s, and the error vs an FP64 run of the same
    initial state at 512^3 and vs FP64 at 256^3 from the truncated state."""
    import ctypes as ct

    import torch

    import azeban_b200 as az
    from azeban_b200 import _lib
    from azeban_b200 import init as azinit
    N, steps = 512, 50
    g = az.Grid(3, N)
    v = az.make_viscosity(VISC_CFG, g)
    u64 = azinit.fractional_brownian(3, N, 0.75, seed=7, precision="f64")
    u32 = u64.to(torch.complex64).contiguous()
    sim = az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f32")), u32)
    torch.cuda.synchronize()
    _lib.lib.az_profile_enable(1)
    e0, e1 = _ev(), _ev()
    e0.record()
    sim.steps(steps)
    e1.record()
    torch.cuda.synchronize()
    _lib.lib.az_profile_enable(0)
    ms = (ct.c_double * 5)()
    by = (ct.c_double * 5)()
    nl = (ct.c_longlong * 5)()
    _lib.check(_lib.lib.az_profile_read(ms, by, nl, 5))
    names = ["inv_x_pad", "inv_y_pad", "z_product", "fwd_y_trunc", "fwd_x_epilogue"]
    passes = {n: {"avg_ms": ms[i] / nl[i], "gbs": by[i] / nl[i] / (ms[i] / nl[i] * 1e-3) / 1e9}
              for i, n in enumerate(names) if nl[i]}
    t_reached = sim.state()[0][0]
    u_fp32 = sim.u().clone()
    del sim
    ref = az.Simulation(g, C_CFL, az.SSP_RK3(az.IncompressibleEuler(g, v, "f64")), u64)
    ref.simulate_until(t_reached)
    r = ref.u()
    err512 = float(torch.linalg.vector_norm(u_fp32.to(torch.complex128) - r) / torch.linalg.vector_norm(r))
    del ref, r
    # FP64 at 256^3 from the truncated initial state, compared on the retained modes
    Nc = 256
    idx = torch.cat([torch.arange(0, Nc // 2 + 1), torch.arange(N - Nc // 2 + 1, N)]).cuda()
    def trunc(a):
        return a.index_select(1, idx).index_select(2, idx)[..., : Nc // 2 + 1] * (Nc / N) ** 3
    gc = az.Grid(3, Nc)
    refc = az.Simulation(gc, C_CFL, az.SSP_RK3(az.IncompressibleEuler(gc, az.make_viscosity(VISC_CFG, gc), "f64")),
                         trunc(u64).contiguous())
    refc.simulate_until(t_reached)
    rc = refc.u()
    err256 = float(torch.linalg.vector_norm(trunc(u_fp32.to(torch.complex128)) - rc) / torch.linalg.vector_norm(rc))
    print(json.dumps({"workload": "fBm-3D 512^3 FP32 bulk, 50 steps", "ms_per_step": e0.elapsed_time(e1) / steps,
                      "member_steps_per_s": steps / (e0.elapsed_time(e1) / 1e3), "t_reached": t_reached,
                      "passes": passes, "l2_vs_fp64_512": err512, "l2_vs_fp64_256_truncated": err256}), flush=True)


def run_serving(args):
    """Poisson arrivals (default 200/s for 60 s) of 2-D double-shear-layer and
    3-D fBm solves, N from {64^2..512^2} and {64^3..256^3} with probability
    proportional to 1/cost, t_end ~ U[0.25, 1]; continuous batching with slots
    sized from an HBM budget.  Beside it, the FP64 one-at-a-time baseline:
    each class's FP64 solve time measured alone, and the same arrivals served
    first-in first-out one at a time with those service times."""
    import numpy as np
    import torch

    import azeban_b200 as az
    from azeban_b200 import serving
    reqs = serving.poisson_stream(args.rate, args.duration, seed=11)
    free, _ = torch.cuda.mem_get_info()
    weights = {c: 1.0 for c in serving.CLASSES}
    for c in [(2, 64), (2, 128)]:
        weights[c] = 4.0
    caps = serving.plan_capacities(int(free * 0.5), "f32", weights)
    caps = {c: min(k, 256) for c, k in caps.items()}
    loop = serving.ServingLoop(caps, "f32")
    records, stats, _ = loop.run(reqs)
    # FP64 one at a time: per-class solve time at the mean t_end, measured alone
    per_class = {}
    for c in serving.CLASSES:
        sub = [r for r in reqs if (r.dim, r.N) == c]
        if not sub:
            continue
        r0 = sub[0]
        g = az.Grid(c[0], c[1])
        u0 = serving.initial_state(r0, "f64")
        sim = az.Simulation(g, 0.2, az.SSP_RK3(az.IncompressibleEuler(g, az.make_viscosity(serving.VISC, g), "f64")), u0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.simulate_until(r0.t_end)
        torch.cuda.synchronize()
        per_class[c] = (time.perf_counter() - t0) / r0.t_end
    clock, lat, busy = 0.0, [], 0.0
    for r in sorted(reqs):
        svc = per_class[(r.dim, r.N)] * r.t_end
        clock = max(clock, r.arrival) + svc
        busy += svc
        lat.append(clock - r.arrival)
    base = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "makespan_s": clock, "busy_s": busy}
    print(json.dumps({"workload": f"serving Poisson {args.rate}/s for {args.duration}s, FP32 bulk continuous batching",
                      "capacities": {f"{d}D-{n}": k for (d, n), k in caps.items()}, "stats": stats,
                      "fp64_one_at_a_time": base,
                      "fp64_class_seconds_per_unit_time": {f"{d}D-{n}": v for (d, n), v in per_class.items()}}),
          flush=True)


def run_dft_gemm_stage(args):
    """One radix-16 DFT stage of FP32 columns in shared memory: the transform
    passes' butterflies against a DFT-as-GEMM stage on the tensor pipe
    (mma.sync m16n8k8 TF32, three-term head/tail split), time per column and
    stage on every SM and the error of one stage."""
    import ctypes as ct

    import torch

    from azeban_b200 import _lib
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    res = {}
    for name, method in (("butterfly", 0), ("gemm_3xtf32", 1)):
        ns, err = ct.c_double(), ct.c_double()
        _lib.check(_lib.lib.az_bench_radix16_stage(method, 8 * sms, ct.byref(ns), ct.byref(err)))
        res[name] = {"ns_per_column_stage": ns.value, "max_rel_err": err.value}
    res["gemm_over_butterfly_time"] = res["gemm_3xtf32"]["ns_per_column_stage"] / res["butterfly"]["ns_per_column_stage"]
    print(json.dumps({"workload": "radix-16 DFT stage, FP32 complex columns in shared memory, "
                                  f"{8 * sms} CTAs of 128 columns", "results": res}), flush=True)


def run_exchange(args):
    """The 384-point FP32 transform of the wide plan (radix 16, exchange,
    radix 24) on every SM, with the exchange through shared memory (the
    transform passes' way) or as a lane transpose with warp shuffles: time per
    column transform and the error of one transform."""
    import ctypes as ct

    import torch

    from azeban_b200 import _lib
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    res = {}
    for name, method in (("shared_memory", 0), ("warp_shuffle", 1), ("warp_shuffle_uncapped", 2)):
        ns, err = ct.c_double(), ct.c_double()
        _lib.check(_lib.lib.az_bench_exchange384(method, 16 * sms, ct.byref(ns), ct.byref(err)))
        res[name] = {"ns_per_column": ns.value, "max_rel_err": err.value}
    res["shuffle_over_shared_time"] = res["warp_shuffle"]["ns_per_column"] / res["shared_memory"]["ns_per_column"]
    print(json.dumps({"workload": "384-point FP32 transform (16 x 24), exchange through shared memory vs warp "
                                  f"shuffles, {16 * sms} CTAs of 32 columns", "results": res}), flush=True)


def launch_ranks(args):
    """--gpus N without a launcher: re-run this command under
    torch.distributed.run with N ranks on this node (one per GPU, rendezvous
    on 127.0.0.1) and return its exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def run_dry(args, rank, world):
    """Rank bookkeeping without a GPU: gloo ranks report in; rank 0 prints the
    number that took part and the max over ranks of a per-rank value."""
    import datetime

    import torch.distributed as dist

    from azeban_b200 import replicas
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    seen = int(replicas.sum_over_ranks(1.0, device="cpu"))
    slowest = replicas.max_over_ranks(float(rank + 1), device="cpu")
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "ranks_seen": seen, "max_over_ranks": slowest,
                          "members": replicas.partition_by_cost([1.0] * (4 * world), world)}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    rank, world, local = dist_env()
    if args.dry_run:
        run_dry(args, rank, world)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    extra = {"tg2d64": run_tg2d64, "tg3d-accuracy": run_tg3d_accuracy, "dsl-ensemble": run_dsl_ensemble,
             "fbm512": run_fbm512, "serving": run_serving, "dft-gemm-stage": run_dft_gemm_stage,
             "exchange": run_exchange, "dsl-classes": run_dsl_classes}
    if args.workload in extra:
        import torch
        torch.cuda.set_device(local)
        if rank == 0:
            extra[args.workload](args)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
