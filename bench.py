"""Benchmark: PhiX explicit FD time step on B200 (sm_100a).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--dtype f64|f32]

Workload (the configuration the metric is quoted on): 2-D Cahn-Hilliard
spinodal decomposition, 1024x1024 periodic, dx=1, f=c^2(1-c)^2, kappa=0.5,
M=1, dt=0.005, single-equation RK4 (M*lap(f'(c) - kappa*lap(c), bcs)),
c0 = 0.5 + U[-0.01, 0.01] (seed 1).

One bench "step" = one output interval: STEPS_PER_INTERVAL RK4 time steps of
the whole field, replayed from a CUDA graph (one launch per RK4 time step:
the four stages run in shared memory; --launch stage: one launch per stage).  L2 is flushed (256 MiB write) between timed steps, outside the timed
events.  `value` = cell-updates/s = cells x time steps / device time.
`e2e` runs the same interval through the C ABI with pinned HOST buffers
(phix_stepper_run_host: H2D, advance, D2H, synchronise) inside the timed
region.  Multi-GPU: independent replicas, one per rank (the single-field
configs do not shard; scaling "weak"), time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEPS_PER_INTERVAL = 100
METRIC = "CH 1024² cell-updates/s & HBM GB/s; surrogate vs FD sim-time/s at ≤2e-2 L2"
WORKLOAD = "CH 1024^2 periodic, single-equation RK4, dt=0.005 (spinodal decomposition)"
DATA = "synthetic: c0 = 0.5 + U[-0.01,0.01], numpy default_rng(1)"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.result = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.p:
            return
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            return
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if sm:
            self.result = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                           "samples": len(sm)}


def flush_l2(buf):
    buf.add_(1.0)


def reference_cpu_rate(fields, g, phys, prm, scheme, dt, nsteps):
    """Reference CPU path (oracle/_ref) on 1 host core: cell-updates/s."""
    from oracle.oracle import Grid, Reference
    ref = Reference()
    grid = Grid(n=tuple(g.n[a] for a in range(g.dim)), d=tuple(g.d[a] for a in range(g.dim)), ghost=g.ghost,
                bc=tuple(g.bc_type), bc_val=tuple(g.bc_val))
    work = [f.copy() for f in fields]
    t0 = time.perf_counter()
    ref.advance(work, phys, prm, scheme, dt, nsteps, grid, use_gpu=False)
    el = time.perf_counter() - t0
    cells = g.n[0] * g.n[1] * g.n[2]
    return cells * nsteps / el, el


def bench_ours(args):
    import torch
    import torch.distributed as dist

    import phix_b200 as px
    from phix_b200 import workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    g, phys, prm, scheme, dt, _, fields = workloads.ch2d(n=args.n)
    cells = g.n[0] * g.n[1] * g.n[2]
    prec = px.F64 if args.dtype == "f64" else px.F32
    w = 8 if prec == px.F64 else 4
    alg_bytes_step = 13 * w * cells  # RK4, one field: R u,W k1 | R u,k1 W k2 | R u,k2 W k3 | R u,k1,k2,k3 W u'

    st = px.Stepper(phys, scheme, prec, prm, dt, g)
    st.set_fusion(args.launch == "step")
    st.set_tiles(args.tiles)
    lps = st.launches_per_step
    d_in = torch.from_numpy(fields[0]).to(dev)
    st.load([d_in])
    st.set_graph(STEPS_PER_INTERVAL)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    for _ in range(args.warmup):
        st.advance(STEPS_PER_INTERVAL, stream)
        flush_l2(flush)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = px.launch_count()
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize(dev)
        for i in range(args.steps):
            starts[i].record(stream)
            st.advance(STEPS_PER_INTERVAL, stream)
            ends[i].record(stream)
            flush_l2(flush)
        torch.cuda.synchronize(dev)
    launches = px.launch_count() - launches0
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * cells * STEPS_PER_INTERVAL * args.steps / (total_ms / 1e3)

    # roofline: algorithmic bytes of one time step (13w per cell, the traffic
    # of one launch per stage) over the device time of one time step
    t_timestep = ms_per_step / 1e3 / STEPS_PER_INTERVAL
    achieved = alg_bytes_step / t_timestep / 1e9
    peak, peak_kind = _peaks()

    # e2e through the C ABI with pinned host buffers
    if args.no_e2e:
        st.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
                              "ms_per_step": ms_per_step, "roofline_achieved_gbs": achieved, "n": args.n,
                              "note": "profiling run (--no-e2e)"}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return None
    h_in = torch.from_numpy(fields[0]).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    for _ in range(2):
        st.run_host([h_in], [h_out], STEPS_PER_INTERVAL)
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_dev = torch.cuda.Event(enable_timing=True)
    e2e_dev2 = torch.cuda.Event(enable_timing=True)
    e2e_dev.record(stream)
    for _ in range(e2e_steps):
        st.run_host([h_in], [h_out], STEPS_PER_INTERVAL)
    e2e_dev2.record(stream)
    torch.cuda.synchronize(dev)
    e2e_wall = time.perf_counter() - t0
    e2e_ms = max(e2e_dev.elapsed_time(e2e_dev2), 1e3 * e2e_wall)
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * cells * STEPS_PER_INTERVAL * e2e_steps / (e2e_ms / 1e3)
    stored_bytes = fields[0].nbytes
    st.close()

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                n_cpu = args.cpu_baseline_steps
                rate, el = reference_cpu_rate(fields, g, phys, prm, scheme, dt, n_cpu)
                cpu = {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                       "sample": f"reference CPU path (computeRHSCPU + applyOnCPU, GPU stage semantics), "
                                 f"{n_cpu} RK4 steps of the same 1024^2 field, {el:.1f} s, 1 thread"}
            except Exception as e:  # oracle/_ref not built on this machine
                cpu = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "cell-updates/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": args.dtype,
            "data": DATA,
            "config": {"workload": WORKLOAD, "cells": cells, "time_steps_per_step": STEPS_PER_INTERVAL,
                       "launches_per_time_step": lps,
                       "precision_note": "FP64 stencils" if prec == px.F64 else "FP32 stencils, FP64 reductions",
                       "l2": "flushed between timed steps (256 MiB write); one step keeps its field L2-resident",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": f"algorithmic {13 * w} B/cell-update (13w RK4) over the CUDA-event time of "
                                 f"one time step ({lps} launch{'es' if lps > 1 else ''} per time step); "
                                 f"peak {peak_kind}"},
            "hbm_gbs_effective": achieved,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": stored_bytes,
                    "d2h_bytes_per_step": stored_bytes},
            "gpu_launches": launches,
            "clocks": clk.result,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def bench_reference(args):
    """Reference arm: the reference's own CPU implementation of the path
    (oracle/_ref, compiled from its sources), one host thread (it has no
    threading), each step a bounded sample of the same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle.oracle import LIB_REF
    if not os.path.exists(LIB_REF):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libphix_ref.so was not built"}))
        return None
    from phix_b200 import workloads
    g, phys, prm, scheme, dt, _, fields = workloads.ch2d()
    cells = g.n[0] * g.n[1] * g.n[2]
    sample = args.ref_sample_steps
    for _ in range(min(args.warmup, 1)):
        reference_cpu_rate(fields, g, phys, prm, scheme, dt, 1)
    times = []
    for _ in range(args.steps):
        rate, el = reference_cpu_rate(fields, g, phys, prm, scheme, dt, sample)
        times.append(el)
    total = sum(times)
    value = cells * sample * args.steps / total
    ref_cuda = None
    try:
        import torch
        if torch.cuda.is_available():
            from oracle.oracle import Grid, Reference
            ref = Reference()
            grid = Grid(n=(g.n[0], g.n[1]), d=(1.0, 1.0), ghost=1, bc=tuple(g.bc_type), bc_val=tuple(g.bc_val))
            work = [f.copy() for f in fields]
            ref.advance(work, phys, prm, scheme, dt, 20, grid, use_gpu=True)
            n = 500
            ms = ref.advance(work, phys, prm, scheme, dt, n, grid, use_gpu=True)
            ref_cuda = {"value": cells * n / (ms / 1e3), "unit": "cell-updates/s", "ms_per_time_step": ms / n,
                        "sample": f"reference GPU path (Solver::advance, RK4) built for sm_100a, {n} steps"}
    except Exception as e:
        ref_cuda = {"value": None, "sample": f"unavailable: {e}"}
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": DATA,
        "config": {"workload": WORKLOAD, "cells": cells, "time_steps_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"reference CPU path, {sample} RK4 steps of the 1024^2 field per step"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": ref_cuda,
    }
    print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dtype", choices=["f64", "f32"], default="f64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="device timing only (profiling runs)")
    ap.add_argument("--n", type=int, default=1024, help="grid size n x n (the metric is quoted at 1024)")
    ap.add_argument("--cpu-baseline-steps", type=int, default=50)
    ap.add_argument("--ref-sample-steps", type=int, default=2)
    ap.add_argument("--tiles", type=int, default=-1, help="2-D stage tile shape (phix_stepper_set_tiles)")
    ap.add_argument("--launch", choices=["step", "stage"], default="step",
                    help="one launch per RK4 time step (default) or one per stage")
    args = ap.parse_args()
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)  # timing rule: at least 3 untimed warm-up steps
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
