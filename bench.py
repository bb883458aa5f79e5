"""Benchmark: PhiX explicit FD time step on B200 (sm_100a).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--dtype f64|f32]

Workload (the configuration the metric is quoted on): 2-D Cahn-Hilliard
spinodal decomposition, 1024x1024 periodic, dx=1, f=c^2(1-c)^2, kappa=0.5,
M=1, dt=0.005, single-equation RK4 (M*lap(f'(c) - kappa*lap(c), bcs)),
c0 = 0.5 + U[-0.01, 0.01] (seed 1).

One bench "step" = one output interval: STEPS_PER_INTERVAL RK4 time steps of
the whole field, replayed from a CUDA graph (the library's default launch
shape: one launch per RK4 time step in FP64 and FP32; --launch overrides it).  --workload selects the other configurations (ac2d, chac3d,
batch, and ch2d_ms: the CH application's multi-step form), reported with
the same keys.  L2 is flushed (256 MiB write) between timed steps, outside the timed
events.  `value` = cell-updates/s = cells x time steps / device time.
`e2e` runs the same interval through the C ABI with pinned HOST buffers
(phix_stepper_run_host: H2D, advance, D2H, synchronise) inside the timed
region.  Multi-GPU: independent replicas, one per rank (the single-field
configs do not shard; scaling "weak"), time = max over ranks.  `--gpus N`
without a launcher starts N ranks itself (torchrun on 127.0.0.1).
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
    from phix_b200 import MULTISTEP  # a constant: the CUDA library is not loaded
    if scheme == MULTISTEP:  # c and mu
        ref.advance_ch_multistep(work[0], work[1], prm, dt, nsteps, grid, use_gpu=False)
    else:
        ref.advance(work, phys, prm, scheme, dt, nsteps, grid, use_gpu=False)
    el = time.perf_counter() - t0
    cells = g.n[0] * g.n[1] * g.n[2]
    return cells * nsteps / el, el


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def openmp_cpu_rate(fields, g, phys, prm, scheme, dt, min_seconds=3.0, max_steps=1000):
    """The oracle's restatement of the same discretisation built with OpenMP
    (oracle/liboracle_omp.so) on all host threads, in the device build's
    rounding pattern (fma_mode 1): time steps are run in growing chunks until
    `min_seconds` of wall time.  Returns (cell-updates/s, seconds, steps,
    threads)."""
    from oracle.oracle import LIB_ORACLE_OMP, Grid, Oracle
    from phix_b200 import MULTISTEP
    omp = Oracle(LIB_ORACLE_OMP)
    grid = Grid(n=tuple(g.n[a] for a in range(g.dim)), d=tuple(g.d[a] for a in range(g.dim)), ghost=g.ghost,
                bc=tuple(g.bc_type), bc_val=tuple(g.bc_val), fma_mode=1)
    work = [f.copy() for f in fields]
    cells = g.n[0] * g.n[1] * g.n[2] * (1 if scheme == MULTISTEP else len(fields))
    done, el, chunk = 0, 0.0, 1
    while el < min_seconds and done < max_steps:
        t0 = time.perf_counter()
        if scheme == MULTISTEP:
            omp.advance_ch_multistep(work[0], work[1], prm, dt, chunk, grid)
        else:
            omp.advance(work, phys, prm, scheme, dt, chunk, grid)
        el += time.perf_counter() - t0
        done += chunk
        chunk = min(2 * chunk, max_steps - done) or 1
    return cells * done / el, el, done, omp.threads()


# ---------------------------------------------------------------------------
# workloads: each runner advances its whole field(s) by `K` time steps per
# bench step and knows its algorithmic bytes and its end-to-end path
# ---------------------------------------------------------------------------
WORKLOADS = {
    "ch2d": ("CH 1024^2 periodic, single-equation RK4, dt=0.005 (spinodal decomposition)",
             "synthetic: c0 = 0.5 + U[-0.01,0.01], numpy default_rng(1)"),
    "ch2d_ms": ("CH 1024^2 periodic, multi-step Euler (mu STEADY, c TRANSIENT: the CH application's form), dt=0.005",
                "synthetic: c0 = 0.5 + U[-0.01,0.01], numpy default_rng(1); mu0 = 0"),
    "ac2d": ("AC 128^2 periodic, Euler, dt=0.01, L=kappa=1 (quickstart form)",
             "synthetic: phi0 = U[-0.05,0.05], numpy default_rng(0)"),
    "chac3d": ("CH+AC 3-D 256^3, zero-flux x, periodic y/z, coupled RK4, dt=0.002",
               "synthetic: c0 = 0.4 + U[-0.01,0.01], eta0 = U[0,0.1], numpy default_rng(2)"),
    "batch": ("64 batched 2-D CH instances, n in {128..1024}, kappa, M per instance, RK4, dt=0.005",
              "synthetic: per-instance size/kappa/M/mean from numpy default_rng(3)"),
}

# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu
# capture of each (cold L2, so an upper bound for the graph-replayed
# launches); keyed by (workload, dtype, kernel).
TRAFFIC = {
    ("ch2d", "f64", "step_pair"): 8.46e6,   # CH 1024^2 RK4, one launch per step
    ("ch2d", "f32", "step_pair"): 8.46e6,
    ("ch2d", "f64", "stage_box"): 12.63e6,  # mean of the stage-1 and stage-2 launches
    ("ch2d", "f32", "step_box"): 8.47e6,
    ("batch", "f32", "step_pair_batched"): 358.3e6,  # 64 instances, one launch per step
    ("ch2d_ms", "f64", "step_pair_ms"): 8.45e6,  # CH 1024^2 multi-step Euler
    # CH+AC 256^3 RK4, one launch per stage: mean over the four launches of a time step
    ("chac3d", "f32", "stage_stream3d"): 510.0e6,
    ("chac3d", "f64", "stage_stream3d"): 914.0e6,
}

# Lane operations (fma = 2) of one RK4 cell-update in step2d_pair.cuh, on the
# tile's own cells: per stage the mu pass (Laplacian 8, f' 7, mu 4 = 19) and
# the k pass (Laplacian 8, k 2, y 2, RK4 sum 0 / 2 / 2; final: sum 1, update 2):
# 4 x 19 + 12 + 14 + 14 + 13 = 129.  FP32's final pass forms dt/6 * sum (1)
# and the compensated two-sum update (10 add/sub) in place of the fma (2).
PAIR_FLOPS_F64 = 129
PAIR_FLOPS_F32 = 138

# step tiles 6 and up are the pair kernels (include/phix_b200.h, phix_stepper_set_tiles)
FIRST_PAIR_TILE = 6


def dominant_kernel(px, g, phys, scheme, lps, fused, tile):
    """Name of the kernel that takes the time step (the key of TRAFFIC)."""
    periodic_ch = phys == px.PHYS_CH and g.dim == 2 and all(g.bc_type[i] == px.BC_PERIODIC for i in range(4))
    if g.dim == 3:
        if lps == 2:
            return "stage2_march3d"
        return "stage_march3d" if tile == 2 or phys == px.PHYS_AC else "stage_stream3d"
    if scheme == px.MULTISTEP:
        return "step_pair_ms" if fused else "stage_box"
    if lps == 1 and scheme == px.RK4 and fused:
        return "step_pair" if (tile >= FIRST_PAIR_TILE or (tile == -1 and periodic_ch)) else "step_box"
    return "stage_box" if tile == -1 else "stage_col"


class StepperRun:
    """One stepper on a single-field or coupled workload (ch2d, ac2d, chac3d)."""

    def __init__(self, px, torch, dev, args):
        from phix_b200 import workloads
        if args.workload == "ch2d":
            g, phys, prm, scheme, dt, _, fields = workloads.ch2d(n=args.n)
            self.K = STEPS_PER_INTERVAL
        elif args.workload == "ch2d_ms":
            g, phys, prm, scheme, dt, _, fields = workloads.ch2d_ms(n=args.n)
            self.K = STEPS_PER_INTERVAL
        elif args.workload == "ac2d":
            g, phys, prm, scheme, dt, _, fields = workloads.ac2d()
            self.K = 100
        else:
            g, phys, prm, scheme, dt, _, fields = workloads.chac3d(n=args.n if args.n != 1024 else 256)
            self.K = 10
        self.prec = px.F64 if args.dtype == "f64" else px.F32
        w = 8 if self.prec == px.F64 else 4
        self.nf = len(fields)
        # field-cell updates per time step (multi-step: c advances, mu is formed)
        self.cells = g.n[0] * g.n[1] * g.n[2] * (1 if scheme == px.MULTISTEP else self.nf)
        # RK4: R u,W k1 | R u,k1 W k2 | R u,k2 W k3 | R u,k1,k2,k3 W u' = 13w; Euler: R u, W u' = 2w;
        # multi-step: R c, W c', W mu = 3w
        self.alg_bytes = {px.RK4: 13, px.MULTISTEP: 3}.get(scheme, 2) * w * self.cells
        self.fields, self.g, self.phys, self.prm, self.scheme, self.dt = fields, g, phys, prm, scheme, dt
        self.st = px.Stepper(phys, scheme, self.prec, prm, dt, g)
        if args.launch != "auto":
            self.st.set_fusion(args.launch == "step")
        self.st.set_tiles(args.tiles)
        self.d = [torch.from_numpy(f).to(dev) for f in fields]
        self.st.load(self.d)
        if args.autotune:
            self.st.autotune(10)  # launch form and tile shape, timed on this grid (state restored)
        fused, tile = self.st.tiles()
        self.launch = {"one_launch_per_time_step": fused, "tile_cfg": tile, "temporal_depth": self.st.depth}
        self.lps = self.st.launches_per_step
        self.kernel = dominant_kernel(px, g, phys, scheme, self.lps, fused, tile)
        self.st.set_graph(self.K)
        self.h_in = [torch.from_numpy(f).pin_memory() for f in fields]
        self.h_out = [torch.empty_like(h).pin_memory() for h in self.h_in]
        self.io_bytes = sum(f.nbytes for f in fields)
        self.shape = (f"{g.n[0]}x{g.n[1]}" + (f"x{g.n[2]}" if g.dim == 3 else "")) + f", {self.nf} field(s)"

    def advance(self, stream):
        self.st.advance(self.K, stream)

    def e2e_step(self):
        self.st.run_host(self.h_in, self.h_out, self.K)

    def cpu_sample(self, nsteps):
        return reference_cpu_rate(self.fields, self.g, self.phys, self.prm, self.scheme, self.dt, nsteps)

    def cpu_sample_openmp(self):
        return openmp_cpu_rate(self.fields, self.g, self.phys, self.prm, self.scheme, self.dt)

    def close(self):
        self.st.close()


class BatchRun:
    """The batched engine on the 64-instance workload."""

    def __init__(self, px, torch, dev, args):
        from phix_b200 import workloads
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        # N ranks: a job of N x 64 instances (the first 64 are the 1-GPU
        # workload), bin-packed across the ranks; no collective on the data path
        grids, phys, prms, scheme, dt, _, fields = workloads.ch2d_batch(ninst=64 * world)
        if world > 1:
            mine = workloads.partition_instances([g.n[0] * g.n[1] for g in grids], world)[rank]
            grids, prms, fields = [grids[i] for i in mine], [prms[i] for i in mine], [fields[i] for i in mine]
        self.K = 20
        self.prec = px.F64 if args.dtype == "f64" else px.F32
        w = 8 if self.prec == px.F64 else 4
        self.nf = 1
        self.cells = sum(g.n[0] * g.n[1] for g in grids)
        self.alg_bytes = 13 * w * self.cells
        self.b = px.Batch(phys, scheme, self.prec, grids, prms, dt)
        self.d = [torch.from_numpy(f).to(dev) for f in fields]
        for i, t in enumerate(self.d):
            self.b.load(i, t)
        if args.launch == "step":
            self.b.set_fusion(True)
        else:
            self.b.autotune(2)  # tile shape, CTAs per SM, one launch per step or per stage
            if args.launch == "stage":
                self.b.set_fusion(False)
        self.lps = self.b.launches_per_step
        self.launch = {"temporal_depth": self.b.depth}
        periodic = all(g.bc_type[i] == px.BC_PERIODIC for g in grids for i in range(4))
        self.kernel = ("step_pair_batched" if periodic and phys == px.PHYS_CH else "step_box_batched") \
            if self.lps == 1 else "stage_box_batched"
        self.b.set_graph(self.K)
        self.h_in = [torch.from_numpy(f).pin_memory() for f in fields]
        self.h_out = [torch.empty_like(h).pin_memory() for h in self.h_in]
        self.io_bytes = sum(f.nbytes for f in fields)
        self.torch, self.dev = torch, dev
        self.grids, self.phys, self.prms, self.scheme, self.dt, self.fields = grids, phys, prms, scheme, dt, fields
        self.shape = f"{len(grids)} instances, {self.cells} cells"

    def advance(self, stream):
        self.b.advance(self.K, stream)

    def e2e_step(self):
        for h, d in zip(self.h_in, self.d):
            d.copy_(h, non_blocking=True)
        for i, d in enumerate(self.d):
            self.b.load(i, d)
        self.b.advance(self.K)
        for i, d in enumerate(self.d):
            self.b.store(i, d)
        for h, d in zip(self.h_out, self.d):
            h.copy_(d, non_blocking=True)
        self.torch.cuda.synchronize(self.dev)

    def cpu_sample(self, nsteps):
        # one 256^2 instance of the batch stands in for the per-instance rate
        i = next(k for k, g in enumerate(self.grids) if g.n[0] == 256)
        return reference_cpu_rate([self.fields[i]], self.grids[i], self.phys, self.prms[i], self.scheme, self.dt,
                                  nsteps)

    def cpu_sample_openmp(self):
        i = next(k for k, g in enumerate(self.grids) if g.n[0] == 256)
        return openmp_cpu_rate([self.fields[i]], self.grids[i], self.phys, self.prms[i], self.scheme, self.dt)

    def close(self):
        self.b.close()


def resolve_world(gpus: int, env=None) -> int:
    """World size of this run: WORLD_SIZE when a launcher set it (it must
    equal --gpus), else 1 (a single process; main() starts N ranks itself
    for --gpus N > 1)."""
    env = os.environ if env is None else env
    if "WORLD_SIZE" not in env:
        return 1
    world = int(env["WORLD_SIZE"])
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but the launcher started WORLD_SIZE={world} ranks")
    return world


def launcher_command(argv, gpus: int, port: int):
    """The torchrun command that starts `gpus` ranks of this script on one
    node with the same arguments (rendezvous on 127.0.0.1)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def free_port() -> int:
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def combine_over_ranks(total_ms: float, cells: float, e2e_ms: float, device, world: int):
    """Job totals over the ranks: the slowest rank's timed-region and e2e
    times (max) and the cells all ranks advanced (sum)."""
    if world == 1:
        return total_ms, cells, e2e_ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0].item()), float(c[0].item()), float(t[1].item())


def job_summary(world: int, steps: int, K: int, total_ms: float, job_cells: float) -> dict:
    """The whole-job keys of the JSON line: `value` = cell-updates of all
    ranks per second of the slowest rank's timed region."""
    return {"n_gpus": world, "ms_per_step": total_ms / steps, "value": job_cells * K * steps / (total_ms / 1e3)}


def bench_ours(args):
    import torch
    import torch.distributed as dist

    import phix_b200 as px

    world = resolve_world(args.gpus)
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    run = (BatchRun if args.workload == "batch" else StepperRun)(px, torch, dev, args)
    K = run.K
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    for _ in range(args.warmup):
        run.advance(stream)
        flush_l2(flush)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = px.launch_count()
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed launches by this range
        for i in range(args.steps):
            starts[i].record(stream)
            run.advance(stream)
            ends[i].record(stream)
            flush_l2(flush)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(dev)
    launches = px.launch_count() - launches0
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms, job_cells, _ = combine_over_ranks(sum(step_ms), run.cells, 0.0, dev, world)
    job = job_summary(world, args.steps, K, total_ms, job_cells)
    ms_per_step, value = job["ms_per_step"], job["value"]

    # roofline: algorithmic bytes of one time step (13w per field-cell for RK4,
    # the traffic of one launch per stage; 2w for Euler) over the device time
    # of one time step
    t_timestep = ms_per_step / 1e3 / K
    achieved = run.alg_bytes / t_timestep / 1e9
    peak, peak_kind = _peaks()
    w = 8 if run.prec == px.F64 else 4
    per_cell = run.alg_bytes // (run.cells * w) * w
    workload, data = WORKLOADS[args.workload]
    if args.workload == "ch2d" and args.n != 1024:
        workload = workload.replace("1024^2", f"{args.n}^2")

    # arithmetic-pipe roofline of the CH pair kernel (L2-resident at 1024^2):
    # lane operations (fma = 2) per cell-update counted from step2d_pair.cuh
    # on the tile's own cells, over the measured FMA peak of this GPU
    pipe = None
    if args.workload == "ch2d" and getattr(run, "kernel", "") == "step_pair":
        fp64 = run.prec == px.F64
        flops = PAIR_FLOPS_F64 if fp64 else PAIR_FLOPS_F32
        peak_t = px.measure_fma_peak(px.F64) if fp64 else px.measure_fma_peak(px.F32, packed=True)
        ach_t = flops * run.cells * K / (ms_per_step / 1e3) / 1e12
        pipe = {"bound": "fp64" if fp64 else "fp32", "achieved": ach_t, "peak": peak_t, "unit": "TFLOP/s",
                "frac": ach_t / peak_t, "flops_per_cell_update": flops,
                "note": "lane operations per cell-update on the tile's own cells (fma = 2), counted from the "
                        "kernel source; the halo recompute of the 4-stage tile adds about 43 % more; peak = "
                        "phix_measure_fma_peak on this GPU (" + ("FP64 FMA" if fp64 else "packed f32x2 FMA") +
                        " chains on every SM)"}

    if args.no_e2e:
        run.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
                              "ms_per_step": ms_per_step, "roofline_achieved_gbs": achieved, "n": args.n,
                              "workload": workload, "dtype": args.dtype, "launches_per_time_step": run.lps,
                              **getattr(run, "launch", {}), "note": "profiling run (--no-e2e)"}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return None

    # e2e through the public API with pinned host buffers: H2D of the inputs,
    # K time steps, D2H of the result, every step
    for _ in range(2):
        run.e2e_step()
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_dev = torch.cuda.Event(enable_timing=True)
    e2e_dev2 = torch.cuda.Event(enable_timing=True)
    e2e_dev.record(stream)
    for _ in range(e2e_steps):
        run.e2e_step()
    e2e_dev2.record(stream)
    torch.cuda.synchronize(dev)
    e2e_wall = time.perf_counter() - t0
    e2e_ms = max(e2e_dev.elapsed_time(e2e_dev2), 1e3 * e2e_wall)
    _, _, e2e_ms = combine_over_ranks(0.0, 0.0, e2e_ms, dev, world)
    e2e_value = job_cells * K * e2e_steps / (e2e_ms / 1e3)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            inst = " (one 256^2 instance)" if args.workload == "batch" else ""
            try:
                rate, el, n_omp, threads = run.cpu_sample_openmp()
                cpu = {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                       "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                       "sample": f"the oracle's C restatement of the same discretisation, OpenMP on {threads} "
                                 f"host threads (oracle/liboracle_omp.so, device rounding pattern), {n_omp} time "
                                 f"steps of the same workload{inst}, {el:.1f} s"}
            except Exception as e:
                cpu = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "port",
                       "sample": f"unavailable: {e}"}
            try:
                n_cpu = args.cpu_baseline_steps if args.workload != "chac3d" else 1
                rate, el = run.cpu_sample(n_cpu)
                if args.workload == "chac3d":
                    rate *= run.nf  # field-cell updates, like `value`
                cpu["reference_1thread"] = {
                    "value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                    "sample": f"reference CPU path (computeRHSCPU + applyOnCPU, GPU stage semantics), "
                              f"{n_cpu} time steps of the same workload{inst}, {el:.1f} s, 1 thread (the "
                              f"reference has no threading)"}
            except Exception as e:  # oracle/_ref not built on this machine
                cpu["reference_1thread"] = {"value": None, "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC,
            "value": job["value"],
            "unit": "cell-updates/s",
            "n_gpus": job["n_gpus"],
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": job["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": args.dtype,
            "data": data,
            "config": {"workload": workload, "shape": run.shape, "field_cells": run.cells,
                       "time_steps_per_step": K, "launches_per_time_step": run.lps,
                       **getattr(run, "launch", {}),
                       "precision_note": "FP64 stencils" if run.prec == px.F64
                       else "FP32 stencils, compensated FP32 state, FP64 reductions",
                       "l2": "flushed between timed steps (256 MiB write); within a step the fields may stay "
                             "L2-resident",
                       "parallelism": (f"instances bin-packed over {world} ranks" if args.workload == "batch"
                                       else f"replicas x{world}")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": TRAFFIC.get((args.workload, args.dtype, run.kernel)),
                         "kernel": run.kernel,
                         "note": f"algorithmic {per_cell} B per field-cell update over the CUDA-event time of "
                                 f"one time step ({run.lps} launch{'es' if run.lps > 1 else ''} per time step); "
                                 f"peak {peak_kind} (MEASURED_PEAKS.json hbm_gbs); traffic = ncu DRAM bytes per "
                                 f"launch of the dominant kernel (bytes, cold L2)"},
            "roofline_pipe": pipe,
            "hbm_gbs_effective": achieved,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": run.io_bytes,
                    "d2h_bytes_per_step": run.io_bytes},
            "gpu_launches": launches,
            "clocks": clk.result,
        }
        print(json.dumps(line), flush=True)
    run.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def bench_surrogate(args):
    """Config 5: the learned CH 512^2 surrogate (committed parameters) against
    the fused FD solver advancing the same simulated time.  One bench step =
    SUR_K surrogate steps (SUR_K * 50 FD steps of simulated time, batch 1, with
    the exact mass projection), timed with CUDA events; the FD legs run the
    same simulated time in FP32 and FP64 (CUDA graphs of 50 steps)."""
    import torch

    import phix_b200 as px
    from phix_b200 import surrogate as S
    SUR_K = 40
    p = S.load_params()
    n = S.N
    dev = torch.device("cuda", 0)
    c0 = S.initial_field(100, n)
    sg = px.Surrogate(n, n, 1, S.IN_SHIFT, S.IN_SCALE, S.OUT_SCALE)
    sg.set_params(p)
    a = torch.from_numpy(c0.copy()).to(dev)[None]
    b = torch.empty_like(a)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        for _ in range(SUR_K):
            sg.step(a, b)
            a, b = b, a
        flush_l2(flush)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = px.launch_count()
    with ClockSampler(dev.index) as clk:
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed launches by this range
        for i in range(args.steps):
            ev[i][0].record(stream)
            for _ in range(SUR_K):
                sg.step(a, b, stream)
                a, b = b, a
            ev[i][1].record(stream)
            flush_l2(flush)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(dev)
    launches = px.launch_count() - launches0
    total_ms = sum(s_.elapsed_time(e_) for s_, e_ in ev)
    ms_per_step = total_ms / args.steps
    sim_per_step = SUR_K * S.STEPS_PER_CALL * S.DT
    value = sim_per_step / (ms_per_step / 1e3)
    # e2e: host c -> device, SUR_K steps, device -> host, every step
    h_in = torch.from_numpy(c0.copy())[None].pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    t0 = time.perf_counter()
    for _ in range(max(3, args.steps // 2)):
        a.copy_(h_in, non_blocking=True)
        for _ in range(SUR_K):
            sg.step(a, b, stream)
            a, b = b, a
        h_out.copy_(a, non_blocking=True)
        torch.cuda.synchronize(dev)
    e2e_ms = 1e3 * (time.perf_counter() - t0) / max(3, args.steps // 2)
    sg.close()
    fd = S.time_speed(p, sur_steps=SUR_K)
    flops = 2 * 9 * (32 + 32 * 32 + 32 * 32 + 32) * n * n  # per surrogate step
    achieved = flops * SUR_K / (ms_per_step / 1e3) / 1e12
    peak, peak_kind = 1590.0, "fallback"  # dense BF16 TFLOP/s measured earlier on this pool's B200s
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peak, peak_kind = float(json.load(f)["bf16_tflops"]), "measured"
    line = {
        "metric": "surrogate vs FD sim-time/s (CH 512^2, one surrogate step = 50 FD steps)",
        "value": value, "unit": "simulated time units/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 activations, fp32 accumulate, fp64 state",
        "data": "synthetic: c0 = U[0.35,0.65] mean + U[-0.01,0.01], numpy default_rng(100); "
                "parameters trained on FD trajectories of seeds 100-299",
        "config": {"workload": "CH 512^2 periodic surrogate rollout, batch 1", "surrogate_steps_per_step": SUR_K,
                   "l2": "flushed between timed steps"},
        "fd_comparison": {"fd_f32_sim_time_per_s": fd["sim_time"] / (fd["fd_f32_ms"] / 1e3),
                          "fd_f64_sim_time_per_s": fd["sim_time"] / (fd["fd_f64_ms"] / 1e3),
                          "speedup_vs_fd_f32": fd["fd_f32_ms"] / fd["surrogate_ms"],
                          "speedup_vs_fd_f64": fd["fd_f64_ms"] / fd["surrogate_ms"]},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": None,
                     "note": "9.97 GFLOP per surrogate step (2*9*(32+1024+1024+32) per pixel) over the "
                             f"CUDA-event time of the whole step (all kernels); peak bf16_tflops {peak_kind}"},
        "e2e": {"value": sim_per_step / (e2e_ms / 1e3), "unit": "simulated time units/s",
                "h2d_bytes_per_step": h_in.numel() * 8, "d2h_bytes_per_step": h_out.numel() * 8},
        "gpu_launches": launches,
        "clocks": clk.result,
    }
    print(json.dumps(line), flush=True)
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
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["surrogate"], default="ch2d",
                    help="ch2d: the headline CH 1024^2 case; ac2d, chac3d, batch, surrogate: the other "
                         "configurations")
    ap.add_argument("--tiles", type=int, default=-1, help="2-D stage tile shape (phix_stepper_set_tiles)")
    ap.add_argument("--launch", choices=["auto", "step", "stage"], default="auto",
                    help="one launch per RK4 time step, one per stage, or the library default (auto)")
    ap.add_argument("--autotune", action="store_true",
                    help="time every launch form and tile shape on the grid first (phix_stepper_autotune)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # --gpus N without a launcher: start N ranks of this script on this node
        import subprocess as sp
        raise SystemExit(sp.call(launcher_command(sys.argv[1:], args.gpus, free_port())))
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)  # timing rule: at least 3 untimed warm-up steps
    if args.impl == "reference":
        bench_reference(args)
    elif args.workload == "surrogate":
        bench_surrogate(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
