"""Training and rollout of the learned Cahn-Hilliard surrogate.

Problem: 2-D CH, 512x512 periodic, dx=1, kappa=0.5, M=1, f=c^2(1-c)^2,
dt=0.005; one surrogate step = 50 FD time steps (t += 0.25).

Training data come from the project's own FD solver (the batched engine,
FP32 stencils): trajectories with c0 = U[0.35, 0.65] mean plus U[-0.01, 0.01]
noise (numpy default_rng(seed)), snapshots every 50 steps, pairs
(c_t, c_{t+50}).  The network is trained with the tensor-core forward and
backward kernels (phix_surrogate_grad) and Adam (phix_surrogate_adam).

Rollout: surrogate steps with the exact mean-mass projection; every
`recheck` steps the FD solver checks the surrogate state:
  * energy: the FP64 free energy must not have increased, and
  * residual: the surrogate's mean rate (c_{n+1} - c_n)/(50 dt) is compared
    with one evaluation of the FD right-hand side at c_n,
and on a violation the FD solver takes over for the next `recheck` steps.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field

import numpy as np

from . import (BC_PERIODIC, F32, F64, PHYS_CH, RK4, Batch, Stepper, Surrogate, make_grid, plane_gather,
               plane_scatter, reduce_mass_energy, stored_shape)

N = 512
KAPPA, MOB, DT = 0.5, 1.0, 0.005
PRM = [MOB, KAPPA, 1.0, 0.0, 1.0]
STEPS_PER_CALL = 50
IN_SHIFT, IN_SCALE, OUT_SCALE = 0.5, 4.0, 0.01
PARAMS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "surrogate_ch512.npz")


def initial_field(seed: int, n: int = N) -> np.ndarray:
    rng = np.random.default_rng(seed)
    cbar = rng.uniform(0.35, 0.65)
    return cbar + rng.uniform(-0.01, 0.01, size=(n, n))


def _stored(g, plane: np.ndarray) -> np.ndarray:
    a = np.zeros(stored_shape(g))
    a[1, 1:-1, 1:-1] = plane
    return a


@dataclass
class TrainLog:
    losses: list = field(default_factory=list)
    seconds_fd: float = 0.0
    seconds_train: float = 0.0
    pairs: int = 0
    updates: int = 0


def generate(seeds, nsteps: int, every: int = STEPS_PER_CALL, n: int = N, precision=F32):
    """FD trajectories of `seeds` on the batched engine: a [len(seeds),
    nsteps // every + 1, n, n] float64 CUDA tensor of snapshots every `every`
    time steps (snapshot 0 = the initial field)."""
    import torch
    g = make_grid((n, n))
    ns = nsteps // every + 1
    data = torch.empty((len(seeds), ns, n, n), dtype=torch.float64, device="cuda")
    b = Batch(PHYS_CH, RK4, precision, [g] * len(seeds), [PRM] * len(seeds), DT)
    stored = torch.zeros((len(seeds),) + tuple(stored_shape(g)), dtype=torch.float64, device="cuda")
    for i, sd in enumerate(seeds):
        stored[i].copy_(torch.from_numpy(_stored(g, initial_field(sd, n))))
        b.load(i, stored[i])
    b.set_graph(every)

    def snapshot(k):
        for i in range(len(seeds)):
            b.store(i, stored[i])
            plane_gather(stored[i], data[i, k], n, n, 1)

    snapshot(0)
    for k in range(1, ns):
        b.advance(every)
        snapshot(k)
    torch.cuda.synchronize()
    b.close()
    return data


def shard_seeds(seeds, rank: int, world: int):
    """Data-parallel training: rank r generates and trains on seeds r,
    r+world, ...  Every seed is assigned, so shards differ in length by at
    most one; train() pads the shorter shards' schedules with zero-weight
    updates so that all ranks take the same number of gradient all-reduces."""
    return list(seeds)[rank::world]


def dp_update_counts(shard_sizes, ns: int, chunk: int, batch: int, epochs: int):
    """Adam updates each rank's shard yields in train(): per chunk of
    `chunk` trajectories of `ns` snapshots, `epochs` passes over the chunk's
    (ns - 1) * T pairs in whole batches."""
    counts = []
    for size in shard_sizes:
        u = 0
        for start in range(0, size, chunk):
            t = min(chunk, size - start)
            u += epochs * ((t * (ns - 1)) // batch)
        counts.append(u)
    return counts


def allreduce_mean_(t, group=None):
    """In-place mean of a gradient tensor over the ranks of `group`
    (torch.distributed: NCCL between GPUs, gloo on CPU)."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t.div_(dist.get_world_size(group))
    return t


def allreduce_active_mean_(t, active: bool, n_active: int, group=None):
    """In-place mean over the ranks that still have a batch: a rank whose
    shard is used up (`active` False) contributes zeros but still takes part
    in the all-reduce, so every rank issues the same collectives and applies
    the same averaged gradient.  `n_active` (>= 1) is the number of active
    ranks, known on every rank from dp_update_counts."""
    import torch.distributed as dist
    if not active:
        t.zero_()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t.div_(n_active)
    return t


class _DeviceVector:
    """A float32 device vector owned by the library, exposed to torch without a
    copy through the CUDA array interface."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def train(seeds, nsteps: int = 40000, every: int = STEPS_PER_CALL, batch: int = 16, lr: float = 1e-3,
          chunk: int = 25, epochs: int = 1, lr_final: float = 1e-4, init_seed: int = 0, n: int = N, params=None,
          log_every: int = 0, shuffle_seed: int = 0, distributed: bool = False):
    """Train on FD trajectories generated chunk by chunk (`chunk` trajectories
    at a time, kept on the GPU): `epochs` passes over the chunk's shuffled
    (c_t, c_{t+every}) pairs per chunk, Adam with a learning rate decaying
    geometrically from `lr` to `lr_final` over the whole run.  With
    `distributed` (an initialised torch.distributed NCCL group, one rank per
    GPU) each rank takes its shard of the seeds and the gradients are averaged
    over the ranks before every Adam step, so every rank holds the same
    parameters.  Returns (flat params, log)."""
    import torch
    if params is None:
        params = init_params(init_seed)
    sg = Surrogate(n, n, batch, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    log = TrainLog()
    seeds = list(seeds)
    grads = None
    ns = nsteps // every + 1
    counts = dp_update_counts([len(seeds)], ns, chunk, batch, epochs)
    if distributed:
        import torch.distributed as dist
        world = dist.get_world_size()
        shards = [shard_seeds(seeds, r, world) for r in range(world)]
        counts = dp_update_counts([len(x) for x in shards], ns, chunk, batch, epochs)
        seeds = shards[dist.get_rank()]
        grads = torch.as_tensor(_DeviceVector(sg.grad_ptr(), sg.nparams), device="cuda")
    rng = np.random.default_rng(shuffle_seed)
    total = max(1, max(counts))  # the same learning-rate schedule on every rank

    def n_active(u):
        return sum(1 for c in counts if c > u)
    for start in range(0, len(seeds), chunk):
        t0 = time.perf_counter()
        data = generate(seeds[start:start + chunk], nsteps, every, n)
        log.seconds_fd += time.perf_counter() - t0
        t0 = time.perf_counter()
        T = data.shape[0]
        npairs = T * (ns - 1)
        for _ in range(epochs):
            perm = torch.from_numpy(rng.permutation(npairs)).cuda()
            for j in range(0, npairs - batch + 1, batch):
                idx = perm[j:j + batch]
                ti, si = idx // (ns - 1), idx % (ns - 1)
                a = data[ti, si].contiguous()
                nxt = data[ti, si + 1].contiguous()
                loss = sg.grad(a, nxt)
                if grads is not None:
                    allreduce_active_mean_(grads, True, n_active(log.updates))
                rate = lr * (lr_final / lr) ** min(1.0, log.updates / total)
                sg.adam(rate)
                log.updates += 1
                log.pairs += batch
                log.losses.append(loss)
                if log_every and log.updates % log_every == 0:
                    print(f"update {log.updates}/{total}: loss {np.mean(log.losses[-log_every:]):.4e} "
                          f"lr {rate:.2e}", flush=True)
        torch.cuda.synchronize()
        log.seconds_train += time.perf_counter() - t0
        del data
    # a shorter shard's rank keeps taking part in the all-reduces (with a
    # zero gradient) and applies the same Adam steps until every rank is done
    while grads is not None and log.updates < total:
        allreduce_active_mean_(grads, False, n_active(log.updates))
        sg.adam(lr * (lr_final / lr) ** min(1.0, log.updates / total))
        log.updates += 1
    p, _ = sg.get_params()
    sg.close()
    return p, log


LAYERS = ((1, 32), (32, 32), (32, 32), (32, 1))


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (std sqrt(2 / (9 cin))), zero biases, the last layer
    scaled by 0.1 so the untrained step is close to the identity; returned as
    the flat FP32 vector of phix_surrogate_set_params (W[cout, ky, kx, cin])."""
    from . import surrogate_params_to_flat
    rng = np.random.default_rng(seed)
    params = []
    for cin, cout in LAYERS:
        w = rng.normal(0.0, np.sqrt(2.0 / (9 * cin)), size=(cout, 3, 3, cin)).astype(np.float32)
        params += [w, np.zeros(cout, dtype=np.float32)]
    params[6] *= 0.1
    return surrogate_params_to_flat(params)


def fd_run(c0: np.ndarray, nsteps: int, precision=F64, graph: int = 100):
    """Plain fused FD solver: c0 [n, n] -> c after nsteps (numpy), elapsed s."""
    import torch
    n = c0.shape[0]
    g = make_grid((n, n))
    st = Stepper(PHYS_CH, RK4, precision, PRM, DT, g)
    d = torch.from_numpy(_stored(g, c0)).cuda()
    st.load([d])
    st.set_graph(graph)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st.advance(nsteps)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    st.store([d])
    torch.cuda.synchronize()
    st.close()
    return d.cpu().numpy()[1, 1:-1, 1:-1].copy(), el


@dataclass
class RolloutLog:
    surrogate_steps: int = 0
    fd_takeovers: int = 0
    rechecks: int = 0
    seconds: float = 0.0


def rollout(params: np.ndarray, c0: np.ndarray, nsteps: int, recheck: int = 10, resid_tol: float = 0.5,
            use_fd_fallback: bool = True):
    """Advance c0 by nsteps surrogate steps (50 FD steps each) with the FD
    re-check; returns (c [n, n] float64, RolloutLog)."""
    import torch
    n = c0.shape[0]
    g = make_grid((n, n))
    sg = Surrogate(n, n, 1, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    st = Stepper(PHYS_CH, RK4, F64, PRM, DT, g)
    st.set_graph(STEPS_PER_CALL)
    stored = torch.from_numpy(_stored(g, c0)).cuda()
    rhs = torch.zeros_like(stored)
    a = torch.from_numpy(c0.copy()).cuda()[None]
    b = torch.empty_like(a)
    log = RolloutLog()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    k = 0
    fd_left = 0
    while k < nsteps:
        if fd_left > 0:
            plane_scatter(a[0], stored, n, n, 1)
            st.load([stored])
            st.advance(STEPS_PER_CALL)
            st.store([stored])
            plane_gather(stored, a[0], n, n, 1)
            fd_left -= 1
            k += 1
            continue
        sg.step(a, b)
        if recheck and use_fd_fallback and (k % recheck == 0):
            log.rechecks += 1
            if not _recheck_ok(g, a[0], b[0], stored, rhs, resid_tol):
                log.fd_takeovers += 1
                fd_left = recheck
                continue
        a, b = b, a
        log.surrogate_steps += 1
        k += 1
    torch.cuda.synchronize()
    log.seconds = time.perf_counter() - t0
    out = a[0].cpu().numpy().copy()
    sg.close()
    st.close()
    return out, log


def _energy(g, plane, stored):
    import torch
    n = plane.shape[0]
    plane_scatter(plane, stored, n, n, 1)
    return reduce_mass_energy([stored], PHYS_CH, PRM, g)[1]


def _rhs_norms(g, plane, stored, rhs, rate):
    """||rate - F(plane)|| / ||F(plane)|| with F the FD right-hand side."""
    import torch
    from . import PW_DW, bc_apply, lap_accumulate, pointwise_accumulate
    n = plane.shape[0]
    plane_scatter(plane, stored, n, n, 1)
    bc_apply(stored, g)
    mu = torch.zeros_like(stored)
    pointwise_accumulate(mu, stored, None, 1.0, PW_DW, PRM, g)
    lap_accumulate(mu, stored, -KAPPA, g)
    bc_apply(mu, g)
    rhs.zero_()
    lap_accumulate(rhs, mu, MOB, g)
    F = rhs[1, 1:-1, 1:-1]
    return float(torch.linalg.norm(rate - F) / torch.clamp(torch.linalg.norm(F), min=1e-30))


def _recheck_ok(g, c_old, c_new, stored, rhs, resid_tol):
    e0 = _energy(g, c_old, stored)
    e1 = _energy(g, c_new, stored)
    if e1 > e0 * (1.0 + 1e-9):
        return False
    rate = (c_new - c_old) / (STEPS_PER_CALL * DT)
    return _rhs_norms(g, c_old, stored, rhs, rate) <= resid_tol


# ---------------------------------------------------------------------------
# evaluation and timing
# ---------------------------------------------------------------------------
def _rel(a, b):
    import torch
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _rel_fluct(a, b):
    import torch
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b - b.mean()))


def evaluate(params: np.ndarray, seeds, checkpoints=(1, 10, 50, 100, 200, 400, 800), n: int = N):
    """Pure surrogate rollouts (no FD take-over) of held-out seeds against the
    FP64 fused FD solution at the same times.  Per seed and checkpoint (in
    surrogate steps of STEPS_PER_CALL FD steps): rel-L2 = ||c_s - c_fd|| /
    ||c_fd||, the same relative to the fluctuation ||c_fd - mean||, the
    no-network baseline (c stays c0) on both measures, and the mass drift."""
    import torch
    g = make_grid((n, n))
    sg = Surrogate(n, n, 1, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    rows = []
    for sd in seeds:
        c0 = initial_field(sd, n)
        # FD FP64 at the checkpoints
        st = Stepper(PHYS_CH, RK4, F64, PRM, DT, g)
        d = torch.from_numpy(_stored(g, c0)).cuda()
        st.load([d])
        st.set_graph(STEPS_PER_CALL)
        fd = {}
        done = 0
        plane = torch.empty((n, n), dtype=torch.float64, device="cuda")
        for cp in checkpoints:
            st.advance((cp - done) * STEPS_PER_CALL)
            done = cp
            st.store([d])
            plane_gather(d, plane, n, n, 1)
            fd[cp] = plane.clone()
        st.close()
        # surrogate
        a = torch.from_numpy(c0.copy()).cuda()[None]
        b = torch.empty_like(a)
        c0t = a[0].clone()
        k = 0
        for cp in checkpoints:
            while k < cp:
                sg.step(a, b)
                a, b = b, a
                k += 1
            ref = fd[cp]
            rows.append({"seed": sd, "step": cp, "rel_l2": _rel(a[0], ref), "rel_l2_fluct": _rel_fluct(a[0], ref),
                         "baseline_rel_l2": _rel(c0t, ref), "baseline_rel_l2_fluct": _rel_fluct(c0t, ref),
                         "mass_rel": abs(float(a[0].mean() - c0t.mean())) / abs(float(c0t.mean()))})
    sg.close()
    return rows


def time_speed(params: np.ndarray, sur_steps: int = 40, n: int = N, warmup: int = 3):
    """Device time of `sur_steps` surrogate steps (batch 1, with the mass
    projection) against the fused FD solver advancing the same simulated time
    (sur_steps * STEPS_PER_CALL steps) in FP32 and FP64; CUDA events on the
    launching stream, graphs for the FD steps.  Returns a dict of ms."""
    import torch
    g = make_grid((n, n))
    c0 = initial_field(100, n)
    sg = Surrogate(n, n, 1, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    a = torch.from_numpy(c0.copy()).cuda()[None]
    b = torch.empty_like(a)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(warmup):
        sg.step(a, b)
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(sur_steps):
        sg.step(a, b)
        a, b = b, a
    ev[1].record()
    torch.cuda.synchronize()
    out = {"surrogate_ms": ev[0].elapsed_time(ev[1])}
    sg.close()
    for prec, key in ((F32, "fd_f32_ms"), (F64, "fd_f64_ms")):
        st = Stepper(PHYS_CH, RK4, prec, PRM, DT, g)
        d = torch.from_numpy(_stored(g, c0)).cuda()
        st.load([d])
        st.set_graph(STEPS_PER_CALL)
        for _ in range(warmup):
            st.advance(STEPS_PER_CALL)
        torch.cuda.synchronize()
        ev[0].record()
        st.advance(sur_steps * STEPS_PER_CALL)
        ev[1].record()
        torch.cuda.synchronize()
        out[key] = ev[0].elapsed_time(ev[1])
        st.close()
    out["sim_time"] = sur_steps * STEPS_PER_CALL * DT
    return out


def tradeoff(params: np.ndarray, seeds=(300, 301), fd_blocks=(0, 10, 50, 100, 200, 400, 600),
             fd_every=(0, 10, 4), total: int = 800, n: int = N):
    """The accuracy / speed trade-off of handing part of a run to the FD
    solver.  For each held-out seed, each W in fd_blocks and each R in
    fd_every: the fused FP64 FD solver advances the first W blocks
    (W * STEPS_PER_CALL steps), and after that every R-th block (R = 0: none);
    the surrogate (with the mass projection) advances the other blocks.  Each
    row reports rel-L2 against the pure FP64 FD state after `total` blocks and
    the schedule's speed-up over pure FD, from the measured device times of
    one surrogate step and of one block of fused FD (FP32 and FP64).  Pure
    surrogate rollouts drift in the early linear regime of spinodal
    decomposition, where differences grow exponentially; the rows show how
    much of the run FD must cover for a given error."""
    import torch
    g = make_grid((n, n))
    tm = time_speed(params, sur_steps=40, n=n)
    per_sur = tm["surrogate_ms"] / 40.0
    per_f32 = tm["fd_f32_ms"] / 40.0
    per_f64 = tm["fd_f64_ms"] / 40.0
    sg = Surrogate(n, n, 1, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    plane = torch.empty((n, n), dtype=torch.float64, device="cuda")
    st = Stepper(PHYS_CH, RK4, F64, PRM, DT, g)
    st.set_graph(STEPS_PER_CALL)
    d = torch.empty(stored_shape(g), dtype=torch.float64, device="cuda")
    rows = []
    for sd in seeds:
        c0 = initial_field(sd, n)
        d.copy_(torch.from_numpy(_stored(g, c0)))
        st.load([d])
        fd, done = {}, 0
        for w in sorted(set(fd_blocks) | {total}):
            st.advance((w - done) * STEPS_PER_CALL)
            done = w
            st.store([d])
            plane_gather(d, plane, n, n, 1)
            fd[w] = plane.clone()
        ref = fd[total]
        for w in fd_blocks:
            for r in fd_every:
                a = fd[w].clone()[None]
                b = torch.empty_like(a)
                nfd = 0
                for k in range(w, total):
                    if r and (k - w) % r == r - 1:  # this block by FD
                        plane_scatter(a[0], d, n, n, 1)
                        st.load([d])
                        st.advance(STEPS_PER_CALL)
                        st.store([d])
                        plane_gather(d, a[0], n, n, 1)
                        nfd += 1
                    else:
                        sg.step(a, b)
                        a, b = b, a
                nsur = total - w - nfd
                t64 = (w + nfd) * per_f64 + nsur * per_sur
                t32 = (w + nfd) * per_f32 + nsur * per_sur
                rows.append({"seed": sd, "fd_warmup_steps": w * STEPS_PER_CALL, "fd_every": r,
                             "fd_blocks": w + nfd, "surrogate_steps": nsur,
                             "rel_l2": _rel(a[0], ref), "rel_l2_fluct": _rel_fluct(a[0], ref),
                             "mass_rel": abs(float(a[0].mean() - fd[0].mean())) / abs(float(fd[0].mean())),
                             "speedup_vs_fd_f64": total * per_f64 / t64,
                             "speedup_vs_fd_f32": total * per_f32 / t32})
                if w == total:
                    break
    st.close()
    sg.close()
    return rows, tm


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train / evaluate / time the CH 512^2 surrogate")
    ap.add_argument("cmd", choices=["train", "evaluate", "time", "rollout", "tradeoff"])
    ap.add_argument("--steps", type=int, default=800, help="rollout: surrogate steps")
    ap.add_argument("--recheck", type=int, default=10, help="rollout: FD re-check every this many steps")
    ap.add_argument("--params", default=PARAMS_FILE)
    ap.add_argument("--seeds", default="100:300", help="training seeds lo:hi")
    ap.add_argument("--eval-seeds", default="300:304")
    ap.add_argument("--nsteps", type=int, default=40000)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--chunk", type=int, default=25)
    ap.add_argument("--log-every", type=int, default=500)
    ap.add_argument("--distributed", action="store_true",
                    help="data-parallel training under torchrun (one rank per GPU, NCCL gradient averaging)")
    args = ap.parse_args(argv)
    lo, hi = (int(v) for v in args.seeds.split(":"))
    elo, ehi = (int(v) for v in args.eval_seeds.split(":"))
    if args.cmd == "train":
        rank = 0
        if args.distributed:
            import datetime

            import torch
            import torch.distributed as dist
            local = int(os.environ.get("LOCAL_RANK", "0"))
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
            rank = dist.get_rank()
        p, log = train(range(lo, hi), nsteps=args.nsteps, batch=args.batch, lr=args.lr, lr_final=args.lr_final,
                       chunk=args.chunk, epochs=args.epochs, log_every=args.log_every if rank == 0 else 0,
                       distributed=args.distributed)
        if args.distributed:
            dist.barrier()
            dist.destroy_process_group()
        if rank != 0:
            return
        np.savez(args.params, params=p, seeds=np.arange(lo, hi), nsteps=args.nsteps, epochs=args.epochs,
                 losses=np.asarray(log.losses[::10], np.float32))
        print(json.dumps({"updates": log.updates, "pairs": log.pairs, "seconds_fd": log.seconds_fd,
                          "seconds_train": log.seconds_train, "loss_first": float(np.mean(log.losses[:50])),
                          "loss_last": float(np.mean(log.losses[-50:]))}))
    else:
        p = load_params(args.params)
        if args.cmd == "evaluate":
            for r in evaluate(p, range(elo, ehi)):
                print(json.dumps(r))
        elif args.cmd == "rollout":
            import torch
            for sd in range(elo, ehi):
                c0 = initial_field(sd)
                out, rl = rollout(p, c0, args.steps, recheck=args.recheck)
                ref, fd_s = fd_run(c0, args.steps * STEPS_PER_CALL, precision=F64)
                a, r = torch.from_numpy(out), torch.from_numpy(ref)
                print(json.dumps({"seed": sd, "steps": args.steps, "recheck": args.recheck, "rel_l2": _rel(a, r),
                                  "rel_l2_fluct": _rel_fluct(a, r), "mass_rel": abs(float(out.mean() - c0.mean()))
                                  / abs(float(c0.mean())), "surrogate_steps": rl.surrogate_steps,
                                  "fd_takeovers": rl.fd_takeovers, "rechecks": rl.rechecks,
                                  "rollout_s": rl.seconds, "fd_f64_s": fd_s}))
        elif args.cmd == "tradeoff":
            rows, tm = tradeoff(p, seeds=tuple(range(elo, ehi)))
            print(json.dumps({"times_ms": tm}))
            for r in rows:
                print(json.dumps(r))
        else:
            print(json.dumps(time_speed(p)))


def load_params(path: str = PARAMS_FILE) -> np.ndarray:
    """Trained parameters (flat FP32 vector) saved by `python -m phix_b200.surrogate train`."""
    return np.load(path)["params"].astype(np.float32)


if __name__ == "__main__":
    main()
