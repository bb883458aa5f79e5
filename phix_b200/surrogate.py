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


def train(seeds, nsteps: int = 40000, every: int = STEPS_PER_CALL, batch: int = 16, lr: float = 1e-3,
          updates_per_snapshot: int = 1, init_seed: int = 0, n: int = N, params=None, log_every: int = 0):
    """Train on FD trajectories generated on the fly; returns (flat params, log)."""
    import torch

    if params is None:
        params = init_params(init_seed)
    sg = Surrogate(n, n, batch, IN_SHIFT, IN_SCALE, OUT_SCALE)
    sg.set_params(params)
    log = TrainLog()
    g = make_grid((n, n))
    seeds = list(seeds)
    for start in range(0, len(seeds), batch):
        chunk = seeds[start:start + batch]
        b = Batch(PHYS_CH, RK4, F32, [g] * len(chunk), [PRM] * len(chunk), DT)
        for i, s in enumerate(chunk):
            b.load(i, _stored(g, initial_field(s, n)))
        b.set_graph(every)
        stored = torch.zeros((len(chunk),) + tuple(stored_shape(g)), dtype=torch.float64, device="cuda")
        prev = torch.empty((len(chunk), n, n), dtype=torch.float64, device="cuda")
        cur = torch.empty_like(prev)

        def snapshot(dst):
            for i in range(len(chunk)):
                b.store(i, stored[i])
                plane_gather(stored[i], dst[i], n, n, 1)

        snapshot(prev)
        for k in range(nsteps // every):
            t0 = time.perf_counter()
            b.advance(every)
            snapshot(cur)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            for _ in range(updates_per_snapshot):
                loss = sg.grad(prev, cur)
                sg.adam(lr)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            log.seconds_fd += t1 - t0
            log.seconds_train += t2 - t1
            log.losses.append(loss)
            log.pairs += len(chunk)
            if log_every and k % log_every == 0:
                print(f"chunk {start // batch} snap {k}: loss {loss:.4e}", flush=True)
            prev, cur = cur, prev
        b.close()
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
