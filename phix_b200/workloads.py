"""Seeded synthetic workloads of the benchmark configurations.

Each builder returns (grid, physics, prm, scheme, dt, nsteps, fields) where
fields are FP64 stored arrays (ghost-padded, x fastest) drawn with
numpy.random.default_rng(seed) in a fixed order.  No dataset is involved: the
reference's cases are seeded synthetic initial conditions.
"""
from __future__ import annotations

import numpy as np

from . import (BC_NOFLUX, BC_PERIODIC, EULER, MULTISTEP, PHYS_AC, PHYS_CH, PHYS_CHAC, RK4, make_grid, stored_shape)


def _stored(g, phys_vals):
    a = np.zeros(stored_shape(g), dtype=np.float64)
    gh = g.ghost
    n0, n1, n2 = g.n[0], g.n[1], g.n[2]
    a[gh:gh + n2, gh:gh + n1, gh:gh + n0] = phys_vals.reshape(n2, n1, n0)
    return a


def ac2d(n=128, seed=0, nsteps=1000):
    """2-D Allen-Cahn, n x n periodic, dx=1, dt=0.01, L=kappa=1, Euler, FP64;
    phi0 i.i.d. uniform in [-0.05, 0.05]."""
    g = make_grid((n, n))
    rng = np.random.default_rng(seed)
    phi = rng.uniform(-0.05, 0.05, size=(1, n, n))
    return g, PHYS_AC, [1.0, 1.0], EULER, 0.01, nsteps, [_stored(g, phi)]


def ch2d(n=1024, seed=1, nsteps=20000, kappa=0.5, M=1.0, c_mean=0.5, noise=0.01, dt=0.005):
    """2-D Cahn-Hilliard spinodal decomposition, n x n periodic, dx=1,
    f = c^2(1-c)^2 (rho=1, ca=0, cb=1), RK4; c0 = c_mean + uniform[-noise, noise]."""
    g = make_grid((n, n))
    rng = np.random.default_rng(seed)
    c = c_mean + rng.uniform(-noise, noise, size=(1, n, n))
    return g, PHYS_CH, [M, kappa, 1.0, 0.0, 1.0], RK4, dt, nsteps, [_stored(g, c)]


def ch2d_ms(n=1024, seed=1, nsteps=20000, kappa=0.5, M=1.0, c_mean=0.5, noise=0.01, dt=0.005):
    """The Cahn-Hilliard application's form (Cahn-Hillard_double-well.cu:
    mu = f'(c) - kappa lap c as a STEADY field, then dc/dt = M lap mu by
    Euler), n x n periodic, dx=1, f = c^2(1-c)^2; c0 as in ch2d, mu0 = 0."""
    g = make_grid((n, n))
    rng = np.random.default_rng(seed)
    c = c_mean + rng.uniform(-noise, noise, size=(1, n, n))
    return g, PHYS_CH, [M, kappa, 1.0, 0.0, 1.0], MULTISTEP, dt, nsteps, [_stored(g, c), _stored(g, np.zeros_like(c))]


def chac3d(n=256, seed=2, nsteps=5000):
    """3-D coupled CH+AC, n^3, zero-flux x, periodic y and z, dx=1, dt=0.002,
    RK4, M=L=1, kappa_c=kappa_eta=0.5, lambda=1; c0 = 0.4 +- 0.01,
    eta0 uniform in [0, 0.1]."""
    g = make_grid((n, n, n), bc=(BC_NOFLUX, BC_NOFLUX, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC))
    rng = np.random.default_rng(seed)
    c = 0.4 + rng.uniform(-0.01, 0.01, size=(n, n, n))
    eta = rng.uniform(0.0, 0.1, size=(n, n, n))
    return g, PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0], RK4, 0.002, nsteps, [_stored(g, c), _stored(g, eta)]


BATCH_SIZES = (128, 256, 384, 512, 768, 1024)


def ch2d_batch(ninst=64, seed=3, nsteps=5000, dt=0.005, sizes=BATCH_SIZES):
    """Batched 2-D Cahn-Hilliard: `ninst` independent periodic instances, grid
    n x n with n drawn uniformly from `sizes`, kappa ~ U[0.25, 2],
    M ~ U[0.5, 2], mean c ~ U[0.3, 0.7] plus U[-0.01, 0.01] noise, RK4.
    Draw order per instance: size, kappa, M, mean, noise field."""
    rng = np.random.default_rng(seed)
    grids, prms, fields = [], [], []
    for _ in range(ninst):
        n = int(rng.choice(sizes))
        kappa = float(rng.uniform(0.25, 2.0))
        M = float(rng.uniform(0.5, 2.0))
        cbar = float(rng.uniform(0.3, 0.7))
        g = make_grid((n, n))
        c = cbar + rng.uniform(-0.01, 0.01, size=(1, n, n))
        grids.append(g)
        prms.append([M, kappa, 1.0, 0.0, 1.0])
        fields.append(_stored(g, c))
    return grids, PHYS_CH, prms, RK4, dt, nsteps, fields


def partition_instances(costs, world: int):
    """Greedy bin-pack of independent instances onto `world` ranks: instances
    in decreasing cost (ties by index) go to the least-loaded rank (ties by
    rank).  Returns one list of instance indices per rank, each ascending."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
