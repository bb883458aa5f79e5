"""Generate the golden vectors in tests/golden/*.npz.

Each case runs the REFERENCE library itself -- its own CPU kernels
(Equation::computeRHSCPU, BoundaryCondition::applyOnCPU) compiled from its
sources by oracle/Makefile into oracle/_ref/libphix_ref.so, driven with the
GPU solver's stage semantics by oracle/ref_harness.cu -- on small seeded
inputs, and stores inputs and outputs.  The fixtures then travel with the
repository; the reference tree does not.

    make -C oracle ref && python tests/golden/gen_golden.py

Inputs are full stored arrays whose ghost cells hold random values, so a
kernel that reads a ghost its BC should have refreshed gets caught.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import (BC_FIXED, BC_NONE, BC_NOFLUX, BC_PERIODIC, EULER, PHYS_AC, PHYS_CH,  # noqa: E402
                           PHYS_CHAC, RK4, Grid, Reference)

P, N, F, X = BC_PERIODIC, BC_NOFLUX, BC_FIXED, BC_NONE

# name: (grid kwargs, physics, prm, scheme, dt, nsteps, init(lo, hi) per field)
CASES = {
    # the reference's own case (config 1) at 16x12
    "ac2d_euler": (dict(n=(16, 12)), PHYS_AC, [1.0, 1.0], EULER, 0.01, 25, [(-0.05, 0.05)]),
    "ac2d_rk4": (dict(n=(16, 12), d=(0.5, 0.5)), PHYS_AC, [1.0, 1.0], RK4, 0.01, 25, [(-0.5, 0.5)]),
    "ac1d_rk4": (dict(n=(33,), d=(0.5,)), PHYS_AC, [1.0, 2.0], RK4, 0.01, 20, [(-0.5, 0.5)]),
    "ac3d_rk4_ghost2": (dict(n=(8, 7, 6), ghost=2, bc=(P, P, N, N, F, F), bc_val=(0, 0, 0, 0, 0.2, -0.1)),
                        PHYS_AC, [1.0, 1.0], RK4, 0.01, 10, [(-0.5, 0.5)]),
    "ac2d_bc_none_y": (dict(n=(12, 9), bc=(P, P, X, X, 0, 0)), PHYS_AC, [1.0, 0.5], EULER, 0.01, 12,
                       [(-0.5, 0.5)]),
    # config 2 (single-equation CH, RK4) at 24x20 with larger noise
    "ch2d_rk4": (dict(n=(66, 18)), PHYS_CH, [1.0, 0.5, 1.0, 0.0, 1.0], RK4, 0.005, 20, [(0.4, 0.6)]),
    "ch2d_rk4_mixed": (dict(n=(17, 13), d=(0.7, 1.3), bc=(N, N, F, F, 0, 0), bc_val=(0, 0, 0.3, 0.7, 0, 0)),
                       PHYS_CH, [1.3, 0.5, 2.0, 0.2, 0.8], RK4, 0.002, 15, [(0.3, 0.7)]),
    "ch2d_euler_noflux": (dict(n=(70, 19), bc=(N, N, N, N, 0, 0)), PHYS_CH, [1.0, 0.5, 1.0, 0.0, 1.0], EULER,
                          0.005, 20, [(0.4, 0.6)]),
    "ch3d_rk4": (dict(n=(9, 8, 7)), PHYS_CH, [1.0, 0.5, 1.0, 0.0, 1.0], RK4, 0.002, 8, [(0.4, 0.6)]),
    # config 3 (coupled CH+AC, noflux x, periodic y z) at 10x9x7 and 40x20x19
    "chac3d_rk4": (dict(n=(10, 9, 7), bc=(N, N, P, P, P, P)), PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0], RK4, 0.002,
                   10, [(0.35, 0.45), (0.0, 0.1)]),
    "chac3d_rk4_tiles": (dict(n=(34, 9, 17), bc=(N, N, P, P, P, P)), PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0], RK4,
                         0.002, 3, [(0.3, 0.5), (0.0, 0.2)]),
    "chac3d_euler": (dict(n=(10, 9, 7), bc=(N, N, P, P, P, P)), PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0], EULER, 0.002,
                     10, [(0.35, 0.45), (0.0, 0.1)]),
    "chac2d_rk4": (dict(n=(20, 14), bc=(N, N, P, P, 0, 0)), PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0], RK4, 0.005, 10,
                   [(0.35, 0.45), (0.0, 0.1)]),
}


def make_inputs(name, grid, inits, seed):
    rng = np.random.default_rng(seed)
    out = []
    for lo, hi in inits:
        a = rng.uniform(-3.0, 3.0, size=grid.stored_shape)  # junk ghosts
        grid.phys(a)[...] = rng.uniform(lo, hi, size=grid.phys(a).shape)
        out.append(a)
    return out


def main():
    ref = Reference()
    for seed, (name, (gk, phys, prm, scheme, dt, nsteps, inits)) in enumerate(sorted(CASES.items())):
        grid = Grid(**gk)
        fields = make_inputs(name, grid, inits, seed)
        outs = [f.copy() for f in fields]
        ref.advance(outs, phys, prm, scheme, dt, nsteps, grid, use_gpu=False)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            n=np.array(grid.n), d=np.array(list(grid.d)[:grid.dim]), ghost=grid.ghost,
            bc=np.array(grid.bc), bc_val=np.array(grid.bc_val), phys=phys, prm=np.array(prm), scheme=scheme,
            dt=dt, nsteps=nsteps, inputs=np.stack(fields), outputs=np.stack(outs))
        print(f"{name}: {grid.n} phys={phys} scheme={scheme} steps={nsteps}")
    # the shipped Cahn-Hilliard app's multi-step Euler form (STEADY mu, TRANSIENT c)
    grid = Grid(n=(16, 12))
    c, mu = make_inputs("ch_multistep", grid, [(0.4, 0.6), (0.0, 0.0)], 99)
    c2, mu2 = c.copy(), mu.copy()
    prm = [1.0, 0.5, 1.0, 0.0, 1.0]
    ref.advance_ch_multistep(c2, mu2, prm, 0.005, 20, grid, use_gpu=False)
    np.savez_compressed(os.path.join(HERE, "ch2d_multistep.npz"), n=np.array(grid.n), d=np.array([1.0, 1.0]),
                        ghost=1, bc=np.array(grid.bc), bc_val=np.array(grid.bc_val), prm=np.array(prm), dt=0.005,
                        nsteps=20, inputs=np.stack([c, mu]), outputs=np.stack([c2, mu2]))
    print("ch2d_multistep")


if __name__ == "__main__":
    main()
