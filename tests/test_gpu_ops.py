"""Single-operator kernels (phix_bc_apply, phix_lap_accumulate, ...) against the
oracle, bit for bit, on grids that exercise every BC kind and odd sizes; and
the FP64 diagnostics against the oracle's sums."""
import numpy as np
import pytest
import torch

import phix_b200 as px
from oracle.oracle import (BC_FIXED, BC_NONE, BC_NOFLUX, BC_PERIODIC, PHYS_AC, PHYS_CH, PHYS_CHAC, PW_AC, PW_CHAC_C,
                           PW_CHAC_E, PW_DW, PW_IDENT, PW_MUL, Grid)

pytestmark = pytest.mark.gpu

P, N, F, X = BC_PERIODIC, BC_NOFLUX, BC_FIXED, BC_NONE
GRIDS = [
    Grid(n=(37,), d=(0.3,), bc=(N, F, 0, 0, 0, 0), bc_val=(0, 1.5, 0, 0, 0, 0)),
    Grid(n=(33, 17), d=(0.7, 1.3), bc=(P, P, N, F, 0, 0), bc_val=(0, 0, 0, -0.5, 0, 0)),
    Grid(n=(9, 8, 7), d=(1.1, 0.6, 1.7), ghost=2, bc=(F, N, P, P, N, N), bc_val=(0.25, 0, 0, 0, 0, 0)),
]


def pgrid(grid):
    return px.make_grid(grid.n, grid.d[:grid.dim], grid.ghost, grid.bc, grid.bc_val)


def rand(grid, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=grid.stored_shape)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("gi", range(len(GRIDS)))
def test_bc_apply_bitwise(cuda, oracle, gi):
    grid = GRIDS[gi]
    a = rand(grid, gi)
    d = dev(a)
    px.bc_apply(d, pgrid(grid))
    oracle.bc_apply(a, grid)
    assert np.array_equal(d.cpu().numpy(), a)


@pytest.mark.parametrize("gi", range(len(GRIDS)))
def test_lap_grad_bitwise(cuda, oracle, gi):
    grid = GRIDS[gi]
    src, rhs = rand(grid, 10 + gi), rand(grid, 20 + gi)
    dsrc, drhs = dev(src), dev(rhs)
    px.lap_accumulate(drhs, dsrc, -0.37, pgrid(grid))
    oracle.lap_acc(rhs, src, -0.37, grid, fma_mode=1)
    assert np.array_equal(drhs.cpu().numpy(), rhs)
    for axis in range(grid.dim):
        px.grad_accumulate(drhs, dsrc, 1.9, axis, pgrid(grid))
        oracle.grad_acc(rhs, src, 1.9, axis, grid, fma_mode=1)
        assert np.array_equal(drhs.cpu().numpy(), rhs)


@pytest.mark.parametrize("func", [PW_IDENT, PW_AC, PW_DW, PW_CHAC_C, PW_CHAC_E, PW_MUL])
def test_pointwise_and_mul_bitwise(cuda, oracle, func):
    grid = GRIDS[1]
    s1, s2, rhs = rand(grid, 1, 0, 1), rand(grid, 2, 0, 1), rand(grid, 3)
    prm = [1.0, 0.5, 1.7, 0.2, 0.9]
    d1, d2, dr = dev(s1), dev(s2), dev(rhs)
    px.pointwise_accumulate(dr, d1, d2, 0.61, func, prm, pgrid(grid))
    oracle.pw_acc(rhs, s1, s2, 0.61, func, prm, grid, fma_mode=1)
    assert np.array_equal(dr.cpu().numpy(), rhs)
    px.mul_accumulate(dr, d1, d2, -1.3, pgrid(grid))
    oracle.mul_acc(rhs, s1, s2, -1.3, grid, fma_mode=1)
    assert np.array_equal(dr.cpu().numpy(), rhs)


def test_axpy_bitwise(cuda, oracle):
    a, b = rand(GRIDS[2], 5), rand(GRIDS[2], 6)
    da, db = dev(a), dev(b)
    px.axpy(da, db, 0.0123)
    oracle.axpy(a, b, 0.0123, fma_mode=1)
    assert np.array_equal(da.cpu().numpy(), a)


@pytest.mark.parametrize("phys,gi", [(PHYS_AC, 0), (PHYS_CH, 1), (PHYS_CHAC, 2), (PHYS_CH, 2)])
def test_mass_energy_vs_oracle(cuda, oracle, phys, gi):
    grid = GRIDS[gi]
    prm = [1.0, 0.5, 1.0, 0.0, 1.0] if phys != PHYS_CHAC else [1.0, 1.0, 0.5, 0.5, 1.0]
    if phys == PHYS_AC:
        prm = [1.0, 0.8]
    nf = 2 if phys == PHYS_CHAC else 1
    fields = [rand(grid, 40 + f, 0.0, 1.0) for f in range(nf)]
    m, e = px.reduce_mass_energy([dev(a) for a in fields], phys, prm, pgrid(grid))
    m_o = oracle.mass(fields[0], grid)
    e_o = oracle.energy(fields, phys, prm, grid)
    assert abs(m - m_o) <= 1e-12 * abs(m_o)
    assert abs(e - e_o) <= 1e-12 * abs(e_o)


def test_diagnostics_flag_nonfinite(cuda):
    grid = GRIDS[1]
    a = rand(grid, 9)
    grid.phys(a)[0, 3, 4] = np.nan
    with pytest.raises(px.PhixError) as ei:
        px.reduce_mass_energy([dev(a)], PHYS_CH, [1, 0.5, 1, 0, 1], pgrid(grid))
    assert ei.value.code == px.ERR_NONFINITE
