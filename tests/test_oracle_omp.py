"""The OpenMP build of the oracle (oracle/liboracle_omp.so, the timed CPU
baseline on all host cores) gives the same bits as the one-thread oracle:
OpenMP only spreads the per-cell loops, whose arithmetic is unchanged."""
import os

import numpy as np
import pytest

from oracle.oracle import LIB_ORACLE_OMP, PHYS_AC, PHYS_CH, PHYS_CHAC, EULER, RK4, BC_NOFLUX, BC_PERIODIC, Grid, Oracle


@pytest.fixture(scope="module")
def omp():
    if not os.path.exists(LIB_ORACLE_OMP):
        pytest.fail("oracle/liboracle_omp.so not built (make -C oracle)")
    return Oracle(LIB_ORACLE_OMP)


CASES = [
    ("ch2d_rk4", Grid(n=(48, 40)), PHYS_CH, [1.0, 0.5, 1.0, 0.0, 1.0], RK4, 0.005, 30, 1),
    ("ac2d_euler", Grid(n=(64, 64)), PHYS_AC, [1.0, 1.0], EULER, 0.01, 50, 1),
    ("chac3d_rk4", Grid(n=(12, 10, 9), bc=(BC_NOFLUX, BC_NOFLUX) + (BC_PERIODIC,) * 4), PHYS_CHAC,
     [1.0, 1.0, 0.5, 0.5, 1.0], RK4, 0.002, 10, 2),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
@pytest.mark.parametrize("fma_mode", [0, 1])
def test_openmp_oracle_equals_serial_oracle(oracle, omp, case, fma_mode):
    name, grid, phys, prm, scheme, dt, nsteps, nf = case
    grid.fma_mode = fma_mode
    rng = np.random.default_rng(11)
    base = [grid.stored_from_phys(rng.uniform(0.3, 0.7, size=tuple(reversed(grid.n)))) for _ in range(nf)]
    a = [f.copy() for f in base]
    b = [f.copy() for f in base]
    oracle.advance(a, phys, prm, scheme, dt, nsteps, grid)
    omp.advance(b, phys, prm, scheme, dt, nsteps, grid)
    for x, y in zip(a, b):
        assert np.array_equal(grid.phys(x), grid.phys(y))


def test_openmp_oracle_uses_the_host_threads(omp):
    assert omp.threads() == (os.cpu_count() if "OMP_NUM_THREADS" not in os.environ
                             else int(os.environ["OMP_NUM_THREADS"]))
