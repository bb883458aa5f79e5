"""Slab-decomposed stepping (phix_b200.slab): the owned rows of every slab,
after any number of steps and row exchanges, equal the whole-grid run bit for
bit.

* CPU: the slab machinery driven by the oracle (the per-slab engine stands in
  for the GPU stepper, which the CPU cannot run), several slabs in one process
  (LocalExchange) and two or three gloo ranks (DistExchange), against the
  oracle's whole-grid run.  The overlapped sides are poisoned with NaN ghost
  rows, so a row that an exchange misses shows; two negative controls check
  that it does.
* GPU: three slabs on one GPU, each a bound FP64 Stepper, row swaps by copies,
  against the whole-grid Stepper.  (Ranks that exchange over NCCL need one GPU
  each.)
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import phix_b200 as px
from phix_b200 import slab as S

CASES = [
    # (phys, scheme, prm, dt, y boundary, x boundary)
    (px.PHYS_CH, px.RK4, [1.0, 0.5, 1.0, 0.0, 1.0], 0.004, px.BC_PERIODIC, px.BC_PERIODIC),
    (px.PHYS_CH, px.RK4, [1.2, 0.7, 1.5, 0.1, 0.9], 0.003, px.BC_NOFLUX, px.BC_PERIODIC),
    (px.PHYS_CH, px.EULER, [1.0, 0.5, 1.0, 0.0, 1.0], 0.004, px.BC_PERIODIC, px.BC_NOFLUX),
    (px.PHYS_AC, px.EULER, [1.0, 1.0], 0.05, px.BC_NOFLUX, px.BC_PERIODIC),
    (px.PHYS_AC, px.RK4, [1.0, 1.0], 0.05, px.BC_PERIODIC, px.BC_PERIODIC),
]


class OracleEngine:
    """The oracle on one extended slab (a test stand-in for GpuEngine)."""

    def __init__(self, phys, scheme, prm, dt, grid, init):
        from oracle.oracle import Grid, Oracle
        self.o = Oracle()
        self.phys, self.scheme, self.prm, self.dt = phys, scheme, prm, dt
        self.grid = Grid(n=(grid.n[0], grid.n[1]), d=(grid.d[0], grid.d[1]), ghost=1, bc=tuple(grid.bc_type),
                         bc_val=tuple(grid.bc_val))
        self.a = np.ascontiguousarray(init.numpy(), dtype=np.float64)
        self.t = torch.from_numpy(self.a)  # shares the array: row swaps land in it

    def advance(self, k):
        self.o.advance([self.a], self.phys, self.prm, self.scheme, self.dt, k, self.grid, fma_mode=1)

    def state(self):
        return self.t


def _problem(case, n, seed):
    from oracle.oracle import Grid
    phys, scheme, prm, dt, by, bx = case
    bc = (bx, bx, by, by, px.BC_PERIODIC, px.BC_PERIODIC)
    grid = Grid(n=n, d=(1.0, 0.9), bc=bc)
    rng = np.random.default_rng(seed)
    lo, hi = (0.3, 0.7) if phys == px.PHYS_CH else (-0.5, 0.5)
    c = grid.stored_from_phys(rng.uniform(lo, hi, size=(1, n[1], n[0])))
    return grid, c, bc


def _whole(case, grid, c, nsteps):
    from oracle.oracle import Oracle
    phys, scheme, prm, dt, *_ = case
    a = c.copy()
    Oracle().advance([a], phys, prm, scheme, dt, nsteps, grid, fma_mode=1)
    return grid.phys(a)[0]


def _slab_steppers(case, n, c, bc, parts, k, ranks=None, engine="oracle", poison=True, w=None):
    phys, scheme, prm, dt, by, _ = case
    w = S.overlap_for(phys, scheme, k) if w is None else w
    layout = S.slabs(n[1], parts, w, by == px.BC_PERIODIC)
    mine = layout if ranks is None else [layout[r] for r in ranks]
    if engine == "oracle":
        fac = lambda grid, init: OracleEngine(phys, scheme, prm, dt, grid, init)
    else:
        fac = None
    return [S.SlabStepper(phys, scheme, prm, dt, n, sl, torch.from_numpy(c), d=(1.0, 0.9), bc=bc[:4],
                          engine_factory=fac, poison=poison) for sl in mine]


@pytest.mark.parametrize("poison", [True, False])
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_slabs_in_one_process_match_whole_grid(ci, parts, poison):
    """poison=True: NaN ghost rows on the overlapped sides, so a row missed
    by an exchange shows; poison=False: the production side conditions."""
    case = CASES[ci]
    n, nsteps, k = (30, 3 * 26), 11, 3
    if case[1] == px.EULER:
        k = 5
    grid, c, bc = _problem(case, n, 10 + ci)
    steppers = _slab_steppers(case, n, c, bc, parts, k, poison=poison)
    S.run(steppers, S.LocalExchange(steppers), nsteps, k)
    got = np.concatenate([st.owned_rows().numpy() for st in steppers], axis=0)
    want = _whole(case, grid, c, nsteps)
    assert np.array_equal(got, want), f"max-abs {np.abs(got - want).max():.3e}"


@pytest.mark.parametrize("fault", ["no exchange", "overlap one step short"])
def test_poison_reaches_owned_rows_when_the_exchange_falls_short(fault):
    """The check above is sensitive: without the swaps, or with an overlap
    one step too narrow for the exchange interval, NaN reaches owned rows."""
    case = CASES[0]
    n, nsteps, k = (30, 3 * 26), 11, 3
    grid, c, bc = _problem(case, n, 10)
    w = S.overlap_for(case[0], case[1], k) - (S.HALO_PER_STEP[(case[0], case[1])] if fault != "no exchange" else 0)
    steppers = _slab_steppers(case, n, c, bc, 3, k, w=w)
    S.run(steppers, (lambda: None) if fault == "no exchange" else S.LocalExchange(steppers), nsteps, k)
    got = np.concatenate([st.owned_rows().numpy() for st in steppers], axis=0)
    assert np.isnan(got).any()


def test_slab_layout_and_overlap_rules():
    assert S.overlap_for(px.PHYS_CH, px.RK4, 4) == 32 and S.overlap_for(px.PHYS_AC, px.EULER, 3) == 3
    p = S.slabs(100, 3, 8, True)
    assert [(s.y0, s.y1, s.lo, s.hi) for s in p] == [(0, 33, 8, 8), (33, 66, 8, 8), (66, 100, 8, 8)]
    q = S.slabs(100, 3, 8, False)
    assert (q[0].lo, q[0].hi, q[2].lo, q[2].hi) == (0, 8, 8, 0)
    one = S.slabs(64, 1, 8, True)[0]
    assert (one.lo, one.hi, one.ny_ext) == (0, 0, 64)
    with pytest.raises(ValueError):
        S.slabs(20, 3, 8, True)
    with pytest.raises(ValueError):
        S.overlap_for(px.PHYS_CHAC, px.RK4, 1)


# ---- gloo ranks ---------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_worker(rank, world, port, ci, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = CASES[ci]
        n, nsteps, k = (24, 3 * 24), 9, 2
        grid, c, bc = _problem(case, n, 30 + ci)
        st = _slab_steppers(case, n, c, bc, world, k, ranks=[rank])[0]
        S.run([st], S.DistExchange(st, dist), nsteps, k)
        parts = [None] * world
        dist.all_gather_object(parts, st.owned_rows().numpy().copy())
        if rank == 0:
            out.put((np.concatenate(parts, axis=0), _whole(case, grid, c, nsteps)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,ci", [(2, 0), (2, 1), (3, 0), (3, 3)])
def test_slab_ranks_over_gloo_match_whole_grid(world, ci):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, world, port, ci, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got, want = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert np.array_equal(got, want), f"max-abs {np.abs(got - want).max():.3e}"


# ---- GPU ----------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("poison", [True, False])
@pytest.mark.parametrize("ci", [0, 1, 3])
def test_gpu_slabs_match_whole_grid_stepper(cuda, ci, poison):
    case = CASES[ci]
    phys, scheme, prm, dt, by, bx = case
    n, nsteps, k = (200, 3 * 64), 37, 4
    grid, c, bc = _problem(case, n, 50 + ci)
    steppers = _slab_steppers(case, n, c, bc, 3, k, engine="gpu", poison=poison)
    try:
        S.run(steppers, S.LocalExchange(steppers), nsteps, k)
        torch.cuda.synchronize()
        got = np.concatenate([st.owned_rows().cpu().numpy() for st in steppers], axis=0)
    finally:
        for st in steppers:
            st.close()
    g = px.make_grid(n, (1.0, 0.9), 1, bc)
    st = px.Stepper(phys, scheme, px.F64, prm, dt, g)
    t = torch.from_numpy(c.copy()).cuda()
    st.load([t])
    st.advance(nsteps)
    st.store([t])
    torch.cuda.synchronize()
    st.close()
    want = grid.phys(t.cpu().numpy())[0]
    assert np.array_equal(got, want), f"max-abs {np.abs(got - want).max():.3e}"
