"""The 3-D kernels with TMA plane staging on a B200: the RK4 step in two
launches of two fused stages (include/phix/detail/march3d_fused.cuh) and the
streamed one-stage kernel (include/phix/detail/stream3d.cuh, the default),
against the marching stage kernel and the oracle.

Grids are chosen to hit the kernel's edge cases: partial in-plane tiles, grids
narrower than the four-cell halo, zero-flux and periodic in-plane sides, z
chunks (several CTAs along z) and a single chunk.  Bar: identical bits on
every physical cell (FP64 against the oracle in fma_mode 1 as well; FP32 with
the compensated state against the four-launch FP32 path), and the stepper's
error flag stays clear.
"""
import numpy as np
import pytest
import torch

import phix_b200 as px
from oracle.oracle import Grid

pytestmark = pytest.mark.gpu

CASES = [
    # (phys, n, bc x, bc y)
    (px.PHYS_CHAC, (40, 33, 21), px.BC_NOFLUX, px.BC_PERIODIC),
    (px.PHYS_CH, (64, 48, 40), px.BC_PERIODIC, px.BC_PERIODIC),
    (px.PHYS_CHAC, (37, 20, 50), px.BC_NOFLUX, px.BC_NOFLUX),
    (px.PHYS_CHAC, (96, 17, 12), px.BC_PERIODIC, px.BC_NOFLUX),
    (px.PHYS_CHAC, (6, 5, 9), px.BC_NOFLUX, px.BC_PERIODIC),
    (px.PHYS_CH, (70, 40, 8), px.BC_NOFLUX, px.BC_NOFLUX),
]
PRM = {px.PHYS_CH: [1.0, 0.5, 1.0, 0.0, 1.0], px.PHYS_CHAC: [1.0, 1.0, 0.5, 0.5, 1.0]}
DT = {px.PHYS_CH: 0.002, px.PHYS_CHAC: 0.002}
NSTEPS = 9
MARCH_TILE = 2  # phix_stepper_set_tiles on 3-D grids: the marching stage kernel (no TMA)
STREAM_TILES = (3, 4, 5)  # the streamed stage kernel's tile variants (-1 = variant 0)


def _inputs(phys, n, grid, seed):
    rng = np.random.default_rng(seed)
    shape = (n[2], n[1], n[0])
    f = [grid.stored_from_phys(rng.uniform(0.3, 0.5, size=shape))]
    if phys == px.PHYS_CHAC:
        f.append(grid.stored_from_phys(rng.uniform(0.0, 0.1, size=shape)))
    return f


def _run(phys, g, prec, fields, fused, nsteps=NSTEPS, graph=0, tile=-1):
    st = px.Stepper(phys, px.RK4, prec, PRM[phys], DT[phys], g)
    st.set_fusion(fused)
    st.set_tiles(tile)
    lps = st.launches_per_step
    d = [torch.from_numpy(f.copy()).cuda() for f in fields]
    st.load(d)
    if graph:
        st.set_graph(graph)
    st.advance(nsteps)
    st.store(d)
    torch.cuda.synchronize()
    st.status()
    st.close()
    return [x.cpu().numpy() for x in d], lps


@pytest.mark.parametrize("prec", [px.F64, px.F32], ids=["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[1])))
def test_fused_3d_step_matches_per_stage_launches(cuda, oracle, prec, case):
    phys, n, bx, by = case
    bcs = (bx, bx, by, by, px.BC_PERIODIC, px.BC_PERIODIC)
    g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
    grid = Grid(n=n, bc=bcs)
    fields = _inputs(phys, n, grid, hash(n) % 1000)
    fused, lps_f = _run(phys, g, prec, fields, True)
    staged, lps_s = _run(phys, g, prec, fields, False)               # streamed TMA stage kernel
    marched, _ = _run(phys, g, prec, fields, False, tile=MARCH_TILE)  # marching stage kernel
    assert lps_f == 2 and lps_s == 4  # odd FP64 rows too: the stepper's own arrays are row-padded
    for other in (fused, marched):
        for a, b in zip(other, staged):
            pa, pb = grid.phys(a), grid.phys(b)
            bad = np.argwhere(pa != pb)
            assert bad.size == 0, f"{len(bad)} cells differ, first (z, y, x) {bad[:4].tolist()}"
    if prec == px.F64:
        want = [f.copy() for f in fields]
        grid.fma_mode = 1
        oracle.advance(want, phys, PRM[phys], px.RK4, DT[phys], NSTEPS, grid)
        for a, b in zip(fused, want):
            assert np.array_equal(grid.phys(a), grid.phys(b))


def test_fused_3d_graph_replay_and_ghosts(cuda, oracle):
    """Graph replay gives the same bits, and the final launch writes the
    ghost faces (not corners) the per-stage path writes."""
    phys, n = px.PHYS_CHAC, (48, 36, 24)
    bcs = (px.BC_NOFLUX, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_PERIODIC, px.BC_PERIODIC, px.BC_PERIODIC)
    g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
    grid = Grid(n=n, bc=bcs)
    fields = _inputs(phys, n, grid, 5)
    a, _ = _run(phys, g, px.F64, fields, True, nsteps=12, graph=5)
    b, _ = _run(phys, g, px.F64, fields, False, nsteps=12)
    sh = grid.stored_shape
    faces = np.zeros(sh, dtype=bool)
    faces[1:-1, 1:-1, :] = True
    faces[1:-1, :, 1:-1] = True
    faces[:, 1:-1, 1:-1] = True
    for x, y in zip(a, b):
        assert np.array_equal(x[faces], y[faces])


def test_fused_3d_on_bound_buffers_with_odd_rows_falls_back(cuda):
    """Caller-owned FP64 buffers keep the grid's layout: rows of 39 doubles
    are not whole 16-byte units, so the step runs one launch per stage (same
    bits); an even row length keeps the fused path."""
    for n0, want in ((37, 4), (38, 2)):
        n = (n0, 20, 12)
        bcs = (px.BC_NOFLUX, px.BC_NOFLUX) + (px.BC_PERIODIC,) * 4
        g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
        grid = Grid(n=n, bc=bcs)
        fields = _inputs(px.PHYS_CHAC, n, grid, 3)
        st = px.Stepper(px.PHYS_CHAC, px.RK4, px.F64, PRM[px.PHYS_CHAC], DT[px.PHYS_CHAC], g)
        st.set_fusion(True)  # the fused two-stage launches (one launch per stage is the 3-D default)
        d = [torch.from_numpy(f.copy()).cuda() for f in fields]
        alt = [x.clone() for x in d]
        st.bind(d, alt)
        assert st.launches_per_step == want
        st.advance(4)
        torch.cuda.synchronize()
        st.status()
        got = [(alt if st.current() else d)[f].cpu().numpy() for f in range(2)]
        st.close()
        ref, _ = _run(px.PHYS_CHAC, g, px.F64, fields, False, nsteps=4)
        for a, b in zip(got, ref):
            assert np.array_equal(grid.phys(a), grid.phys(b))


@pytest.mark.parametrize("prec", [px.F64, px.F32], ids=["f64", "f32"])
@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[3]], ids=lambda c: "x".join(map(str, c[1])))
def test_fused_3d_tile_variants_agree(cuda, prec, case):
    """Tile variant 1 (stages 3-4 on 32x8 tiles; FP64 also stages 1-2) gives
    the bits of variant 0."""
    phys, n, bx, by = case
    bcs = (bx, bx, by, by, px.BC_PERIODIC, px.BC_PERIODIC)
    g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
    grid = Grid(n=n, bc=bcs)
    fields = _inputs(phys, n, grid, 17)
    a, _ = _run(phys, g, prec, fields, True, tile=0)
    b, lps = _run(phys, g, prec, fields, True, tile=1)
    assert lps == 2
    for x, y in zip(a, b):
        assert np.array_equal(grid.phys(x), grid.phys(y))


@pytest.mark.parametrize("prec", [px.F64, px.F32], ids=["f64", "f32"])
def test_streamed_3d_euler_and_graph_replay(cuda, oracle, prec):
    """Euler steps and graph-replayed RK4 steps through the streamed stage
    kernel give the marching kernel's bits (FP64: and the oracle's)."""
    phys, n = px.PHYS_CHAC, (40, 24, 18)
    bcs = (px.BC_NOFLUX, px.BC_NOFLUX) + (px.BC_PERIODIC,) * 4
    g = px.make_grid(n, (1.0, 0.9, 1.1), 1, bcs)
    grid = Grid(n=n, d=(1.0, 0.9, 1.1), bc=bcs)
    fields = _inputs(phys, n, grid, 23)
    for scheme, graph in ((px.EULER, 0), (px.RK4, 4)):
        outs = []
        for tile in (-1, MARCH_TILE):
            st = px.Stepper(phys, scheme, prec, PRM[phys], DT[phys], g)
            st.set_tiles(tile)
            d = [torch.from_numpy(f.copy()).cuda() for f in fields]
            st.load(d)
            st.set_graph(graph)
            st.advance(10)
            st.store(d)
            torch.cuda.synchronize()
            st.status()
            st.close()
            outs.append([x.cpu().numpy() for x in d])
        for a, b in zip(*outs):
            assert np.array_equal(grid.phys(a), grid.phys(b)), scheme
        if prec == px.F64:
            want = [f.copy() for f in fields]
            grid.fma_mode = 1
            oracle.advance(want, phys, PRM[phys], scheme, DT[phys], 10, grid)
            for a, b in zip(outs[0], want):
                assert np.array_equal(grid.phys(a), grid.phys(b)), scheme


@pytest.mark.parametrize("prec", [px.F64, px.F32], ids=["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[1])))
def test_streamed_3d_tile_variants_agree(cuda, prec, case):
    """Every tile variant of the streamed stage kernel (TX x TY tiles, R rows
    of a column per thread) gives the marching kernel's bits."""
    phys, n, bx, by = case
    bcs = (bx, bx, by, by, px.BC_PERIODIC, px.BC_PERIODIC)
    g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
    grid = Grid(n=n, bc=bcs)
    fields = _inputs(phys, n, grid, 29)
    ref, _ = _run(phys, g, prec, fields, False, nsteps=5, tile=MARCH_TILE)
    for tile in STREAM_TILES:
        got, lps = _run(phys, g, prec, fields, False, nsteps=5, tile=tile)
        assert lps == 4
        for a, b in zip(got, ref):
            pa, pb = grid.phys(a), grid.phys(b)
            bad = np.argwhere(pa != pb)
            assert bad.size == 0, f"tile {tile}: {len(bad)} cells differ, first (z, y, x) {bad[:4].tolist()}"


@pytest.mark.parametrize("prec", [px.F64, px.F32], ids=["f64", "f32"])
def test_3d_autotune_keeps_state_and_bits(cuda, prec):
    """The autotuner times every 3-D candidate (streamed tile variants, the
    marching kernel, the fused two-stage launches), restores the loaded
    state, and the form it keeps gives the marching kernel's bits."""
    phys, n = px.PHYS_CHAC, (40, 24, 18)
    bcs = (px.BC_NOFLUX, px.BC_NOFLUX) + (px.BC_PERIODIC,) * 4
    g = px.make_grid(n, (1.0, 1.0, 1.0), 1, bcs)
    grid = Grid(n=n, bc=bcs)
    fields = _inputs(phys, n, grid, 31)
    st = px.Stepper(phys, px.RK4, prec, PRM[phys], DT[phys], g)
    d = [torch.from_numpy(f.copy()).cuda() for f in fields]
    st.load(d)
    assert st.autotune(2) > 0
    fused, tile = st.tiles()
    assert st.launches_per_step == (2 if fused else 4)
    assert tile in ((0, 1) if fused else (-1, 2, 4, 5))
    st.advance(6)
    st.store(d)
    torch.cuda.synchronize()
    st.status()
    st.close()
    ref, _ = _run(phys, g, prec, fields, False, nsteps=6, tile=MARCH_TILE)
    for a, b in zip([x.cpu().numpy() for x in d], ref):
        assert np.array_equal(grid.phys(a), grid.phys(b))
