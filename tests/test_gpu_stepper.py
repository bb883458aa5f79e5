"""Parity of the fused sm_100a stepper (phix_stepper_*) on a B200.

For every golden case (tests/golden, produced by the reference library's own
CPU path):
  * FP64 kernels vs the oracle in fma_mode 1 (the contracted multiply-adds the
    kernels pin with __fma_rn): identical bits in every stored cell that the
    reference defines (physical cells, ghost faces, untouched padding planes;
    ghost corners excluded, they depend on the order of the BC objects).
  * FP64 kernels vs the reference's CPU vectors: max-abs <= 1e-12 (the two
    differ only by FMA contraction).
  * FP32 kernels vs the FP32 oracle: identical bits on physical cells.
Graph replay, caller-owned buffers (bind) and host buffers (run_host) must
give the same bits as plain launches.
"""
import glob
import os

import numpy as np
import pytest
import torch

import phix_b200 as px
from oracle.oracle import Grid

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if "multistep" not in p)
IDS = [os.path.basename(p)[:-4] for p in CASES]


def load(path):
    z = np.load(path)
    n = tuple(int(v) for v in z["n"])
    d = tuple(float(v) for v in z["d"])
    bc = tuple(int(v) for v in z["bc"])
    bcv = tuple(float(v) for v in z["bc_val"])
    grid = Grid(n=n, d=d, ghost=int(z["ghost"]), bc=bc, bc_val=bcv)
    g = px.make_grid(n, d, int(z["ghost"]), bc, bcv)
    return z, grid, g


def corner_mask(grid):
    """True on cells that lie outside the physical range on 2+ active axes."""
    sh = grid.stored_shape
    gh = grid.ghost
    n0, n1, n2 = grid.n3
    out = np.zeros(sh, dtype=np.int8)
    ranges = [(2, n0), (1, n1), (0, n2)][:grid.dim]
    for axis, n in ranges:
        idx = np.arange(sh[axis])
        o = ((idx < gh) | (idx >= gh + n)).astype(np.int8)
        shape = [1, 1, 1]
        shape[axis] = sh[axis]
        out = out + o.reshape(shape)
    return out >= 2


def _where(a, b, keep):
    """First mismatching stored cells (z, y, x): got / want."""
    bad = np.argwhere((a != b) & keep)
    return f"{len(bad)} cells differ, first: " + ", ".join(
        f"{tuple(int(v) for v in i)} {a[tuple(i)]:.6g}/{b[tuple(i)]:.6g}" for i in bad[:6])


def run_gpu(z, g, precision, graph=0, bind=False, nsteps=None):
    phys, scheme = int(z["phys"]), int(z["scheme"])
    st = px.Stepper(phys, scheme, precision, list(z["prm"]), float(z["dt"]), g)
    fields = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in z["inputs"]]
    n = int(z["nsteps"]) if nsteps is None else nsteps
    if graph:
        st.set_graph(graph)
    if bind:
        alt = [f.clone() for f in fields]
        st.bind(fields, alt)
        st.advance(n)
        torch.cuda.synchronize()
        cur = st.current()
        res = [(alt if cur else fields)[f].cpu().numpy() for f in range(len(fields))]
    else:
        st.load(fields)
        st.advance(n)
        outs = [torch.empty_like(f) for f in fields]
        st.store(outs)
        torch.cuda.synchronize()
        res = [o.cpu().numpy() for o in outs]
    st.close()
    return res


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_fp64_bitwise_vs_oracle_and_close_to_reference(cuda, oracle, path):
    z, grid, g = load(path)
    got = run_gpu(z, g, px.F64)
    want = [np.ascontiguousarray(a) for a in z["inputs"]]
    oracle.advance(want, int(z["phys"]), list(z["prm"]), int(z["scheme"]), float(z["dt"]), int(z["nsteps"]),
                   grid, fma_mode=1)
    keep = ~corner_mask(grid)
    for a, b, r in zip(got, want, z["outputs"]):
        assert np.array_equal(a[keep], b[keep]), f"kernel vs oracle max diff {np.abs(a - b)[keep].max()}"
        assert np.abs(grid.phys(a) - grid.phys(r)).max() <= 1e-12


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_fp32_bitwise_vs_fp32_oracle(cuda, oracle, path):
    """FP32 stencils with the compensated (hi + lo) FP32 state."""
    z, grid, g = load(path)
    got = run_gpu(z, g, px.F32)
    x = [np.ascontiguousarray(a) for a in z["inputs"]]
    hi = [a.astype(np.float32) for a in x]
    lo = [(a - h.astype(np.float64)).astype(np.float32) for a, h in zip(x, hi)]
    oracle.advance_comp(hi, lo, int(z["phys"]), list(z["prm"]), int(z["scheme"]), float(z["dt"]),
                        int(z["nsteps"]), grid, fma_mode=1)
    want = [h.astype(np.float64) + l.astype(np.float64) for h, l in zip(hi, lo)]
    for a, b, r in zip(got, want, z["outputs"]):
        pa, pb = grid.phys(a), grid.phys(b)
        assert np.array_equal(pa, pb), f"max diff {np.abs(pa - pb).max()}"
        # and FP32 stays close to the FP64 reference on these short runs
        assert np.abs(pa - grid.phys(r)).max() < 1e-4


@pytest.mark.parametrize("path", [p for p in CASES if "ch2d_rk4.npz" in p or "chac3d_rk4.npz" in p
                                  or "ac2d_euler" in p])
def test_graph_and_bind_paths_identical(cuda, path):
    z, grid, g = load(path)
    base = run_gpu(z, g, px.F64)
    for graph, bind in ((3, False), (4, False), (0, True), (5, True)):
        other = run_gpu(z, g, px.F64, graph=graph, bind=bind)
        for a, b in zip(base, other):
            assert np.array_equal(grid.phys(a), grid.phys(b)), (graph, bind)


def test_run_host_matches_device_path(cuda):
    z, grid, g = load(os.path.join(GOLDEN, "ch2d_rk4.npz"))
    base = run_gpu(z, g, px.F64)
    st = px.Stepper(int(z["phys"]), int(z["scheme"]), px.F64, list(z["prm"]), float(z["dt"]), g)
    hin = [np.ascontiguousarray(a) for a in z["inputs"]]
    hout = [np.empty_like(a) for a in hin]
    st.run_host(hin, hout, int(z["nsteps"]))
    st.close()
    assert np.array_equal(grid.phys(hout[0]), grid.phys(base[0]))


def test_zero_steps_is_identity(cuda):
    z, grid, g = load(os.path.join(GOLDEN, "chac3d_rk4.npz"))
    got = run_gpu(z, g, px.F64, nsteps=0)
    for a, b in zip(got, z["inputs"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("fused", [True, False])
def test_launch_counter_counts_stage_kernels(cuda, fused):
    z, grid, g = load(os.path.join(GOLDEN, "ch2d_rk4.npz"))
    st = px.Stepper(px.PHYS_CH, px.RK4, px.F64, list(z["prm"]), float(z["dt"]), g)
    st.set_fusion(fused)
    assert st.launches_per_step == (1 if fused else 4)
    f = [torch.from_numpy(np.ascontiguousarray(z["inputs"][0])).cuda()]
    st.load(f)
    st.advance(1)  # the first step after a load also fills every ghost layer once
    torch.cuda.synchronize()
    before = px.launch_count()
    st.advance(7)
    torch.cuda.synchronize()
    assert px.launch_count() - before == 7 * st.launches_per_step
    st.close()


FUSED_CASES = [
    # (phys, n, bc x, bc y, d)
    (px.PHYS_CH, (70, 37), px.BC_PERIODIC, px.BC_PERIODIC, (1.0, 1.0)),
    (px.PHYS_CH, (130, 47), px.BC_NOFLUX, px.BC_PERIODIC, (0.9, 1.1)),
    (px.PHYS_CH, (64, 16), px.BC_PERIODIC, px.BC_NOFLUX, (1.0, 1.0)),
    (px.PHYS_CH, (9, 30), px.BC_NOFLUX, px.BC_NOFLUX, (1.0, 1.0)),
    (px.PHYS_AC, (200, 33), px.BC_PERIODIC, px.BC_PERIODIC, (1.0, 0.7)),
    (px.PHYS_AC, (66, 65), px.BC_NOFLUX, px.BC_NOFLUX, (1.0, 1.0)),
    (px.PHYS_CH, (300, 170), px.BC_PERIODIC, px.BC_PERIODIC, (1.0, 0.8)),
]

# one-launch step tiles: 0-5 the box kernel, 6-15 the pair kernel (CH with
# four periodic sides), 16-19 the pair kernel two steps per launch; those
# that do not fit in shared memory per precision
STEP_TILES = {px.F64: (0, 1, 2, 3, 7, 8, 9, 10, 11, 13, 14, 15, 16, 17, 18, 19), px.F32: tuple(range(20))}
PAIR_TILES = set(range(6, 20))
DEPTH2_TILES = set(range(16, 20))


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("case", range(len(FUSED_CASES)))
def test_one_launch_step_matches_per_stage_launches(cuda, oracle, prec, case):
    """The four-stages-in-one-launch RK4 step gives the bits of the per-stage
    kernels (and, in FP64, of the oracle) on every stored cell but the ghost
    corners, for periodic and zero-flux sides, odd sizes and partial tiles."""
    phys, n, bx, by, d = FUSED_CASES[case]
    bcs = (bx, bx, by, by, 0, 0)
    g = px.make_grid(n, d, 1, bcs)
    grid = Grid(n=n, d=d, bc=bcs, bc_val=(0,) * 6)
    rng = np.random.default_rng(100 + case)
    lo_hi = (0.3, 0.7) if phys == px.PHYS_CH else (-0.6, 0.6)
    x = grid.stored_from_phys(rng.uniform(*lo_hi, size=(1, n[1], n[0])))
    prm = [1.0, 0.6, 1.2, 0.05, 0.95] if phys == px.PHYS_CH else [0.8, 1.3]
    dt = 0.004 if phys == px.PHYS_CH else 0.02
    outs = []
    for fused in (True, False):
        st = px.Stepper(phys, px.RK4, prec, prm, dt, g)
        st.set_fusion(fused)
        assert st.launches_per_step == (1 if fused else 4)
        t = torch.from_numpy(x.copy()).cuda()
        st.load([t])
        st.set_graph(3)
        st.advance(11)
        st.store([t])
        torch.cuda.synchronize()
        st.close()
        outs.append(t.cpu().numpy())
    keep = ~corner_mask(grid)
    assert np.array_equal(outs[0][keep], outs[1][keep])
    if prec == px.F64:
        want = [x.copy()]
        oracle.advance(want, phys, prm, px.RK4, dt, 11, grid, fma_mode=1)
        assert np.array_equal(outs[0][keep], want[0][keep])


def test_multistep_ch_matches_oracle_and_reference(cuda, oracle):
    """Fused multi-step Euler CH (the shipped app's form): c and mu vs the
    oracle bit for bit, and vs the reference's CPU vectors."""
    z, grid, g = load(os.path.join(GOLDEN, "ch2d_multistep.npz"))
    c_in, mu_in = [np.ascontiguousarray(a) for a in z["inputs"]]
    st = px.Stepper(px.PHYS_CH, px.MULTISTEP, px.F64, list(z["prm"]), float(z["dt"]), g)
    fields = [torch.from_numpy(c_in.copy()).cuda(), torch.from_numpy(mu_in.copy()).cuda()]
    st.load(fields)
    st.advance(int(z["nsteps"]))
    outs = [torch.empty_like(f) for f in fields]
    st.store(outs)
    torch.cuda.synchronize()
    st.close()
    c_o, mu_o = c_in.copy(), mu_in.copy()
    oracle.advance_ch_multistep(c_o, mu_o, list(z["prm"]), float(z["dt"]), int(z["nsteps"]), grid, fma_mode=1)
    keep = ~corner_mask(grid)
    got_c, got_mu = outs[0].cpu().numpy(), outs[1].cpu().numpy()
    assert np.array_equal(got_c[keep], c_o[keep]), _where(got_c, c_o, keep)
    assert np.array_equal(got_mu[keep], mu_o[keep]), _where(got_mu, mu_o, keep)
    assert np.abs(got_c - z["outputs"][0])[keep].max() <= 1e-12


@pytest.mark.parametrize("bc", [px.BC_NOFLUX, px.BC_FIXED])
def test_multistep_ch_multi_tile_bcs(cuda, oracle, bc):
    n = (150, 37)
    bcs = (bc, bc, px.BC_PERIODIC, px.BC_PERIODIC, 0, 0)
    bcv = (0.3, 0.6, 0, 0, 0, 0)
    g = px.make_grid(n, (0.9, 1.1), 1, bcs, bcv)
    grid = Grid(n=n, d=(0.9, 1.1), bc=bcs, bc_val=bcv)
    rng = np.random.default_rng(21)
    c = grid.stored_from_phys(rng.uniform(0.3, 0.7, size=(1, 37, 150)))
    mu = np.zeros_like(c)
    prm = [1.2, 0.7, 1.5, 0.1, 0.9]
    st = px.Stepper(px.PHYS_CH, px.MULTISTEP, px.F64, prm, 0.002, g)
    fields = [torch.from_numpy(c.copy()).cuda(), torch.from_numpy(mu.copy()).cuda()]
    alt = [torch.zeros_like(fields[0]), torch.zeros_like(fields[1])]
    alt[0].copy_(fields[0])
    st.bind(fields, alt)
    st.advance(9)
    torch.cuda.synchronize()
    got_c = (alt[0] if st.current() else fields[0]).cpu().numpy()
    got_mu = fields[1].cpu().numpy()
    st.close()
    oracle.advance_ch_multistep(c, mu, prm, 0.002, 9, grid, fma_mode=1)
    keep = ~corner_mask(grid)
    assert np.array_equal(got_c[keep], c[keep]), _where(got_c, c, keep)
    assert np.array_equal(got_mu[keep], mu[keep]), _where(got_mu, mu, keep)


MS_PAIR_TILES = range(6)  # tile shapes of the multi-step pair kernel (kMsCfgs)


@pytest.mark.parametrize("tile", MS_PAIR_TILES)
@pytest.mark.parametrize("n", [(150, 37), (64, 32), (300, 170)])
def test_multistep_pair_tiles_match_oracle(cuda, oracle, n, tile):
    """The multi-step pair kernel (four periodic sides) with every tile shape:
    c and mu bit for bit against the oracle, partial tiles included."""
    bcs = (px.BC_PERIODIC,) * 4 + (0, 0)
    g = px.make_grid(n, (0.9, 1.1), 1, bcs)
    grid = Grid(n=n, d=(0.9, 1.1), bc=bcs, bc_val=(0,) * 6)
    rng = np.random.default_rng(31 + tile)
    c = grid.stored_from_phys(rng.uniform(0.3, 0.7, size=(1, n[1], n[0])))
    mu = np.zeros_like(c)
    prm = [1.2, 0.7, 1.5, 0.1, 0.9]
    st = px.Stepper(px.PHYS_CH, px.MULTISTEP, px.F64, prm, 0.002, g)
    st.set_tiles(tile)
    assert st.tiles() == (True, tile) and st.launches_per_step == 1
    fields = [torch.from_numpy(c.copy()).cuda(), torch.from_numpy(mu.copy()).cuda()]
    st.load(fields)
    st.advance(9)
    st.store(fields)
    torch.cuda.synchronize()
    st.close()
    oracle.advance_ch_multistep(c, mu, prm, 0.002, 9, grid, fma_mode=1)
    keep = ~corner_mask(grid)
    got_c, got_mu = fields[0].cpu().numpy(), fields[1].cpu().numpy()
    assert np.array_equal(got_c[keep], c[keep]), _where(got_c, c, keep)
    assert np.array_equal(got_mu[keep], mu[keep]), _where(got_mu, mu, keep)


@pytest.mark.parametrize("prec", [px.F32, px.F64])
def test_multistep_pair_matches_stage_box_and_autotune(cuda, prec):
    """FP32 and FP64: the multi-step pair kernel and stage_box (one launch per
    step switched off) give the same bits; autotuning restores the loaded c
    and mu and keeps those bits."""
    n = (200, 90)
    bcs = (px.BC_PERIODIC,) * 4 + (0, 0)
    g = px.make_grid(n, (1.0, 1.0), 1, bcs)
    grid = Grid(n=n, d=(1.0, 1.0), bc=bcs, bc_val=(0,) * 6)
    c = grid.stored_from_phys(np.random.default_rng(8).uniform(0.35, 0.65, size=(1, n[1], n[0])))
    prm = [1.0, 0.5, 1.0, 0.0, 1.0]
    outs = []
    for mode in ("box", "pair", "tuned"):
        st = px.Stepper(px.PHYS_CH, px.MULTISTEP, prec, prm, 0.005, g)
        fields = [torch.from_numpy(c.copy()).cuda(), torch.from_numpy(np.zeros_like(c)).cuda()]
        st.load(fields)
        if mode == "box":
            st.set_fusion(False)
            assert st.tiles()[0] is False
        elif mode == "tuned":
            before = [torch.empty_like(f) for f in fields]
            st.advance(3)
            st.store(before)
            assert st.autotune(2) > 0
            after = [torch.empty_like(f) for f in fields]
            st.store(after)
            for b, a in zip(before, after):
                assert torch.equal(b, a)
        else:
            assert st.tiles()[0] is True
        st.advance(12 if mode != "tuned" else 9)
        st.store(fields)
        torch.cuda.synchronize()
        st.close()
        outs.append([f.cpu().numpy() for f in fields])
    keep = ~corner_mask(grid)
    for other in outs[1:]:
        for f in range(2):
            assert np.array_equal(other[f][keep], outs[0][f][keep]), _where(other[f], outs[0][f], keep)


TILE_CASES = [
    # (phys, n, bcs, bc values)
    (px.PHYS_CH, (300, 70), (px.BC_PERIODIC,) * 4, (0,) * 4),
    (px.PHYS_CH, (131, 45), (px.BC_NOFLUX, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_PERIODIC), (0,) * 4),
    (px.PHYS_CH, (70, 37), (px.BC_FIXED, px.BC_FIXED, px.BC_NOFLUX, px.BC_NOFLUX), (0.3, 0.6, 0, 0)),
    (px.PHYS_AC, (129, 33), (px.BC_PERIODIC, px.BC_PERIODIC, px.BC_NONE, px.BC_NONE), (0,) * 4),
    (px.PHYS_CHAC, (140, 66), (px.BC_NOFLUX, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_PERIODIC), (0,) * 4),
]


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("case", range(len(TILE_CASES)))
def test_stage_tile_shapes_give_identical_bits(cuda, oracle, prec, case):
    """Every 2-D stage tile shape (column-walking 0..3, generic box -1), with
    one launch per stage, gives the same bits; FP64 equals the oracle."""
    phys, n, bc4, bv4 = TILE_CASES[case]
    bcs, bcv = tuple(bc4) + (0, 0), tuple(bv4) + (0, 0)
    d = (1.0, 0.9)
    g = px.make_grid(n, d, 1, bcs, bcv)
    grid = Grid(n=n, d=d, bc=bcs, bc_val=bcv)
    rng = np.random.default_rng(200 + case)
    nf = px.NFIELDS[phys]
    lo_hi = (-0.6, 0.6) if phys == px.PHYS_AC else (0.3, 0.7)
    xs = [grid.stored_from_phys(rng.uniform(*lo_hi, size=(1, n[1], n[0]))) for _ in range(nf)]
    prm = {px.PHYS_CH: [1.0, 0.6, 1.2, 0.05, 0.95], px.PHYS_AC: [0.8, 1.3],
           px.PHYS_CHAC: [1.0, 0.9, 0.5, 0.7, 1.1]}[phys]
    dt = 0.02 if phys == px.PHYS_AC else 0.003
    outs = {}
    for tile in (-1, 0, 1, 2, 3):
        st = px.Stepper(phys, px.RK4, prec, prm, dt, g)
        st.set_fusion(False)
        st.set_tiles(tile)
        ts = [torch.from_numpy(x.copy()).cuda() for x in xs]
        st.load(ts)
        st.advance(6)
        st.store(ts)
        torch.cuda.synchronize()
        st.close()
        outs[tile] = [t.cpu().numpy() for t in ts]
    keep = ~corner_mask(grid)
    for tile in (0, 1, 2, 3):
        for a, b in zip(outs[tile], outs[-1]):
            assert np.array_equal(a[keep], b[keep]), (tile, _where(a, b, keep))
    if prec == px.F64:
        want = [x.copy() for x in xs]
        oracle.advance(want, phys, prm, px.RK4, dt, 6, grid, fma_mode=1)
        for a, b in zip(outs[0], want):
            assert np.array_equal(a[keep], b[keep]), _where(a, b, keep)


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("case", [0, 1, 5, 6])
def test_one_launch_step_tile_shapes(cuda, prec, case):
    """Every tile shape of the one-launch RK4 step gives the per-stage bits
    (the pair kernels on the CH grids with four periodic sides)."""
    phys, n, bx, by, d = FUSED_CASES[case]
    bcs = (bx, bx, by, by, 0, 0)
    g = px.make_grid(n, d, 1, bcs)
    grid = Grid(n=n, d=d, bc=bcs, bc_val=(0,) * 6)
    rng = np.random.default_rng(300 + case)
    lo_hi = (0.3, 0.7) if phys == px.PHYS_CH else (-0.6, 0.6)
    x = grid.stored_from_phys(rng.uniform(*lo_hi, size=(1, n[1], n[0])))
    prm = [1.0, 0.6, 1.2, 0.05, 0.95] if phys == px.PHYS_CH else [0.8, 1.3]
    dt = 0.004 if phys == px.PHYS_CH else 0.02
    outs = {}
    pair_ok = phys == px.PHYS_CH and bx == by == px.BC_PERIODIC
    tiles = ((False, -1), (True, -1)) + tuple(
        (True, t) for t in STEP_TILES[prec] if pair_ok or t not in PAIR_TILES)
    for fused, tile in tiles:
        st = px.Stepper(phys, px.RK4, prec, prm, dt, g)
        st.set_fusion(fused)
        st.set_tiles(tile)
        t = torch.from_numpy(x.copy()).cuda()
        st.load([t])
        st.advance(7)
        st.store([t])
        torch.cuda.synchronize()
        st.close()
        outs[(fused, tile)] = t.cpu().numpy()
    keep = ~corner_mask(grid)
    base = outs[(False, -1)]
    for key, a in outs.items():
        assert np.array_equal(a[keep], base[keep]), (key, _where(a, base, keep))


def test_pair_step_tiles_need_periodic_ch(cuda):
    g = px.make_grid((64, 40), bc=(px.BC_NOFLUX,) * 2 + (px.BC_PERIODIC,) * 4)
    st = px.Stepper(px.PHYS_CH, px.RK4, px.F32, [1.0, 0.6, 1.2, 0.05, 0.95], 0.004, g)
    st.set_fusion(True)
    st.set_tiles(7)
    t = torch.full(px.stored_shape(g), 0.5, dtype=torch.float64, device="cuda")
    st.load([t])
    with pytest.raises(px.PhixError):
        st.advance(1)
    st.close()


@pytest.mark.parametrize("prec", [px.F64, px.F32])
def test_autotune_restores_state_and_keeps_bits(cuda, prec):
    """Autotuning leaves the loaded state as it was, and the launch form and
    tile it keeps give the per-stage bits."""
    phys, n, bx, by, d = FUSED_CASES[6]
    bcs = (bx, bx, by, by, 0, 0)
    g = px.make_grid(n, d, 1, bcs)
    grid = Grid(n=n, d=d, bc=bcs, bc_val=(0,) * 6)
    x = grid.stored_from_phys(np.random.default_rng(77).uniform(0.3, 0.7, size=(1, n[1], n[0])))
    prm, dt = [1.0, 0.6, 1.2, 0.05, 0.95], 0.004
    outs, loaded = [], []
    for tune in (False, True):
        st = px.Stepper(phys, px.RK4, prec, prm, dt, g)
        t = torch.from_numpy(x.copy()).cuda()
        st.load([t])
        if tune:
            assert st.autotune(2) > 0
            fused, tile = st.tiles()
            assert st.launches_per_step == (1 if fused else 4)
        else:
            st.set_fusion(False)
        back = torch.empty_like(t)
        st.store([back])  # FP32: the compensated pair of x, as loaded
        st.advance(6)
        st.store([t])
        torch.cuda.synchronize()
        st.close()
        loaded.append(back.cpu().numpy())
        outs.append(t.cpu().numpy())
    keep = ~corner_mask(grid)
    assert np.array_equal(loaded[0][keep], loaded[1][keep])
    assert np.array_equal(outs[0][keep], outs[1][keep]), _where(outs[1], outs[0], keep)


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("tile", sorted(DEPTH2_TILES))
@pytest.mark.parametrize("nsteps,graph", [(11, 0), (12, 5), (9, 4)])
def test_temporal_blocking_depth2_matches_single_steps(cuda, oracle, prec, tile, nsteps, graph):
    """Two RK4 steps per launch (the first step's update kept in shared
    memory on the tile + 8) give the bits of one launch per step, for odd
    step counts (a single-step launch finishes), graph groups of either
    parity, partial tiles and grids smaller than the 16-cell halo; the ghost
    faces equal the single-step path's."""
    n = (150, 37) if tile != 19 else (13, 20)
    g = px.make_grid(n, (1.0, 0.9), 1)
    grid = Grid(n=n, d=(1.0, 0.9))
    rng = np.random.default_rng(7 + tile)
    x = grid.stored_from_phys(rng.uniform(0.3, 0.7, size=(1, n[1], n[0])))
    prm = [1.0, 0.6, 1.2, 0.05, 0.95]
    outs, launches = [], []
    for t in (tile, -1):
        st = px.Stepper(px.PHYS_CH, px.RK4, prec, prm, 0.004, g)
        st.set_tiles(t)
        assert st.depth == (2 if t == tile else 1)
        d = torch.from_numpy(x.copy()).cuda()
        st.load([d])
        st.set_graph(graph)
        before = px.launch_count()
        st.advance(nsteps)
        torch.cuda.synchronize()
        launches.append(px.launch_count() - before)
        st.store([d])
        torch.cuda.synchronize()
        st.close()
        outs.append(d.cpu().numpy())
    # the single-step run: the first step's BC fills plus one launch per step;
    # depth 2 pairs the steps of each graph group (an odd group or remainder
    # ends with a single-step launch)
    pairs = lambda k: k // 2 + k % 2
    want = pairs(nsteps) if not graph else (nsteps // graph) * pairs(graph) + pairs(nsteps % graph)
    assert launches[0] == launches[1] - nsteps + want
    keep = ~corner_mask(grid)
    assert np.array_equal(outs[0][keep], outs[1][keep])
    if prec == px.F64:
        want = [x.copy()]
        oracle.advance(want, px.PHYS_CH, prm, px.RK4, 0.004, nsteps, grid, fma_mode=1)
        assert np.array_equal(outs[0][keep], want[0][keep])
