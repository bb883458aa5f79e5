"""Batched engine (phix_batch_*): every instance of a batch of uneven grids
and parameters must produce exactly the bits of the single-field stepper run
on that instance alone (same kernels, same arithmetic), for every tile shape;
per-instance FP64 mass matches the reduction of the single-field path."""
import numpy as np
import pytest
import torch

import phix_b200 as px
from phix_b200 import workloads

pytestmark = pytest.mark.gpu


def small_batch(prec):
    grids, phys, prms, scheme, dt, _, fields = workloads.ch2d_batch(ninst=7, seed=11, sizes=(16, 40, 64, 96, 130))
    # one zero-flux instance and one odd-sized one, to cover the BC paths
    grids[1] = px.make_grid((40, 40), bc=(px.BC_NOFLUX,) * 6)
    f1 = np.zeros(px.stored_shape(grids[1]))
    f1[1, 1:41, 1:41] = 0.5 + np.random.default_rng(4).uniform(-0.05, 0.05, size=(40, 40))
    fields[1] = f1
    grids[3] = px.make_grid((70, 37))
    g3 = grids[3]
    f3 = np.zeros(px.stored_shape(g3))
    f3[1, 1:38, 1:71] = 0.5 + np.random.default_rng(5).uniform(-0.05, 0.05, size=(37, 70))
    fields[3] = f3
    return grids, phys, prms, scheme, dt, fields


def single(g, phys, prm, scheme, dt, field, nsteps, prec):
    st = px.Stepper(phys, scheme, prec, prm, dt, g)
    d = torch.from_numpy(field.copy()).cuda()
    st.load([d])
    st.advance(nsteps)
    st.store([d])
    torch.cuda.synchronize()
    st.close()
    return d.cpu().numpy()


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("cfg", range(6))
def test_batch_matches_single_field_stepper(cuda, prec, cfg):
    grids, phys, prms, scheme, dt, fields = small_batch(prec)
    b = px.Batch(phys, scheme, prec, grids, prms, dt)
    b.set_fusion(False)  # one launch per stage, with this tile shape
    assert b.launches_per_step == 4
    b.set_tiles(cfg, 0)
    for i, f in enumerate(fields):
        b.load(i, f)
    b.set_graph(3 if cfg % 2 else 0)
    nsteps = 7
    b.advance(nsteps)
    torch.cuda.synchronize()
    for i, (g, prm, f) in enumerate(zip(grids, prms, fields)):
        out = np.empty_like(f)
        b.store(i, out)
        want = single(g, phys, prm, scheme, dt, f, nsteps, prec)
        gh = g.ghost
        sl = (slice(gh, gh + g.n[2]), slice(gh, gh + g.n[1]), slice(gh, gh + g.n[0]))
        assert np.array_equal(out[sl], want[sl]), (cfg, i)
    b.close()


def test_batch_mass_and_autotune(cuda):
    grids, phys, prms, scheme, dt, fields = small_batch(px.F32)
    b = px.Batch(phys, scheme, px.F32, grids, prms, dt)
    for i, f in enumerate(fields):
        b.load(i, f)
    m0 = b.mass()
    ms = b.autotune(2)
    assert ms > 0
    assert b.mass() == m0  # autotuning leaves the state untouched
    b.advance(50)
    m1 = b.mass()
    for i, g in enumerate(grids):
        d = torch.from_numpy(fields[i]).cuda()
        ref, _ = px.reduce_mass_energy([d], phys, prms[i], g)
        assert abs(m0[i] - ref) <= 1e-6 * abs(ref)  # FP32 state vs FP64 input
        assert abs(m1[i] - m0[i]) <= 1e-5 * abs(m0[i])
    b.close()


@pytest.mark.parametrize("prec", [px.F64, px.F32])
@pytest.mark.parametrize("graph", [0, 3])
@pytest.mark.parametrize("all_periodic", [False, True])
def test_batch_one_launch_step_matches_single_field_stepper(cuda, prec, graph, all_periodic):
    """One launch per RK4 step over the whole batch gives each instance the
    bits of the single-field stepper (the pair kernels when every instance
    is periodic, the cell-per-thread kernel with a zero-flux instance)."""
    grids, phys, prms, scheme, dt, fields = small_batch(prec)
    if all_periodic:
        grids[1] = px.make_grid((40, 40))
    b = px.Batch(phys, scheme, prec, grids, prms, dt)
    assert b.launches_per_step == 1  # the default where every side allows it
    b.set_fusion(False)
    assert b.launches_per_step == 4
    b.set_fusion(True)
    assert b.launches_per_step == 1
    for i, f in enumerate(fields):
        b.load(i, f)
    b.set_graph(graph)
    nsteps = 7
    before = px.launch_count()
    b.advance(nsteps)
    torch.cuda.synchronize()
    assert px.launch_count() - before == nsteps
    for i, (g, prm, f) in enumerate(zip(grids, prms, fields)):
        out = np.empty_like(f)
        b.store(i, out)
        want = single(g, phys, prm, scheme, dt, f, nsteps, prec)
        gh = g.ghost
        sl = (slice(gh, gh + g.n[2]), slice(gh, gh + g.n[1]), slice(gh, gh + g.n[0]))
        assert np.array_equal(out[sl], want[sl]), i
    b.close()


def test_batch_one_launch_step_needs_periodic_or_noflux_sides(cuda):
    grids, phys, prms, scheme, dt, fields = small_batch(px.F32)
    grids[2] = px.make_grid((grids[2].n[0], grids[2].n[1]), bc=(px.BC_FIXED,) * 4 + (px.BC_PERIODIC,) * 2)
    b = px.Batch(phys, scheme, px.F32, grids, prms, dt)
    assert b.launches_per_step == 4
    with pytest.raises(px.PhixError):
        b.set_fusion(True)
    b.set_fusion(False)
    assert b.launches_per_step == 4
    b.close()


@pytest.mark.parametrize("prec", [px.F64, px.F32])
def test_batch_temporal_blocking_depth2(cuda, prec):
    """Two RK4 steps per launch over the whole batch (pair kernels, every
    instance periodic) give each instance the bits of the single-field
    stepper, with an odd step count and graph replay."""
    grids, phys, prms, scheme, dt, fields = small_batch(prec)
    grids[1] = px.make_grid((40, 40))
    b = px.Batch(phys, scheme, prec, grids, prms, dt)
    b.set_fusion(True)
    b.set_depth(2)
    assert b.depth == 2
    for i, f in enumerate(fields):
        b.load(i, f)
    b.set_graph(4)
    nsteps = 9
    before = px.launch_count()
    b.advance(nsteps)
    torch.cuda.synchronize()
    assert px.launch_count() - before == nsteps // 2 + 1
    for i, (g, prm, f) in enumerate(zip(grids, prms, fields)):
        out = np.empty_like(f)
        b.store(i, out)
        want = single(g, phys, prm, scheme, dt, f, nsteps, prec)
        gh = g.ghost
        sl = (slice(gh, gh + g.n[2]), slice(gh, gh + g.n[1]), slice(gh, gh + g.n[0]))
        assert np.array_equal(out[sl], want[sl]), i
    b.close()


def test_batch_depth2_needs_the_pair_kernels(cuda):
    grids, phys, prms, scheme, dt, fields = small_batch(px.F32)  # one zero-flux instance
    b = px.Batch(phys, scheme, px.F32, grids, prms, dt)
    with pytest.raises(px.PhixError):
        b.set_depth(2)
    assert b.depth == 1
    b.close()
