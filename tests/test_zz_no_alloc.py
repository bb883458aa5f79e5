"""The allocation-free diagnostics entry point (phix_reduce_mass_energy_noalloc).

It serves callers that cannot allocate device memory: its scratch lives in a
static device array inside the library.  It is called here through the C ABI
and must agree with the allocating entry point (phix_reduce_mass_energy) to
the relative tolerance the other diagnostics tests use, on two calls in a row
(the static scratch keeps the first call's contents, which must not leak into
the second).  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

import phix_b200 as px

TOL = 1e-12  # relative, as in tests/test_gpu_ops.py


def _fields(seed, grid, nf):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nf):
        a = rng.uniform(0.0, 1.0, size=px.stored_shape(grid))
        out.append(torch.from_numpy(a).cuda())
    return out


def _call_noalloc(fields, phys, prm, g):
    """Direct C-ABI call of the allocation-free entry point."""
    lib = px.lib()
    ptrs = (C.c_void_p * len(fields))(*[f.data_ptr() for f in fields])
    prmc = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
    out = (C.c_double * 2)()
    rc = lib.phix_reduce_mass_energy_noalloc(ptrs, phys, prmc, C.byref(g), out, None)
    assert rc == px.OK, lib.phix_last_error()
    return out[0], out[1]


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda):
    cases = [
        (px.PHYS_CH, [1.0, 0.5, 1.0, 0.0, 1.0], px.make_grid((300, 170)), 1),
        (px.PHYS_CHAC, [1.0, 1.0, 0.5, 0.5, 1.0],
         px.make_grid((40, 33, 21), bc=(px.BC_NOFLUX, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_PERIODIC, px.BC_PERIODIC,
                                        px.BC_PERIODIC)), 2),
    ]
    for seed, (phys, prm, g, nf) in enumerate(cases):
        # two calls in a row on the same grid with different fields: the
        # second must not see the first call's rows (stale rows beyond a
        # smaller grid are covered by test_noalloc_second_call_on_smaller_grid)
        for call in range(2):
            fields = _fields(10 * seed + call, g, nf)
            want = px.reduce_mass_energy(fields, phys, prm, g)
            got = _call_noalloc(fields, phys, prm, g)
            for a, b in zip(got, want):
                assert abs(a - b) <= TOL * abs(b), (phys, call, a, b)
            # the Python binding of the same entry point marshals the same call
            wrapped = px.reduce_mass_energy_noalloc(fields, phys, prm, g)
            assert wrapped == got


@pytest.mark.gpu
def test_noalloc_second_call_on_smaller_grid(cuda):
    prm = [1.0, 0.5, 1.0, 0.0, 1.0]
    big, small = px.make_grid((64, 1000)), px.make_grid((50, 7))
    for g, seed in ((big, 1), (small, 2)):
        fields = _fields(seed, g, 1)
        want = px.reduce_mass_energy(fields, px.PHYS_CH, prm, g)
        got = _call_noalloc(fields, px.PHYS_CH, prm, g)
        for a, b in zip(got, want):
            assert abs(a - b) <= TOL * abs(b)


@pytest.mark.gpu
def test_noalloc_flags_non_finite_cells_then_recovers(cuda):
    """One NaN physical cell gives PHIX_ERR_NONFINITE; the next clean call on
    the same (shared) scratch matches the allocating entry point again."""
    prm = [1.0, 0.5, 1.0, 0.0, 1.0]
    g = px.make_grid((96, 80))
    bad = _fields(5, g, 1)
    bad[0][1, 40, 30] = float("nan")  # a physical cell: z plane 1 of the 2-D stored array (ghost 1)
    lib = px.lib()
    ptrs = (C.c_void_p * 1)(bad[0].data_ptr())
    prmc = (C.c_double * 8)(*(prm + [0.0] * 3))
    out = (C.c_double * 2)()
    rc = lib.phix_reduce_mass_energy_noalloc(ptrs, px.PHYS_CH, prmc, C.byref(g), out, None)
    assert rc == px.ERR_NONFINITE
    assert b"non-finite" in lib.phix_last_error()
    with pytest.raises(px.PhixError):
        px.reduce_mass_energy_noalloc(bad, px.PHYS_CH, prm, g)
    clean = _fields(6, g, 1)
    want = px.reduce_mass_energy(clean, px.PHYS_CH, prm, g)
    got = _call_noalloc(clean, px.PHYS_CH, prm, g)
    for a, b in zip(got, want):
        assert abs(a - b) <= TOL * abs(b)


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Checked before any device work, so this runs without a GPU too."""
    lib = px.lib()
    g = px.make_grid((4, 300, 300))  # 90000 rows > PHIX_NOALLOC_MAX_ROWS
    ptrs = (C.c_void_p * 1)(C.c_void_p(16))
    prmc = (C.c_double * 8)(1.0, 0.5, 1.0, 0.0, 1.0, 0, 0, 0)
    out = (C.c_double * 2)()
    rc = lib.phix_reduce_mass_energy_noalloc(ptrs, px.PHYS_CH, prmc, C.byref(g), out, None)
    assert rc == px.ERR_ARG
    assert b"65536" in lib.phix_last_error()
