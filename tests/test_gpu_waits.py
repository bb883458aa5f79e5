"""Bounded device-side waits: the give-up path returns an error status.

The tensor-core kernels wait on mbarriers with a wall-clock limit and, when a
wait gives up, set a device error flag and return.  phix_wait_selftest runs
that same wait (tc::mbar_wait_bounded) on a barrier of count 1 in one thread,
with or without the arrival.  Without it nothing ever completes the barrier:
the wait must run out after the given limit, the call must return
PHIX_ERR_TIMEOUT, and the context must stay usable for the next kernels.
Nothing here faults: no UMMA or TMEM is in flight when the wait gives up.
"""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import phix_b200 as px

pytestmark = pytest.mark.gpu


def test_bounded_wait_completes_when_the_barrier_completes(cuda):
    assert px.lib().phix_wait_selftest(1, 1.0, None) == px.OK


def test_bounded_wait_gives_up_and_reports_timeout(cuda):
    lib = px.lib()
    limit = 0.05
    t0 = time.perf_counter()
    rc = lib.phix_wait_selftest(0, C.c_double(limit), None)
    el = time.perf_counter() - t0
    assert rc == px.ERR_TIMEOUT
    assert b"gave up" in lib.phix_last_error()
    assert limit <= el < 2.0, el
    # the context is still usable: a stepper runs and agrees with itself
    g = px.make_grid((64, 64))
    rng = np.random.default_rng(0)
    a = np.zeros(px.stored_shape(g))
    a[1, 1:65, 1:65] = 0.5 + rng.uniform(-0.01, 0.01, size=(64, 64))
    outs = []
    for _ in range(2):
        st = px.Stepper(px.PHYS_CH, px.RK4, px.F64, [1.0, 0.5, 1.0, 0.0, 1.0], 0.005, g)
        d = [torch.from_numpy(a.copy()).cuda()]
        st.load(d)
        st.advance(10)
        st.store(d)
        torch.cuda.synchronize()
        st.close()
        outs.append(d[0].cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.isfinite(outs[0]).all()


def test_wait_selftest_rejects_limits_outside_range(cuda):
    lib = px.lib()
    assert lib.phix_wait_selftest(0, C.c_double(0.0), None) == px.ERR_ARG
    assert lib.phix_wait_selftest(0, C.c_double(3.0), None) == px.ERR_ARG


def test_surrogate_status_is_clean_after_normal_steps(cuda):
    from phix_b200 import surrogate as S
    n = 256
    sg = px.Surrogate(n, n, 1, S.IN_SHIFT, S.IN_SCALE, S.OUT_SCALE)
    sg.set_params(S.load_params())
    c = torch.from_numpy(S.initial_field(300, n))[None].cuda()
    out = torch.empty_like(c)
    for _ in range(3):
        sg.step(c, out)
        c, out = out, c
    sg.status()  # raises PhixError(ERR_TIMEOUT) had a wait given up
    sg.close()
