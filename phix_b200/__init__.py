"""phix_b200 -- B200-native (sm_100a) PhiX finite-difference time step.

This module is the ctypes binding of the C ABI in include/phix_b200.h
(libphix_b200.so, built in-tree by phix_b200/build.py).  It is what a Python
caller of the library binds; the C++ drop-in API lives in include/phix/.
Device memory and streams come from PyTorch (plumbing only); every kernel is
the library's own.  There is no CPU fallback: without the shared library or a
GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphix_b200.so")

OK, ERR_ARG, ERR_CUDA, ERR_UNSUPPORTED, ERR_NONFINITE, ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
BC_NONE, BC_PERIODIC, BC_NOFLUX, BC_FIXED = 0, 1, 2, 3
PHYS_AC, PHYS_CH, PHYS_CHAC = 0, 1, 2
EULER, RK4, MULTISTEP = 0, 1, 2
F64, F32 = 0, 1
PW_IDENT, PW_AC, PW_DW, PW_CHAC_C, PW_CHAC_E, PW_MUL = range(6)

NFIELDS = {PHYS_AC: 1, PHYS_CH: 1, PHYS_CHAC: 2}


class PhixError(RuntimeError):
    """Status < 0 from the library.  `code` is the PHIX_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class PhixArgumentError(PhixError, ValueError):
    """PHIX_ERR_ARG: the analogue of the reference's std::invalid_argument."""


class GridT(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("n", C.c_int32 * 3),
        ("ghost", C.c_int32),
        ("bc_type", C.c_int32 * 6),
        ("reserved", C.c_int32),
        ("d", C.c_double * 3),
        ("bc_val", C.c_double * 6),
    ]


def make_grid(n: Sequence[int], d: Sequence[float] = (1.0, 1.0, 1.0), ghost: int = 1,
              bc: Sequence[int] = (BC_PERIODIC,) * 6, bc_val: Sequence[float] = (0.0,) * 6) -> GridT:
    g = GridT()
    g.dim = len(n)
    n3 = list(n) + [1] * (3 - len(n))
    d3 = list(d) + [1.0] * (3 - len(d))
    for i in range(3):
        g.n[i] = int(n3[i])
        g.d[i] = float(d3[i])
    g.ghost = ghost
    for i in range(6):
        g.bc_type[i] = int(bc[i])
        g.bc_val[i] = float(bc_val[i])
    g.reserved = 0
    return g


def stored_shape(g: GridT):
    return (g.n[2] + 2 * g.ghost, g.n[1] + 2 * g.ghost, g.n[0] + 2 * g.ghost)


_lib = None


def lib() -> C.CDLL:
    """The loaded libphix_b200.so; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m phix_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER(C.c_double)
    G = C.POINTER(GridT)
    vp = C.c_void_p
    sig = {
        "phix_abi_version": ([], C.c_int),
        "phix_last_error": ([], C.c_char_p),
        "phix_launch_count": ([], C.c_longlong),
        "phix_bc_apply": ([vp, G, vp], C.c_int),
        "phix_lap_accumulate": ([vp, vp, C.c_double, G, vp], C.c_int),
        "phix_grad_accumulate": ([vp, vp, C.c_double, C.c_int, G, vp], C.c_int),
        "phix_pointwise_accumulate": ([vp, vp, vp, C.c_double, C.c_int, P, G, vp], C.c_int),
        "phix_mul_accumulate": ([vp, vp, vp, C.c_double, G, vp], C.c_int),
        "phix_axpy": ([vp, vp, C.c_double, C.c_size_t, vp], C.c_int),
        "phix_stepper_create": ([C.POINTER(vp), C.c_int, C.c_int, C.c_int, P, C.c_double, G], C.c_int),
        "phix_stepper_destroy": ([vp], C.c_int),
        "phix_stepper_nfields": ([vp], C.c_int),
        "phix_stepper_load": ([vp, C.POINTER(vp), vp], C.c_int),
        "phix_stepper_store": ([vp, C.POINTER(vp), vp], C.c_int),
        "phix_stepper_advance": ([vp, C.c_int, vp], C.c_int),
        "phix_stepper_status": ([vp, vp], C.c_int),
        "phix_stepper_set_graph": ([vp, C.c_int], C.c_int),
        "phix_stepper_set_fusion": ([vp, C.c_int], C.c_int),
        "phix_stepper_launches_per_step": ([vp], C.c_int),
        "phix_stepper_depth": ([vp], C.c_int),
        "phix_stepper_set_tiles": ([vp, C.c_int], C.c_int),
        "phix_stepper_autotune": ([vp, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "phix_stepper_get_tiles": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "phix_stepper_bind": ([vp, C.POINTER(vp), C.POINTER(vp)], C.c_int),
        "phix_stepper_current": ([vp], C.c_int),
        "phix_stepper_run_host": ([vp, C.POINTER(vp), C.POINTER(vp), C.c_int], C.c_int),
        "phix_reduce_mass_energy": ([C.POINTER(vp), C.c_int, P, G, P, vp], C.c_int),
        "phix_reduce_mass_energy_noalloc": ([C.POINTER(vp), C.c_int, P, G, P, vp], C.c_int),
        "phix_batch_create": ([C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_int, G, P, C.c_double], C.c_int),
        "phix_batch_destroy": ([vp], C.c_int),
        "phix_batch_launches_per_step": ([vp], C.c_int),
        "phix_batch_set_fusion": ([vp, C.c_int], C.c_int),
        "phix_batch_set_depth": ([vp, C.c_int], C.c_int),
        "phix_batch_depth": ([vp], C.c_int),
        "phix_batch_load": ([vp, C.c_int, vp, C.c_int, vp], C.c_int),
        "phix_batch_store": ([vp, C.c_int, vp, C.c_int, vp], C.c_int),
        "phix_batch_advance": ([vp, C.c_int, vp], C.c_int),
        "phix_batch_set_graph": ([vp, C.c_int], C.c_int),
        "phix_batch_set_tiles": ([vp, C.c_int, C.c_int], C.c_int),
        "phix_batch_get_tiles": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "phix_batch_autotune": ([vp, C.c_int, P], C.c_int),
        "phix_batch_mass": ([vp, P], C.c_int),
        "phix_surrogate_create": ([C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double],
                                  C.c_int),
        "phix_surrogate_destroy": ([vp], C.c_int),
        "phix_surrogate_nparams": ([], C.c_int),
        "phix_surrogate_set_params": ([vp, vp], C.c_int),
        "phix_surrogate_get_params": ([vp, vp, vp], C.c_int),
        "phix_surrogate_step": ([vp, vp, vp, C.c_int, vp], C.c_int),
        "phix_surrogate_set_fused": ([vp, C.c_int], C.c_int),
        "phix_surrogate_forward": ([vp, vp, vp, C.c_int, vp], C.c_int),
        "phix_surrogate_grad": ([vp, vp, vp, C.c_int, P, vp], C.c_int),
        "phix_surrogate_adam": ([vp, vp, C.c_float, vp], C.c_int),
        "phix_surrogate_grad_ptr": ([vp], C.c_void_p),
        "phix_surrogate_status": ([vp, vp], C.c_int),
        "phix_wait_selftest": ([C.c_int, C.c_double, vp], C.c_int),
        "phix_measure_fma_peak": ([C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "phix_plane_gather": ([vp, vp, C.c_int, C.c_int, C.c_int, vp], C.c_int),
        "phix_plane_scatter": ([vp, vp, C.c_int, C.c_int, C.c_int, vp], C.c_int),
        "phix_stepper_diagnostics": ([vp, P], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc: int) -> int:
    if rc < 0:
        msg = lib().phix_last_error().decode(errors="replace")
        if rc == ERR_ARG:
            raise PhixArgumentError(rc, msg)
        raise PhixError(rc, msg)
    return rc


def launch_count() -> int:
    return int(lib().phix_launch_count())


def measure_fma_peak(precision: int, packed: bool = False) -> float:
    """Measured FMA throughput of the current GPU in TFLOP/s (fma = 2 flops)."""
    t = C.c_double()
    check(lib().phix_measure_fma_peak(precision, 1 if packed else 0, C.byref(t)))
    return t.value


def _prm(prm: Sequence[float]):
    v = list(prm) + [0.0] * (8 - len(prm))
    return (C.c_double * 8)(*v)


def _ptrs(tensors):
    return (C.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _dev(t):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise PhixArgumentError(ERR_ARG, "expected a contiguous float64 CUDA tensor")
    return C.c_void_p(t.data_ptr())


# ---------------------------------------------------------------------------
# single operators (device tensors in the stored layout)
# ---------------------------------------------------------------------------
def bc_apply(field, g: GridT, stream=None):
    check(lib().phix_bc_apply(_dev(field), C.byref(g), _stream(stream)))


def lap_accumulate(rhs, src, coeff: float, g: GridT, stream=None):
    check(lib().phix_lap_accumulate(_dev(rhs), _dev(src), coeff, C.byref(g), _stream(stream)))


def grad_accumulate(rhs, src, coeff: float, axis: int, g: GridT, stream=None):
    check(lib().phix_grad_accumulate(_dev(rhs), _dev(src), coeff, axis, C.byref(g), _stream(stream)))


def pointwise_accumulate(rhs, s1, s2, coeff: float, func: int, prm: Sequence[float], g: GridT, stream=None):
    p = _prm(prm)
    check(lib().phix_pointwise_accumulate(_dev(rhs), _dev(s1), _dev(s2) if s2 is not None else None, coeff,
                                          func, p, C.byref(g), _stream(stream)))


def mul_accumulate(rhs, s1, s2, coeff: float, g: GridT, stream=None):
    check(lib().phix_mul_accumulate(_dev(rhs), _dev(s1), _dev(s2), coeff, C.byref(g), _stream(stream)))


def axpy(dst, src, coeff: float, stream=None):
    check(lib().phix_axpy(_dev(dst), _dev(src), coeff, dst.numel(), _stream(stream)))


def reduce_mass_energy(fields, phys: int, prm: Sequence[float], g: GridT, stream=None):
    out = (C.c_double * 2)()
    check(lib().phix_reduce_mass_energy(_ptrs(fields), phys, _prm(prm), C.byref(g), out, _stream(stream)))
    return out[0], out[1]


def reduce_mass_energy_noalloc(fields, phys: int, prm: Sequence[float], g: GridT, stream=None):
    """Allocation-free diagnostics (scratch in a static device array)."""
    out = (C.c_double * 2)()
    check(lib().phix_reduce_mass_energy_noalloc(_ptrs(fields), phys, _prm(prm), C.byref(g), out, _stream(stream)))
    return out[0], out[1]


# ---------------------------------------------------------------------------
# fused stepper
# ---------------------------------------------------------------------------
class Stepper:
    """Owning wrapper of phix_stepper_t (one built-in physics on one grid)."""

    def __init__(self, phys: int, scheme: int, precision: int, prm: Sequence[float], dt: float, g: GridT):
        self.g = g
        self.phys, self.scheme, self.precision = phys, scheme, precision
        self.prm = list(prm)
        self.dt = dt
        h = C.c_void_p()
        check(lib().phix_stepper_create(C.byref(h), phys, scheme, precision, _prm(prm), dt, C.byref(g)))
        self.h = h
        self.nf = 2 if scheme == MULTISTEP else NFIELDS[phys]  # multi-step: c and mu

    def close(self):
        if getattr(self, "h", None):
            lib().phix_stepper_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def load(self, fields, stream=None):
        check(lib().phix_stepper_load(self.h, _ptrs(fields), _stream(stream)))

    def store(self, fields, stream=None):
        check(lib().phix_stepper_store(self.h, _ptrs(fields), _stream(stream)))

    def advance(self, nsteps: int, stream=None):
        check(lib().phix_stepper_advance(self.h, nsteps, _stream(stream)))

    def status(self, stream=None):
        """Raise PhixError (ERR_TIMEOUT) if a fused 3-D step gave up waiting
        for a plane copy since the last check; clears the flag."""
        check(lib().phix_stepper_status(self.h, _stream(stream)))

    def set_graph(self, steps_per_graph: int):
        check(lib().phix_stepper_set_graph(self.h, steps_per_graph))

    def set_fusion(self, on: bool):
        """One launch per RK4 step (True, default where supported) or per stage."""
        check(lib().phix_stepper_set_fusion(self.h, 1 if on else 0))

    @property
    def launches_per_step(self) -> int:
        return lib().phix_stepper_launches_per_step(self.h)

    @property
    def depth(self) -> int:
        """Time steps one launch advances (temporal-block depth)."""
        return lib().phix_stepper_depth(self.h)

    def set_tiles(self, cfg: int):
        """2-D tile shape: one launch per stage -1 (box) or 0..3 (column
        tiles); one launch per RK4 step 0..19 (6..15 pair tiles, 16..19
        temporally blocked pair tiles: two steps per launch), -1 by grid."""
        check(lib().phix_stepper_set_tiles(self.h, cfg))

    def tiles(self):
        """(one launch per RK4 step?, tile configuration) currently in use."""
        f, t = C.c_int(), C.c_int()
        check(lib().phix_stepper_get_tiles(self.h, C.byref(f), C.byref(t)))
        return bool(f.value), t.value

    def autotune(self, trial_steps: int = 3) -> float:
        """Time every launch form and tile shape on the current state (which
        is restored), keep the fastest; returns its ms per step."""
        ms = C.c_double()
        check(lib().phix_stepper_autotune(self.h, trial_steps, C.byref(ms)))
        return ms.value

    def bind(self, fields, alt):
        check(lib().phix_stepper_bind(self.h, _ptrs(fields), _ptrs(alt)))

    def current(self) -> int:
        return check(lib().phix_stepper_current(self.h))

    def run_host(self, host_in, host_out, nsteps: int):
        """host_in/host_out: float64 numpy arrays or pinned CPU tensors (stored layout)."""
        def hp(a):
            if isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
                return a.ctypes.data
            return a.data_ptr()
        pin = (C.c_void_p * self.nf)(*[hp(a) for a in host_in])
        pout = (C.c_void_p * self.nf)(*[hp(a) for a in host_out])
        check(lib().phix_stepper_run_host(self.h, pin, pout, nsteps))

    def diagnostics(self):
        out = (C.c_double * 2)()
        check(lib().phix_stepper_diagnostics(self.h, out))
        return out[0], out[1]


class Batch:
    """Owning wrapper of phix_batch_t: many independent 2-D fields of one
    single-field physics advanced in lockstep, one persistent launch per stage."""

    def __init__(self, phys: int, scheme: int, precision: int, grids, prms, dt: float):
        self.n = len(grids)
        self.grids = list(grids)
        garr = (GridT * self.n)(*grids)
        flat = []
        for p in prms:
            flat += list(p) + [0.0] * (8 - len(p))
        parr = (C.c_double * len(flat))(*flat)
        h = C.c_void_p()
        check(lib().phix_batch_create(C.byref(h), phys, scheme, precision, self.n, garr, parr, dt))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().phix_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_field(self, inst: int, field):
        if not 0 <= inst < self.n:
            raise IndexError(f"batch instance {inst} out of range [0, {self.n})")
        want = int(np.prod(stored_shape(self.grids[inst])))
        if isinstance(field, np.ndarray):
            ok = field.dtype == np.float64 and field.flags["C_CONTIGUOUS"]
        else:
            import torch
            ok = field.dtype == torch.float64 and field.is_contiguous()
        if not ok:
            raise ValueError("batch field must be a contiguous float64 array")
        n = field.size if isinstance(field, np.ndarray) else field.numel()
        if n != want:
            raise ValueError(f"batch instance {inst}: field has {n} values, its stored grid has {want}")

    def load(self, inst: int, field, stream=None):
        """field: FP64 stored array; numpy (host) or CUDA tensor (device)."""
        self._check_field(inst, field)
        if isinstance(field, np.ndarray):
            check(lib().phix_batch_load(self.h, inst, C.c_void_p(field.ctypes.data), 1, _stream(stream)))
        else:
            check(lib().phix_batch_load(self.h, inst, _dev(field), 0, _stream(stream)))

    def store(self, inst: int, field, stream=None):
        self._check_field(inst, field)
        if isinstance(field, np.ndarray):
            check(lib().phix_batch_store(self.h, inst, C.c_void_p(field.ctypes.data), 1, _stream(stream)))
        else:
            check(lib().phix_batch_store(self.h, inst, _dev(field), 0, _stream(stream)))

    def advance(self, nsteps: int, stream=None):
        check(lib().phix_batch_advance(self.h, nsteps, _stream(stream)))

    def set_graph(self, steps: int):
        check(lib().phix_batch_set_graph(self.h, steps))

    def set_fusion(self, on: bool):
        """One launch per RK4 step for the whole batch (True) or one per stage."""
        check(lib().phix_batch_set_fusion(self.h, 1 if on else 0))

    def set_depth(self, depth: int):
        """Temporal-block depth of the one-launch step: 1, or 2 (two RK4 steps per launch)."""
        check(lib().phix_batch_set_depth(self.h, depth))

    @property
    def depth(self) -> int:
        return lib().phix_batch_depth(self.h)

    @property
    def launches_per_step(self) -> int:
        return lib().phix_batch_launches_per_step(self.h)

    def set_tiles(self, cfg: int, ctas_per_sm: int = 0):
        check(lib().phix_batch_set_tiles(self.h, cfg, ctas_per_sm))

    def tiles(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().phix_batch_get_tiles(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def autotune(self, trial_steps: int = 5) -> float:
        ms = C.c_double()
        check(lib().phix_batch_autotune(self.h, trial_steps, C.byref(ms)))
        return ms.value

    def mass(self):
        out = (C.c_double * self.n)()
        check(lib().phix_batch_mass(self.h, out))
        return list(out)


class Surrogate:
    """Owning wrapper of phix_surrogate_t.  States are [B, H, W] float64 CUDA
    tensors; parameters travel as flat float32 numpy vectors in the order
    W1[32][9] b1[32] W2[32][9][32] b2[32] W3[32][9][32] b3[32] W4[9][32] b4[1]."""

    def __init__(self, H: int, W: int, batch_max: int, in_shift: float, in_scale: float, out_scale: float):
        self.H, self.W, self.bmax = H, W, batch_max
        self.in_shift, self.in_scale, self.out_scale = in_shift, in_scale, out_scale
        h = C.c_void_p()
        check(lib().phix_surrogate_create(C.byref(h), H, W, batch_max, in_shift, in_scale, out_scale))
        self.h = h
        self.nparams = lib().phix_surrogate_nparams()

    def close(self):
        if getattr(self, "h", None):
            lib().phix_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        assert flat.size == self.nparams
        check(lib().phix_surrogate_set_params(self.h, C.c_void_p(flat.ctypes.data)))

    def get_params(self):
        p = np.empty(self.nparams, np.float32)
        g = np.empty(self.nparams, np.float32)
        check(lib().phix_surrogate_get_params(self.h, C.c_void_p(p.ctypes.data), C.c_void_p(g.ctypes.data)))
        return p, g

    def set_fused(self, on: bool):
        """step(): one fused kernel (True, default) or the per-layer kernels."""
        check(lib().phix_surrogate_set_fused(self.h, 1 if on else 0))

    def step(self, c, c_out, stream=None):
        check(lib().phix_surrogate_step(self.h, C.c_void_p(c.data_ptr()), C.c_void_p(c_out.data_ptr()),
                                        c.shape[0], _stream(stream)))

    def forward(self, c, o, stream=None):
        check(lib().phix_surrogate_forward(self.h, C.c_void_p(c.data_ptr()), C.c_void_p(o.data_ptr()),
                                           c.shape[0], _stream(stream)))

    def grad(self, c, c_next, stream=None) -> float:
        loss = C.c_double()
        check(lib().phix_surrogate_grad(self.h, C.c_void_p(c.data_ptr()), C.c_void_p(c_next.data_ptr()),
                                        c.shape[0], C.byref(loss), _stream(stream)))
        return loss.value

    def grad_ptr(self) -> int:
        return lib().phix_surrogate_grad_ptr(self.h)

    def status(self, stream=None):
        """Raise PhixError (code ERR_TIMEOUT) if a bounded tensor-core wait of
        this surrogate's kernels gave up since the last check; clears it."""
        check(lib().phix_surrogate_status(self.h, _stream(stream)))

    def adam(self, lr: float, grads=None, stream=None):
        gp = C.c_void_p(grads.data_ptr()) if grads is not None else None
        check(lib().phix_surrogate_adam(self.h, gp, lr, _stream(stream)))


def plane_gather(stored, plane, H: int, W: int, ghost: int = 1, stream=None):
    check(lib().phix_plane_gather(C.c_void_p(stored.data_ptr()), C.c_void_p(plane.data_ptr()), H, W, ghost,
                                  _stream(stream)))


def plane_scatter(plane, stored, H: int, W: int, ghost: int = 1, stream=None):
    check(lib().phix_plane_scatter(C.c_void_p(plane.data_ptr()), C.c_void_p(stored.data_ptr()), H, W, ghost,
                                   _stream(stream)))


def surrogate_params_to_flat(params) -> np.ndarray:
    """Oracle parameter list [W1,b1,...,W4,b4] (W[n,ky,kx,ci]) -> flat vector."""
    W1, b1, W2, b2, W3, b3, W4, b4 = params
    parts = [W1.reshape(32, 9), b1, W2.reshape(32, 9, 32), b2, W3.reshape(32, 9, 32), b3, W4.reshape(9, 32), b4]
    return np.concatenate([np.asarray(p, np.float32).ravel() for p in parts])


def surrogate_flat_to_params(flat: np.ndarray):
    o = 0
    out = []
    for shape in ((32, 3, 3, 1), (32,), (32, 3, 3, 32), (32,), (32, 3, 3, 32), (32,), (1, 3, 3, 32), (1,)):
        n = int(np.prod(shape))
        out.append(np.asarray(flat[o:o + n], np.float32).reshape(shape))
        o += n
    return out


def build_library(verbose: bool = False) -> str:
    """Compile libphix_b200.so in-tree (nvcc, sm_100a)."""
    from .build import build as _build
    return _build(verbose=verbose)
