"""ctypes bindings for the CPU oracle (liboracle.so) and the reference harness
(_ref/libphix_ref.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the product package.

Fields are numpy arrays in the reference's ghost-padded stored layout
(ScalarField.h:15-27): shape (n2+2g, n1+2g, n0+2g), x fastest.  Unused axes of
a 1-D/2-D mesh still carry 2*ghost padding planes, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_ORACLE_OMP = os.path.join(HERE, "liboracle_omp.so")  # same restatement, OpenMP loops
LIB_REF = os.path.join(HERE, "_ref", "libphix_ref.so")

BC_NONE, BC_PERIODIC, BC_NOFLUX, BC_FIXED = 0, 1, 2, 3
PHYS_AC, PHYS_CH, PHYS_CHAC = 0, 1, 2
EULER, RK4 = 0, 1
PW_IDENT, PW_AC, PW_DW, PW_CHAC_C, PW_CHAC_E, PW_MUL = range(6)


class GridT(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("n", C.c_int32 * 3),
        ("ghost", C.c_int32),
        ("bc_type", C.c_int32 * 6),
        ("fma_mode", C.c_int32),
        ("d", C.c_double * 3),
        ("bc_val", C.c_double * 6),
    ]


@dataclass
class Grid:
    """Mesh + boundary description shared by oracle, reference and kernels."""

    n: Sequence[int]
    d: Sequence[float] = (1.0, 1.0, 1.0)
    ghost: int = 1
    bc: Sequence[int] = (BC_PERIODIC,) * 6  # [x_lo, x_hi, y_lo, y_hi, z_lo, z_hi]
    bc_val: Sequence[float] = (0.0,) * 6
    fma_mode: int = 0

    @property
    def dim(self) -> int:
        return len(self.n)

    @property
    def n3(self):
        return list(self.n) + [1] * (3 - len(self.n))

    @property
    def stored_shape(self):
        n0, n1, n2 = self.n3
        g = self.ghost
        return (n2 + 2 * g, n1 + 2 * g, n0 + 2 * g)

    def phys(self, a: np.ndarray) -> np.ndarray:
        """Physical-cell view (n2, n1, n0) of a stored array."""
        g = self.ghost
        n0, n1, n2 = self.n3
        return a[g:g + n2, g:g + n1, g:g + n0]

    def ctype(self, fma_mode: int | None = None) -> GridT:
        t = GridT()
        t.dim = self.dim
        for i, v in enumerate(self.n3):
            t.n[i] = v
        t.ghost = self.ghost
        for i in range(6):
            t.bc_type[i] = self.bc[i]
            t.bc_val[i] = self.bc_val[i]
        t.fma_mode = self.fma_mode if fma_mode is None else fma_mode
        d = list(self.d) + [1.0] * (3 - len(self.d))
        for i in range(3):
            t.d[i] = d[i]
        return t

    def stored_from_phys(self, phys: np.ndarray, dtype=np.float64) -> np.ndarray:
        a = np.zeros(self.stored_shape, dtype=dtype)
        self.phys(a)[...] = phys.reshape(self.phys(a).shape)
        return a


def _ptr(a: np.ndarray, ct):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """The C restatement.  Every call works on stored arrays in place."""

    def __init__(self, path: str = LIB_ORACLE):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = C.CDLL(path)
        for sfx, ct in (("_f64", C.c_double), ("_f32", C.c_float)):
            P = C.POINTER(ct)
            PP = C.POINTER(P)
            g = C.POINTER(GridT)
            L = self.lib
            getattr(L, "or_bc_apply" + sfx).argtypes = [P, g]
            getattr(L, "or_lap_acc" + sfx).argtypes = [P, P, C.c_double, g]
            getattr(L, "or_grad_acc" + sfx).argtypes = [P, P, C.c_double, C.c_int, g]
            getattr(L, "or_pw_acc" + sfx).argtypes = [P, P, P, C.c_double, C.c_int, C.POINTER(C.c_double), g]
            getattr(L, "or_mul_acc" + sfx).argtypes = [P, P, P, C.c_double, g]
            getattr(L, "or_rhs" + sfx).argtypes = [PP, PP, C.c_int, C.POINTER(C.c_double), g, P]
            getattr(L, "or_advance" + sfx).argtypes = [PP, C.c_int, C.POINTER(C.c_double), C.c_int,
                                                       C.c_double, C.c_int, g]
            getattr(L, "or_advance" + sfx).restype = C.c_int
            getattr(L, "or_advance_comp" + sfx).argtypes = [PP, PP, C.c_int, C.POINTER(C.c_double), C.c_int,
                                                            C.c_double, C.c_int, g]
            getattr(L, "or_advance_comp" + sfx).restype = C.c_int
            getattr(L, "or_advance_ch_multistep" + sfx).argtypes = [P, P, C.POINTER(C.c_double), C.c_double,
                                                                    C.c_int, g]
            getattr(L, "or_axpy" + sfx).argtypes = [P, P, C.c_double, C.c_long, C.c_int]
            getattr(L, "or_mass" + sfx).argtypes = [P, g]
            getattr(L, "or_mass" + sfx).restype = C.c_double
            getattr(L, "or_energy" + sfx).argtypes = [PP, C.c_int, C.POINTER(C.c_double), g]
            getattr(L, "or_energy" + sfx).restype = C.c_double

    def threads(self) -> int:
        """Host threads the library's loops run on (1 for liboracle.so)."""
        f = getattr(self.lib, "or_threads", None)
        return int(f()) if f else 1

    @staticmethod
    def _sfx(a):
        if a.dtype == np.float64:
            return "_f64", C.c_double
        if a.dtype == np.float32:
            return "_f32", C.c_float
        raise TypeError(a.dtype)

    def _pp(self, arrs, ct):
        P = C.POINTER(ct)
        return (P * len(arrs))(*[_ptr(a, ct) for a in arrs])

    def bc_apply(self, a, grid: Grid, fma_mode=None):
        s, ct = self._sfx(a)
        gt = grid.ctype(fma_mode)
        getattr(self.lib, "or_bc_apply" + s)(_ptr(a, ct), C.byref(gt))

    def lap_acc(self, rhs, src, coeff, grid: Grid, fma_mode=None):
        s, ct = self._sfx(rhs)
        gt = grid.ctype(fma_mode)
        getattr(self.lib, "or_lap_acc" + s)(_ptr(rhs, ct), _ptr(src, ct), coeff, C.byref(gt))

    def grad_acc(self, rhs, src, coeff, axis, grid: Grid, fma_mode=None):
        s, ct = self._sfx(rhs)
        gt = grid.ctype(fma_mode)
        getattr(self.lib, "or_grad_acc" + s)(_ptr(rhs, ct), _ptr(src, ct), coeff, axis, C.byref(gt))

    def pw_acc(self, rhs, s1, s2, coeff, func, prm, grid: Grid, fma_mode=None):
        s, ct = self._sfx(rhs)
        gt = grid.ctype(fma_mode)
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        s2p = _ptr(s2, ct) if s2 is not None else None
        getattr(self.lib, "or_pw_acc" + s)(_ptr(rhs, ct), _ptr(s1, ct), s2p, coeff, func, p, C.byref(gt))

    def mul_acc(self, rhs, s1, s2, coeff, grid: Grid, fma_mode=None):
        s, ct = self._sfx(rhs)
        gt = grid.ctype(fma_mode)
        getattr(self.lib, "or_mul_acc" + s)(_ptr(rhs, ct), _ptr(s1, ct), _ptr(s2, ct), coeff, C.byref(gt))

    def rhs(self, outs, ins, phys, prm, grid: Grid, fma_mode=None):
        s, ct = self._sfx(outs[0])
        gt = grid.ctype(fma_mode)
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        scratch = np.zeros(grid.stored_shape, dtype=outs[0].dtype)
        getattr(self.lib, "or_rhs" + s)(self._pp(outs, ct), self._pp(ins, ct), phys, p, C.byref(gt),
                                        _ptr(scratch, ct))

    def advance(self, fields, phys, prm, scheme, dt, nsteps, grid: Grid, fma_mode=None):
        s, ct = self._sfx(fields[0])
        gt = grid.ctype(fma_mode)
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        rc = getattr(self.lib, "or_advance" + s)(self._pp(fields, ct), phys, p, scheme, dt, nsteps, C.byref(gt))
        if rc != 0:
            raise RuntimeError(f"or_advance failed: {rc}")

    def advance_comp(self, hi, lo, phys, prm, scheme, dt, nsteps, grid: Grid, fma_mode=None):
        """Compensated (hi + lo) state, the FP32 kernels' scheme."""
        s, ct = self._sfx(hi[0])
        gt = grid.ctype(fma_mode)
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        rc = getattr(self.lib, "or_advance_comp" + s)(self._pp(hi, ct), self._pp(lo, ct), phys, p, scheme, dt,
                                                      nsteps, C.byref(gt))
        if rc != 0:
            raise RuntimeError(f"or_advance_comp failed: {rc}")

    def advance_ch_multistep(self, c, mu, prm, dt, nsteps, grid: Grid, fma_mode=None):
        s, ct = self._sfx(c)
        gt = grid.ctype(fma_mode)
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        getattr(self.lib, "or_advance_ch_multistep" + s)(_ptr(c, ct), _ptr(mu, ct), p, dt, nsteps, C.byref(gt))

    def axpy(self, dst, src, coeff, fma_mode=1):
        s, ct = self._sfx(dst)
        getattr(self.lib, "or_axpy" + s)(_ptr(dst, ct), _ptr(src, ct), coeff, dst.size, fma_mode)

    def mass(self, a, grid: Grid) -> float:
        s, ct = self._sfx(a)
        gt = grid.ctype()
        return getattr(self.lib, "or_mass" + s)(_ptr(a, ct), C.byref(gt))

    def energy(self, fields, phys, prm, grid: Grid) -> float:
        s, ct = self._sfx(fields[0])
        gt = grid.ctype()
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        return getattr(self.lib, "or_energy" + s)(self._pp(fields, ct), phys, p, C.byref(gt))


class Reference:
    """The reference library itself (compiled from its sources by oracle/Makefile)."""

    def __init__(self, path: str = LIB_REF):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.lib = C.CDLL(path)
        P = C.POINTER(C.c_double)
        g = C.POINTER(GridT)
        L = self.lib
        L.ref_has_gpu.restype = C.c_int
        L.ref_advance.argtypes = [C.c_int, C.c_int, P, C.c_double, C.c_int, g, C.POINTER(P), C.c_int, P]
        L.ref_advance.restype = C.c_int
        L.ref_advance_ch_multistep.argtypes = [P, C.c_double, C.c_int, g, P, P, C.c_int]
        L.ref_advance_ch_multistep.restype = C.c_int
        L.ref_bc_apply.argtypes = [P, g, C.c_int]
        L.ref_bc_apply.restype = C.c_int
        L.ref_lap.argtypes = [P, P, C.c_double, g, C.c_int]
        L.ref_lap.restype = C.c_int

    def has_gpu(self) -> bool:
        return bool(self.lib.ref_has_gpu())

    def advance(self, fields, phys, prm, scheme, dt, nsteps, grid: Grid, use_gpu=False) -> float:
        """Advance in place; returns elapsed ms of the step loop (GPU path only)."""
        gt = grid.ctype()
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        P = C.POINTER(C.c_double)
        pp = (P * len(fields))(*[_ptr(f, C.c_double) for f in fields])
        ms = C.c_double(0.0)
        rc = self.lib.ref_advance(phys, scheme, p, dt, nsteps, C.byref(gt), pp, int(use_gpu), C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"ref_advance failed: {rc}")
        return ms.value

    def advance_ch_multistep(self, c, mu, prm, dt, nsteps, grid: Grid, use_gpu=False):
        gt = grid.ctype()
        p = (C.c_double * 8)(*(list(prm) + [0.0] * (8 - len(prm))))
        rc = self.lib.ref_advance_ch_multistep(p, dt, nsteps, C.byref(gt), _ptr(c, C.c_double),
                                               _ptr(mu, C.c_double), int(use_gpu))
        if rc != 0:
            raise RuntimeError(f"ref_advance_ch_multistep failed: {rc}")

    def bc_apply(self, a, grid: Grid, use_gpu=False):
        gt = grid.ctype()
        rc = self.lib.ref_bc_apply(_ptr(a, C.c_double), C.byref(gt), int(use_gpu))
        if rc != 0:
            raise RuntimeError("ref_bc_apply failed")

    def lap(self, rhs, src, coeff, grid: Grid, use_gpu=False):
        gt = grid.ctype()
        rc = self.lib.ref_lap(_ptr(rhs, C.c_double), _ptr(src, C.c_double), coeff, C.byref(gt), int(use_gpu))
        if rc != 0:
            raise RuntimeError("ref_lap failed")


def build(ref_tree: str | None = None, quiet: bool = True) -> None:
    """Compile the oracle, and, given the reference project's source tree
    (`ref_tree`, else $PHIX_REFERENCE_TREE), oracle/_ref and the drop-in
    driver pairs."""
    import subprocess
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "liboracle.so", "liboracle_omp.so"], check=True, stdout=out)
    ref_src = ref_tree or os.environ.get("PHIX_REFERENCE_TREE")
    if ref_src and os.path.isdir(os.path.join(ref_src, "src")):
        subprocess.run(["make", "-C", HERE, "-j8", "ref", f"REF={ref_src}"], check=True, stdout=out)
        cxx = os.path.join(os.path.dirname(HERE), "phix_b200", "libphix_cxx.so")
        if os.path.exists(cxx):
            from phix_b200.build import json_include
            subprocess.run(["make", "-C", HERE, "-j4", "dropin", f"REF={ref_src}", f"JSON_INC={json_include() or ''}"],
                           check=True, stdout=out)
