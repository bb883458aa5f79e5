"""C ABI checks that need no GPU: the library loads, exports every entry point
declared in include/phix_b200.h, and rejects bad arguments with PHIX_ERR_ARG
before touching the device (the reference's std::invalid_argument cases)."""
import ctypes as C
import os
import re

import pytest

import phix_b200 as px

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", "phix_b200.h")]


def declared_symbols():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(phix_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    lib = px.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.phix_abi_version() == 1


def test_grid_struct_layout_matches_header():
    assert C.sizeof(px.GridT) == 4 * (1 + 3 + 1 + 6 + 1) + 8 * (3 + 6)
    assert px.GridT.d.offset == 48


@pytest.mark.parametrize("bad", [
    dict(n=(8, 8), bc=(px.BC_PERIODIC, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_PERIODIC, 0, 0)),  # mismatched periodic
    dict(n=(8, 0)),
    dict(n=(8, 8), ghost=0),
    dict(n=(8, 8), d=(1.0, -1.0)),
])
def test_stepper_create_rejects_bad_grids(bad):
    g = px.make_grid(**bad)
    with pytest.raises(px.PhixArgumentError):
        px.Stepper(px.PHYS_CH, px.RK4, px.F64, [1, 0.5, 1, 0, 1], 0.005, g)


def test_unused_axis_must_be_degenerate():
    g = px.make_grid(n=(8, 8))
    g.n[2] = 4  # dim 2 with nz != 1
    with pytest.raises(px.PhixArgumentError):
        px.Stepper(px.PHYS_AC, px.EULER, px.F64, [1, 1], 0.01, g)


def test_stepper_create_rejects_bad_enums():
    g = px.make_grid(n=(8, 8))
    for phys, scheme, prec in ((7, px.RK4, px.F64), (px.PHYS_AC, 9, px.F64), (px.PHYS_AC, px.RK4, 5)):
        with pytest.raises(px.PhixArgumentError):
            px.Stepper(phys, scheme, prec, [1, 1], 0.01, g)


def test_ops_reject_null_pointers_and_bad_axis():
    lib = px.lib()
    g = px.make_grid(n=(8, 8))
    assert lib.phix_lap_accumulate(None, None, 1.0, C.byref(g), None) == px.ERR_ARG
    assert lib.phix_bc_apply(None, C.byref(g), None) == px.ERR_ARG
    assert lib.phix_grad_accumulate(C.c_void_p(16), C.c_void_p(16), 1.0, 2, C.byref(g), None) == px.ERR_ARG
    assert b"axis" in lib.phix_last_error()
    assert lib.phix_pointwise_accumulate(C.c_void_p(16), C.c_void_p(16), None, 1.0, px.PW_MUL, None, C.byref(g),
                                         None) == px.ERR_ARG
    assert lib.phix_stepper_advance(None, 1, None) == px.ERR_ARG
    assert lib.phix_stepper_destroy(None) == px.OK


def test_error_message_names_the_axis():
    g = px.make_grid(n=(8, 8), bc=(px.BC_NOFLUX, px.BC_NOFLUX, px.BC_PERIODIC, px.BC_NOFLUX, 0, 0))
    with pytest.raises(px.PhixArgumentError, match="axis Y"):
        px.Stepper(px.PHYS_CH, px.RK4, px.F64, [1, 0.5, 1, 0, 1], 0.005, g)
