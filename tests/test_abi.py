"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; the ctypes struct mirrors fin_params exactly."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT
from finess_b200 import solver
from finess_b200._abi import FinParams, default_params


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(fin_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from finess_b200.build import build
    build()
    return solver.load_library()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fin_create" in names and "fin_solve" in names and len(names) >= 15


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(lib, name):
    assert hasattr(lib, name), name


def test_params_default_matches_python(lib):
    p = FinParams()
    lib.fin_params_default(C.byref(p))
    q = default_params()
    assert p.as_dict() == q.as_dict()
    assert lib.fin_abi_version() == 2


def test_create_fails_cleanly_without_gpu_or_with_bad_args(lib):
    h = C.c_void_p()
    bad = default_params(mbc=2)
    rc = lib.fin_create(C.byref(bad), C.byref(h))
    assert rc != 0 and not h.value
    assert b"mbc" in lib.fin_last_error()


def test_mhd_create_validates_without_gpu(lib):
    from finess_b200 import problems as P
    h = C.c_void_p()
    lib.fin_mhd_last_error.restype = C.c_char_p
    bad = P.orszag_tang_params(n=16, meqn=5)
    assert lib.fin_mhd_create(C.byref(bad), C.byref(h)) == 1 and not h.value
    assert b"meqn 8" in lib.fin_mhd_last_error()
    bad = P.orszag_tang_params(n=16, mbc=3)
    assert lib.fin_mhd_create(C.byref(bad), C.byref(h)) == 1
    assert b"mbc" in lib.fin_mhd_last_error()


def test_space_order_validation_without_gpu(lib):
    """The (space_order, weno_version) pairs GetWenoReconstruct
    (lib/WenoReconstruct.cpp:40-71) throws for are refused with its message;
    the others need mbc >= (order + 1) / 2 and FP64 Runge-Kutta stepping."""
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_PREC_FP32, FIN_TS_LXW, FIN_TS_MD, FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z
    h = C.c_void_p()
    for so, w in ((3, FIN_WENO_JS), (11, FIN_WENO_Z), (11, FIN_WENO_FD), (13, FIN_WENO_JS), (0, FIN_WENO_Z)):
        bad = P.riemann_params(n=16, weno=w, space_order=so, mbc=7)
        assert lib.fin_create(C.byref(bad), C.byref(h)) != 0 and not h.value
        assert b"Requested WENO Reconstruction not implemented." in lib.fin_last_error()
    bad = P.riemann_params(n=16, weno=FIN_WENO_JS, space_order=11, mbc=5)
    assert lib.fin_create(C.byref(bad), C.byref(h)) != 0
    assert b"mbc must be >= (space_order + 1) / 2" in lib.fin_last_error()
    for kw in ({"precision": FIN_PREC_FP32}, {"time_stepping_method": FIN_TS_LXW, "time_order": 3},
               {"time_stepping_method": FIN_TS_MD, "time_order": 4}):
        bad = P.riemann_params(n=16, weno=FIN_WENO_Z, space_order=7, mbc=5, **kw)
        assert lib.fin_create(C.byref(bad), C.byref(h)) != 0
        assert b"space orders other than 5" in lib.fin_last_error()
    # an accepted pair gets past validation (without a GPU it stops at the device)
    ok = P.riemann_params(n=16, weno=FIN_WENO_FD, space_order=9, mbc=5)
    if lib.fin_create(C.byref(ok), C.byref(h)) == 0:
        lib.fin_destroy(h)
    else:
        assert b"Requested WENO" not in lib.fin_last_error() and b"space order" not in lib.fin_last_error()


def test_get_cfl_alpha_matches_reference_arithmetic(lib):
    """GetCFL from the global wave speeds (lib/2d/GetCFL.cpp:76-101) is host
    arithmetic: max(dt a1/dx, dt a2/dy) and the reference's two errors."""
    from finess_b200._abi import FIN_ERR_CFL_BOUNDS, FIN_ERR_DT_BOUNDS, FIN_OK
    p = default_params(mx=40, my=25, xlow=0.0, xhigh=2.0, ylow=-1.0, yhigh=1.5)
    lib.fin_get_cfl_alpha.argtypes = [C.POINTER(FinParams), C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.POINTER(C.c_double)]
    cfl = C.c_double()
    dt, a1, a2 = 1e-3, 3.7, 2.9
    assert lib.fin_get_cfl_alpha(C.byref(p), dt, 1.0, a1, a2, C.byref(cfl)) == FIN_OK
    dx, dy = (2.0 - 0.0) / 40, (1.5 - -1.0) / 25
    assert cfl.value == max(dt * a1 / dx, dt * a2 / dy, -100.0)
    assert lib.fin_get_cfl_alpha(C.byref(p), 2.0, 1.0, a1, a2, C.byref(cfl)) == FIN_ERR_DT_BOUNDS
    assert lib.fin_get_cfl_alpha(C.byref(p), dt, 1.0, 1e12, a2, C.byref(cfl)) == FIN_ERR_CFL_BOUNDS
