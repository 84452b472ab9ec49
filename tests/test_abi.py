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
