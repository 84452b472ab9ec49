"""The drop-in boundary end to end: the reference's own driver objects (the
same objects as oracle/_ref/libfinref.so) relinked against libfinb200.so
through the relink shim, which replaces ConstructL.o, GlobalWaveSpd.o and
FinSolveRK.o by name as an application Makefile would; likewise the MHD
application's objects (oracle/_ref/libfinref_mhd.so) with its FinSolveRK.o
replaced.  Their results must match the golden fixtures the unmodified
reference produced."""
import os

import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, rel_linf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shimlib():
    from oracle import REF_SHIM_SO, RefLib
    if not RefLib.available(REF_SHIM_SO):
        pytest.skip("oracle/_ref/libfinref_shim.so not built (needs the reference checkout)")
    return RefLib(REF_SHIM_SO)


@pytest.mark.parametrize("path", golden_cases("constructl_"))
def test_relinked_construct_l(shimlib, path):
    g = load_golden(path)
    p = g["p"]
    L, smax = shimlib.construct_l(p, g["q"])
    assert rel_linf(interior(p, L), interior(p, g["L"])) <= 1e-12
    assert rel_linf(smax, g["smax"]) <= 1e-14
    a1, a2 = shimlib.global_wave_spd(p, g["q"])
    assert abs(a1 - g["alpha"][0]) <= 1e-15 * g["alpha"][0]


@pytest.mark.parametrize("path", golden_cases("finsolverk_"))
def test_relinked_finsolve_rk(shimlib, path):
    g = load_golden(path)
    p = g["p"]
    rc, q1, t1, dt1 = shimlib.finsolve(p, g["q0"], float(g["t0"]), float(g["tend"]), float(g["dt0"]))
    assert rc == 0
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= 1e-11
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dt1 - float(g["dt1"])) <= 1e-10 * float(g["dt1"])


@pytest.fixture(scope="module")
def mhdshim():
    from oracle import REF_MHD_SHIM_SO, MhdRefLib
    if not MhdRefLib.available(REF_MHD_SHIM_SO):
        pytest.skip("oracle/_ref/libfinref_mhd_shim.so not built (needs the reference checkout)")
    return MhdRefLib(REF_MHD_SHIM_SO)


@pytest.mark.parametrize("path", golden_cases("mhd_finsolverk_"))
def test_relinked_mhd_finsolve_rk(mhdshim, path):
    g = load_golden(path)
    p = g["p"]
    rc, q1, aux1, t1, dt1 = mhdshim.finsolve(p, g["q0"], g["aux0"], float(g["t0"]), float(g["tend"]),
                                             float(g["dt0"]))
    assert rc == 0
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= 1e-11
    assert rel_linf(interior(p, aux1), interior(p, g["aux1"])) <= 1e-11
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dt1 - float(g["dt1"])) <= 1e-10 * float(g["dt1"])
