"""The drop-in boundary end to end: the reference's own objects (the same
objects as oracle/_ref/libfinref.so) relinked against libfinb200.so through
the relink shim, which replaces object files by name as an application
Makefile would:

* libfinref_shim.so: the steppers FinSolveRK.o, FinSolveMD.o and
  FinSolveLxW.o (with ConstructL.o and GlobalWaveSpd.o) replaced, so whole
  runs go to the device;
* libfinref_shim_parts.so: the reference's own steppers kept and their
  building blocks ConstructL.o, GlobalWaveSpd.o, UpdateSoln.o, GetCFL.o,
  ConstructIntegratedR.o and ConstructLxWL.o replaced, so the reference's
  FinSolveRK / FinSolveMD / FinSolveLxW drive device calls;
* the MHD application's objects (oracle/_ref/libfinref_mhd.so) with its
  FinSolveRK.o replaced.

Their results must match the golden fixtures the unmodified reference
produced: 1e-12 relative L-infinity per evaluation, 1e-11 per adaptive frame."""
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


@pytest.mark.parametrize("path", golden_cases("finsolvemd") + golden_cases("finsolvelxw"))
def test_relinked_finsolve_md_lxw(shimlib, path):
    """FinSolveMD.o / FinSolveLxW.o replaced: multiderivative (orders 4 and
    5), Lax-Wendroff and Lax-Wendroff with the MPP limiter on the device."""
    _frame(shimlib, path)


@pytest.fixture(scope="module")
def partslib():
    from oracle import REF_SHIM_PARTS_SO, RefLib
    if not RefLib.available(REF_SHIM_PARTS_SO):
        pytest.skip("oracle/_ref/libfinref_shim_parts.so not built (needs the reference checkout)")
    return RefLib(REF_SHIM_PARTS_SO)


def _frame(lib, path):
    g = load_golden(path)
    p = g["p"]
    rc, q1, t1, dt1 = lib.finsolve(p, g["q0"], float(g["t0"]), float(g["tend"]), float(g["dt0"]))
    assert rc == 0
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= 1e-11
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dt1 - float(g["dt1"])) <= 1e-10 * float(g["dt1"])


@pytest.mark.parametrize("path", golden_cases("finsolverk") + golden_cases("finsolvemd") + golden_cases("finsolvelxw"))
def test_reference_steppers_over_device_parts(partslib, path):
    """The reference's own FinSolveRK (orders 1-5, both UpdateSoln forms),
    FinSolveMD (orders 4, 5: all three ConstructIntegratedR forms) and
    FinSolveLxW (ConstructLxWL with and without the face fluxes the MPP
    limiter reads) calling ConstructL, UpdateSoln, GetCFL,
    ConstructIntegratedR and ConstructLxWL on the device."""
    _frame(partslib, path)


@pytest.mark.parametrize("path", golden_cases("intr_"))
def test_relinked_construct_integrated_r(partslib, path):
    from finess_b200._abi import FIN_TS_LXW, FIN_TS_MD
    g = load_golden(path)
    p = g["p"].copy()
    # the relinked application's stepper: Lax-Wendroff for time_order 2 or 3
    # (FinSolveMD takes orders 4 and 5); the integrated flux depends on the
    # order alone
    p.time_stepping_method = FIN_TS_LXW if p.time_order <= 3 else FIN_TS_MD
    F, G = partslib.construct_integrated_r(p, float(g["dt"]), g["q"])
    mb = p.mbc
    fr = (slice(mb - 3, mb + p.mx + 3), slice(mb - 3, mb + p.my + 3))
    assert rel_linf(F[fr], g["F"][fr]) <= 1e-12
    assert rel_linf(G[fr], g["G"][fr]) <= 1e-12


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
