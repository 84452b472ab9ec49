"""The ideal-MHD restatement (oracle/mhd_oracle.c) against the reference's
own compiled MHD sources (lib/2d/ConstructL.cpp with apps/2d/mhd/lib and the
Orszag-Tang case): golden fixtures (always) and live runs (where
oracle/_ref/libfinref_mhd.so exists).  Bit-exact: same operation order, no
FMA contraction on either side."""
import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden
from finess_b200 import problems as P
from finess_b200._abi import FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z


@pytest.fixture(scope="module")
def mhdref():
    from oracle import MhdRefLib
    if not MhdRefLib.available():
        pytest.skip("oracle/_ref/libfinref_mhd.so not built (needs the reference checkout)")
    return MhdRefLib()


@pytest.mark.parametrize("path", golden_cases("mhd_constructl_"))
def test_mhd_construct_l_hj_ct_match_golden(oracle, path):
    g = load_golden(path)
    p, q, aux = g["p"], g["q"], g["aux"]
    L, smax = oracle.mhd_construct_l(p, q)
    assert np.array_equal(interior(p, L), interior(p, g["L"]))
    assert np.array_equal(smax, g["smax"])
    assert oracle.mhd_global_wave_spd(p, q) == tuple(g["alpha"])
    assert np.array_equal(oracle.mhd_construct_hj_l(p, q, aux), g["Laux"])
    assert np.array_equal(interior(p, oracle.mhd_after_step(p, q, aux)), interior(p, g["qct"]))


@pytest.mark.parametrize("path", golden_cases("mhd_finsolverk_"))
def test_mhd_finsolve_matches_golden(oracle, path):
    g = load_golden(path)
    p = g["p"]
    rc, q1, aux1, t1, dt1, n = oracle.mhd_finsolve(p, g["q0"], g["aux0"], float(g["t0"]), float(g["tend"]),
                                                    float(g["dt0"]))
    assert rc == 0 and n > 0
    assert np.array_equal(interior(p, q1), interior(p, g["q1"]))
    assert np.array_equal(interior(p, aux1), interior(p, g["aux1"]))
    assert t1 == float(g["t1"])
    assert dt1 == float(g["dt1"])


def test_orszag_tang_init_matches_numpy(oracle):
    """The numpy initial state of finess_b200.problems equals the C one to
    rounding of the library sin/cos (both sample cell centres)."""
    p = P.orszag_tang_params(n=32)
    q, aux = oracle.orszag_tang(p)
    q2, aux2 = P.orszag_tang_init(p)
    assert np.abs(q - q2).max() < 1e-13
    assert np.abs(aux - aux2).max() < 1e-13


def test_constrained_transport_is_discretely_divergence_free(oracle):
    """After AfterStep, B = curl A3 by the same 4th-order central operator
    in both directions, so the matching discrete divergence vanishes to
    rounding."""
    p = P.orszag_tang_params(n=40)
    rng = np.random.default_rng(3)
    q, aux = P.mhd_random_state(p, rng)
    q, aux = oracle.mhd_set_bnd(p, q, aux)
    qc = oracle.mhd_after_step(p, q, aux)
    qc, _ = oracle.mhd_set_bnd(p, qc, aux)
    dx = (p.xhigh - p.xlow) / p.mx
    dy = (p.yhigh - p.ylow) / p.my
    B1, B2 = qc[..., 5], qc[..., 6]

    def d4(a, axis, h):
        return (np.roll(a, 2, axis) - 8 * np.roll(a, 1, axis) + 8 * np.roll(a, -1, axis) - np.roll(a, -2, axis)) / (
            12 * h)
    div = d4(B1, 0, dx) + d4(B2, 1, dy)
    mb = p.mbc
    assert np.abs(div[mb + 2:-mb - 2, mb + 2:-mb - 2]).max() < 1e-12


def test_mhd_oracle_live_vs_reference(oracle, mhdref):
    rng = np.random.default_rng(11)
    for weno, ga in ((FIN_WENO_JS, 0), (FIN_WENO_Z, 1), (FIN_WENO_FD, 0)):
        p = P.orszag_tang_params(n=18, weno=weno, global_alpha=ga)
        p.my = 21
        q, aux = oracle.mhd_set_bnd(p, *P.mhd_random_state(p, rng))
        q2, aux2 = mhdref.set_bnd(p, q, aux)
        assert np.array_equal(q, q2) and np.array_equal(aux, aux2)
        L1, s1 = oracle.mhd_construct_l(p, q)
        L2, s2 = mhdref.construct_l(p, q, aux)
        assert np.array_equal(interior(p, L1), interior(p, L2))
        assert np.array_equal(s1, s2)
        assert np.array_equal(oracle.mhd_construct_hj_l(p, q, aux), mhdref.construct_hj_l(p, q, aux))
    p = P.orszag_tang_params(n=16, weno=FIN_WENO_Z)
    q0, aux0 = mhdref.set_bnd(p, *mhdref.qinit(p))
    r1 = mhdref.finsolve(p, q0, aux0, 0.0, 0.04, 1e-3)
    r2 = oracle.mhd_finsolve(p, q0, aux0, 0.0, 0.04, 1e-3)
    assert r1[0] == 0 and r2[0] == 0
    assert np.array_equal(interior(p, r1[1]), interior(p, r2[1]))
    assert np.array_equal(interior(p, r1[2]), interior(p, r2[2]))
    assert r1[3] == r2[3] and r1[4] == r2[4]
