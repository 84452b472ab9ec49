"""The ideal-MHD hybrid form: troubled-face samples against the oracle
(oracle_mhd_face_samples), the per-face choice at its two ends (no face
troubled: the linear FD5 weights everywhere, i.e. the FP32 form with
weno_version FD; every face troubled: the FP32 full-WENO form), the judge
step, and the trained network's accuracy against the FP64 form."""
import os

import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID, FIN_WENO_FD, FIN_WENO_JS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    from finess_b200 import mhd
    return mhd


def _weights():
    from finess_b200.indicator import DEFAULT_MHD_WEIGHTS
    if not os.path.exists(DEFAULT_MHD_WEIGHTS):
        pytest.skip("MHD indicator weights not trained")
    z = np.load(DEFAULT_MHD_WEIGHTS)
    return z["params"], float(z["z_threshold"])


def _run(M, p, q, aux, dt, steps, params=None, zthr=0.0, judge_every=0, judge_tol=1e-3, every=1):
    with M.MhdSolver(p) as s:
        s.set_state(q, aux)
        if params is not None:
            s.set_indicator(params, zthr, judge_every, judge_tol, every)
        for _ in range(steps):
            s.step_fixed(dt)
        qq, aa, _ = s.get_state()
        stats = s.hybrid_stats() if params is not None else None
    return qq, aa, stats


def test_face_samples_match_oracle(M, oracle):
    p = P.orszag_tang_params(n=40)
    p.my = 36
    rng = np.random.default_rng(2)
    q, aux = oracle.mhd_set_bnd(p, *P.mhd_random_state(p, rng, amp=0.6))
    Xo, yo = oracle.mhd_face_samples(p, q)
    with M.MhdSolver(p) as s:
        s.set_state(q, aux)
        X, y = s.face_samples()
    assert len(y) == len(yo)
    assert np.mean(y == yo) >= 0.995
    close = np.all(np.abs(X - Xo) <= 2e-3, axis=1)
    assert np.mean(close) >= 0.99


def test_no_face_troubled_is_linear_fd5(M, oracle):
    """zthr = +inf: every face takes the component-wise linear flux, which
    equals the characteristic FD5 (WenoReconstruct_FD5) of the FP32 form."""
    p = P.orszag_tang_params(n=48, weno=FIN_WENO_FD)
    q, aux = oracle.orszag_tang(p)
    dt = M.first_dt(p, q)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    pf = p.copy(); pf.precision = FIN_PREC_FP32
    from finess_b200.indicator import MLP
    npar = MLP(seed=0).nparam
    qh, ah, st = _run(M, ph, q, aux, dt, 3, np.zeros(npar, np.float32), zthr=1e30)
    qf, af, _ = _run(M, pf, q, aux, dt, 3)
    assert st["troubled_faces"] == 0
    assert rel_linf(interior(p, qh), interior(p, qf)) < 2e-5
    assert rel_linf(interior(p, ah), interior(p, af)) < 2e-5


def test_every_face_troubled_is_full_weno(M, oracle):
    from finess_b200.indicator import MLP
    npar = MLP(seed=0).nparam
    p = P.orszag_tang_params(n=48, weno=FIN_WENO_JS)
    q, aux = oracle.orszag_tang(p)
    dt = M.first_dt(p, q)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    pf = p.copy(); pf.precision = FIN_PREC_FP32
    qh, ah, st = _run(M, ph, q, aux, dt, 3, np.zeros(npar, np.float32), zthr=-1e30)
    qf, af, _ = _run(M, pf, q, aux, dt, 3)
    assert st["troubled_faces"] == st["faces"] > 0
    assert rel_linf(interior(p, qh), interior(p, qf)) < 1e-6


def test_judge_reverts_to_full_weno(M, oracle):
    """judge_tol = 0 and judge_every = 1: every hybrid step is judged and
    reverted (256^2, where the network leaves faces smooth), so the run
    equals the FP32 full-WENO form bit for bit."""
    params, zthr = _weights()
    p = P.orszag_tang_params(n=256)
    q, aux = oracle.orszag_tang(p)
    dt = M.first_dt(p, q)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    pf = p.copy(); pf.precision = FIN_PREC_FP32
    qh, _, st = _run(M, ph, q, aux, dt, 4, params, zthr=zthr, judge_every=1, judge_tol=0.0)
    qf, _, _ = _run(M, pf, q, aux, dt, 4)
    assert st["judges"] >= 2 and st["reverts"] == st["judges"]
    assert np.array_equal(interior(p, qh), interior(p, qf))


def test_trained_network_accuracy(M, oracle):
    """Orszag-Tang 256^2 to t = 0.5: the hybrid form's density error against
    the FP64 form stays at the FP32 form's level."""
    params, zthr = _weights()
    p = P.orszag_tang_params(n=256)
    q0, aux0 = P.orszag_tang_init(p)
    dt0 = M.first_dt(p, q0)
    out = {}
    for name, prec in (("fp64", FIN_PREC_FP64), ("fp32", FIN_PREC_FP32), ("hyb", FIN_PREC_HYBRID)):
        pp = p.copy(); pp.precision = prec
        with M.MhdSolver(pp) as s:
            s.set_state(q0, aux0)
            if prec == FIN_PREC_HYBRID:
                s.set_indicator(params, zthr, 50, 1e-3, 2)
            s.FinSolveRK(0.5, np.array([0.0, dt0, pp.max_dt]))
            out[name] = s.get_state()[0]
            if prec == FIN_PREC_HYBRID:
                st = s.hybrid_stats()
                assert st["troubled_faces"] < st["faces"]
            assert s.div_b() < 1e-9
    l1_32, _ = P.density_errors(p, out["fp32"], out["fp64"])
    l1_h, linf_h = P.density_errors(p, out["hyb"], out["fp64"])
    assert l1_h < 1e-4, (l1_h, l1_32)
    assert linf_h < 5e-2
