"""Indicator features and labels on the device against the oracle's FP64
restatement (oracle_face_samples), and the hybrid form against full WENO."""
import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_PREC_FP32, FIN_PREC_HYBRID, FIN_WENO_JS, FIN_WENO_Z

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(17)
    out = []
    p = P.riemann_params(n=40, weno=FIN_WENO_JS)
    p.my = 33
    out.append((p, P.random_riemann_state(p, rng)))
    p = P.vortex_params(n=48, weno=FIN_WENO_JS)
    out.append((p, P.vortex_exact(p)))
    p = P.shock_entropy_params(nx=64, ny=12)
    out.append((p, P.shock_entropy_init(p)))
    return out


@pytest.mark.parametrize("case", range(3))
def test_features_and_labels_match_oracle(oracle, case):
    from finess_b200.solver import Solver
    p, q = _cases()[case]
    q = oracle.set_bnd(p, q)
    with Solver(p) as s:
        s.set_state(q)
        X, y = s.face_samples()
    Xo, yo = oracle.face_samples(p, q)
    assert X.shape == Xo.shape
    # FP32 features of normalised characteristic differences
    assert np.max(np.abs(X - Xo)) <= 2e-3
    # FP64 labels: equal except at faces within rounding of the 10 % threshold
    assert np.mean(y != yo) <= 0.005
    assert 0 < yo.sum() < len(yo) or case == 1


def test_hybrid_with_everything_flagged_equals_fp32_full_weno():
    """A network that flags every face (bias +10) makes the hybrid form the
    FP32 full-WENO form exactly."""
    from finess_b200.indicator import MLP
    from finess_b200.solver import Solver
    import mlp_oracle as M
    Pm = np.zeros(M.NPARAM, dtype=np.float32)
    Pm[M.OFF_B3] = 10.0
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    q = P.riemann_init(p)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    pf = p.copy(); pf.precision = FIN_PREC_FP32
    with Solver(ph) as a, Solver(pf) as b:
        a.set_indicator(Pm, 0.0, judge_every=0)
        a.set_state(q); b.set_state(q)
        for _ in range(3):
            a.step_fixed(5e-4)
            b.step_fixed(5e-4)
        qa, _ = a.get_state()
        qb, _ = b.get_state()
        st = a.hybrid_stats()
    assert st["troubled_faces"] == st["faces"]
    assert rel_linf(interior(p, qa), interior(p, qb)) <= 1e-6


def test_hybrid_with_nothing_flagged_is_linear_fd5_and_judge_reverts():
    """A network that flags nothing gives the linear FD5 scheme; on a shock
    problem the judge step sees the departure from full WENO and reverts."""
    from finess_b200.solver import Solver
    import mlp_oracle as M
    Pm = np.zeros(M.NPARAM, dtype=np.float32)
    Pm[M.OFF_B3] = -10.0
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    q = P.riemann_init(p)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    with Solver(ph) as a:
        a.set_indicator(Pm, 0.0, judge_every=1, judge_tol=1e-6)
        a.set_state(q)
        a.step_fixed(5e-4)
        st = a.hybrid_stats()
    assert st["troubled_faces"] == 0 and st["judges"] == 1 and st["reverts"] == 1
