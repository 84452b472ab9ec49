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


def test_hybrid_smooth_faces_equal_reference_fd5(oracle):
    """With nothing flagged every face takes the component-wise 6-point form of
    the linear FD5 flux.  The reference's FD5 path projects onto characteristic
    fields, reconstructs and projects back; the two agree because the
    reconstruction is linear and R L = I, so one hybrid step must match the
    oracle's FP64 weno_version=FD step to FP32 rounding."""
    from finess_b200.solver import Solver
    import mlp_oracle as M
    from finess_b200._abi import FIN_WENO_FD
    Pm = np.zeros(M.NPARAM, dtype=np.float32)
    Pm[M.OFF_B3] = -10.0
    p = P.vortex_params(n=48, weno=FIN_WENO_JS)
    q = oracle.set_bnd(p, P.vortex_exact(p))
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    dt = 0.02
    with Solver(ph) as a:
        a.set_indicator(Pm, 0.0, judge_every=0)
        a.set_state(q)
        a.step_fixed(dt)
        qa, _ = a.get_state()
        assert a.hybrid_stats()["troubled_faces"] == 0
    po = p.copy(); po.weno_version = FIN_WENO_FD
    qo, _ = oracle.step_fixed(po, q, dt)
    err = rel_linf(interior(p, qa), interior(p, qo))
    assert err <= 1e-6, err


@pytest.mark.parametrize("case", [0, 2])
def test_indicator_flags_match_oracle_network(oracle, case):
    """The device indicator (features + network on tensor cores + threshold)
    flags the same number of faces as the oracle network applied to the
    oracle's FP64 features, up to faces within rounding of the threshold."""
    from finess_b200.indicator import DEFAULT_WEIGHTS
    from finess_b200.solver import Solver
    import mlp_oracle as M
    W = np.load(DEFAULT_WEIGHTS)
    params, zthr = W["params"], float(W["z_threshold"])
    p, q = _cases()[case]
    q = oracle.set_bnd(p, q)
    Xo, _ = oracle.face_samples(p, q)
    zo = M.forward_emulated(params, Xo)
    n_oracle = int(np.sum(zo > zthr))
    near = int(np.sum(np.abs(zo - zthr) < 0.05))
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    with Solver(ph) as a:
        a.set_indicator(params, zthr, judge_every=0)
        a.set_state(q)
        a.step_fixed(1e-5)
        st = a.hybrid_stats()
    assert st["faces"] == len(Xo)
    assert abs(st["troubled_faces"] - n_oracle) <= max(near, 2), (st, n_oracle, near)


@pytest.mark.parametrize("kind", ["riemann_init", "random"])
def test_indicator_flags_face_by_face(oracle, kind):
    """Face by face, the device's flags equal the oracle network's decisions
    on the oracle's FP64 features, except faces within rounding of the
    threshold; faces whose stencil is constant (features exactly 0, which the
    kernel skips when the network's zero-row output is below the threshold)
    are never flagged."""
    from finess_b200.indicator import DEFAULT_WEIGHTS
    from finess_b200.solver import Solver
    import mlp_oracle as M
    W = np.load(DEFAULT_WEIGHTS)
    params, zthr = W["params"], float(W["z_threshold"])
    if kind == "riemann_init":
        p = P.riemann_params(n=70, weno=FIN_WENO_JS)
        p.my = 53
        q = P.riemann_init(p)
    else:
        p, q = _cases()[0]
    q = oracle.set_bnd(p, q)
    Xo, _ = oracle.face_samples(p, q)
    zo = M.forward_emulated(params, Xo)
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    with Solver(ph) as a:
        a.set_indicator(params, zthr, judge_every=0)
        a.set_state(q)
        a.step_fixed(1e-5)
        fl = a.hybrid_flags()
    assert fl.size == len(Xo)
    const = np.all(Xo == 0.0, axis=1)
    if kind == "riemann_init":
        assert const.mean() > 0.5
    assert not np.any(fl[const])
    sure = np.abs(zo - zthr) >= 0.05
    assert np.array_equal(fl[sure], (zo > zthr)[sure])


def test_hybrid_after_revert_continues_on_the_right_buffers():
    """A revert swaps the hybrid attempt's buffer with the full-WENO one; the
    hybrid steps after it must read the swapped buffers (their TMA maps travel
    with them).  Schedule with a network that flags nothing, judge every 2nd
    hybrid step at tolerance 0 (always reverts): FD5, JS, JS, JS, FD5, JS --
    replayed with FP32 solvers of the two reconstructions."""
    from finess_b200.solver import Solver
    import mlp_oracle as M
    from finess_b200._abi import FIN_WENO_FD
    Pm = np.zeros(M.NPARAM, dtype=np.float32)
    Pm[M.OFF_B3] = -10.0
    p = P.vortex_params(n=64, weno=FIN_WENO_JS)
    q0 = P.vortex_exact(p)
    dt = 0.02
    ph = p.copy(); ph.precision = FIN_PREC_HYBRID
    with Solver(ph) as a:
        a.set_indicator(Pm, 0.0, judge_every=2, judge_tol=0.0)
        a.set_state(q0)
        for _ in range(6):
            a.step_fixed(dt)
        qa, _ = a.get_state()
        st = a.hybrid_stats()
    assert st["judges"] == 2 and st["reverts"] == 2
    pf = p.copy(); pf.precision = FIN_PREC_FP32
    pd = pf.copy(); pd.weno_version = FIN_WENO_FD
    q = q0
    with Solver(pf) as js, Solver(pd) as fd:
        for form in ("FD", "JS", "JS", "JS", "FD", "JS"):
            s = fd if form == "FD" else js
            s.set_state(q)
            s.step_fixed(dt)
            q, _ = s.get_state()
    err = rel_linf(interior(p, qa), interior(p, q))
    assert err <= 1e-5, err


def test_indicator_period():
    """With period 2 the indicator runs on every other step; the flags of a
    network that flags everything give the same state either way."""
    from finess_b200.solver import Solver
    import mlp_oracle as M
    Pm = np.zeros(M.NPARAM, dtype=np.float32)
    Pm[M.OFF_B3] = 10.0
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    p.precision = FIN_PREC_HYBRID
    q0 = P.riemann_init(p)
    out = {}
    for every in (1, 2):
        with Solver(p) as a:
            a.set_indicator(Pm, 0.0, judge_every=0, every=every)
            a.set_state(q0)
            n0 = a.launch_count()
            for _ in range(4):
                a.step_fixed(5e-4)
            out[every] = (a.launch_count() - n0, a.get_state()[0])
    assert out[1][0] - out[2][0] == 2
    assert rel_linf(interior(p, out[2][1]), interior(p, out[1][1])) == 0.0
