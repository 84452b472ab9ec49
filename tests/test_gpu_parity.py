"""CUDA path (through the C ABI) against the oracle and the reference's golden
fixtures.  Tolerances, all relative L-infinity (max|a-b| / max|b|):

* plain FP64 form: 1e-12 per ConstructL and per time step (the bar for the
  plain method); FinSolveRK frames, whose adaptive dt follows the CFL of
  every step, to 1e-11;
* FP32-bulk form: stated per test against the FP64 result.
"""
import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import (FIN_BC_PERIODIC, FIN_PREC_FP32, FIN_PREC_FP64, FIN_WENO_FD, FIN_WENO_JS,
                              FIN_WENO_Z)

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_FRAME = 1e-11


@pytest.fixture(scope="module")
def Solver():
    from finess_b200.solver import Solver as S
    return S


@pytest.mark.parametrize("path", golden_cases("constructl_"))
def test_construct_l_golden(Solver, path):
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        L, smax = s.ConstructL(g["q"])
        a1, a2 = s.GlobalWaveSpd(g["q"])
    assert rel_linf(interior(p, L), interior(p, g["L"])) <= TOL_STEP
    assert rel_linf(smax, g["smax"]) <= 1e-14
    assert abs(a1 - g["alpha"][0]) <= 1e-15 * g["alpha"][0]
    assert abs(a2 - g["alpha"][1]) <= 1e-15 * g["alpha"][1]


@pytest.mark.parametrize("path", golden_cases("finsolverk_"))
def test_finsolve_rk_golden(Solver, path):
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        s.set_state(g["q0"], float(g["t0"]))
        dtv, n = s.FinSolveRK(float(g["tend"]), [0.0, float(g["dt0"]), p.max_dt])
        q1, t1 = s.get_state()
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= TOL_FRAME
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dtv[1] - float(g["dt1"])) <= 1e-10 * float(g["dt1"])


@pytest.mark.parametrize("weno", [FIN_WENO_JS, FIN_WENO_Z, FIN_WENO_FD])
@pytest.mark.parametrize("kind", ["riemann", "smooth", "shock_entropy"])
def test_step_vs_oracle(Solver, oracle, weno, kind):
    """Three RK3 steps of fixed dt on ragged grids (sizes not multiples of the tile)."""
    rng = np.random.default_rng(11)
    if kind == "riemann":
        p = P.riemann_params(n=45, weno=weno)
        p.my = 37
        q = P.random_riemann_state(p, rng)
    elif kind == "smooth":
        p = P.vortex_params(n=33, weno=weno)
        p.my = 50
        q = P.random_smooth_state(p, rng)
    else:
        p = P.shock_entropy_params(nx=70, ny=17, weno=weno)
        q = P.shock_entropy_init(p)
    q = oracle.set_bnd(p, q)
    dt = 0.2 * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / 4.0
    from finess_b200.solver import FinError
    with Solver(p) as s:
        s.set_state(q)
        qo = q
        for _ in range(3):
            qo, cfl_o = oracle.step_fixed(p, qo, dt)
            if not np.all(np.isfinite(interior(p, qo))):
                # FD5 (linear weights, no limiting) at a jump goes negative and
                # NaN in the reference too; the C ABI reports it as an error.
                with pytest.raises(FinError) as ei:
                    s.step_fixed(dt)
                assert ei.value.code == 7
                assert weno == FIN_WENO_FD
                return
            cfl_g = s.step_fixed(dt)
            qg, _ = s.get_state()
            assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL_STEP
            assert abs(cfl_g - cfl_o) <= 1e-14 * cfl_o


def test_local_alpha_and_power(Solver, oracle):
    """global_alpha off (pure local LLF) and a non-default WENO power."""
    rng = np.random.default_rng(3)
    p = P.riemann_params(n=30, weno=FIN_WENO_JS, global_alpha=0, power_param=1.5)
    q = oracle.set_bnd(p, P.random_riemann_state(p, rng))
    with Solver(p) as s:
        L, smax = s.ConstructL(q)
    Lo, so = oracle.construct_l(p, q)
    assert rel_linf(interior(p, L), interior(p, Lo)) <= TOL_STEP
    assert rel_linf(smax, so) <= 1e-14


def test_tiny_and_single_row_grids(Solver, oracle):
    """Edge sizes: grids smaller than one tile, a single row (transmissive)."""
    rng = np.random.default_rng(5)
    for mx, my in ((3, 3), (1, 9), (9, 1), (17, 2)):
        p = P.riemann_params(n=mx, weno=FIN_WENO_Z)
        p.my = my
        q = oracle.set_bnd(p, P.random_riemann_state(p, rng))
        with Solver(p) as s:
            L, smax = s.ConstructL(q)
        Lo, so = oracle.construct_l(p, q)
        assert rel_linf(interior(p, L), interior(p, Lo)) <= TOL_STEP, (mx, my)
        assert rel_linf(smax, so) <= 1e-14


def test_parity_128_riemann_frame(Solver, oracle):
    """A whole adaptive-dt frame at 128x128 against the oracle."""
    p = P.riemann_params(n=128, weno=FIN_WENO_Z)
    q = oracle.set_bnd(p, P.riemann_init(p))
    rc, qo, to, dto, n = oracle.finsolve(p, q, 0.0, 0.02, 1e-3)
    with Solver(p) as s:
        s.set_state(q)
        dtv, ng = s.FinSolveRK(0.02, [0.0, 1e-3, p.max_dt])
        qg, tg = s.get_state()
    assert ng == n
    assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL_FRAME


def test_periodic_conservation_and_shift(Solver):
    """Size-independent properties at 1024^2: periodic totals conserved to
    round-off, and a periodic shift of the data shifts the result exactly."""
    p = P.vortex_params(n=1024)
    q0 = P.vortex_exact(p)
    dt = 0.002
    with Solver(p) as s:
        s.set_state(q0)
        t0 = s.conservation_totals()
        for _ in range(3):
            s.step_fixed(dt)
        t1 = s.conservation_totals()
        qa, _ = s.get_state()
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.maximum(1.0, np.abs(t0)))
    mb = p.mbc
    qs = q0.copy()
    qs[mb:mb + p.mx, mb:mb + p.my] = np.roll(interior(p, q0), (37, -101), axis=(0, 1))
    with Solver(p) as s:
        s.set_state(qs)
        for _ in range(3):
            s.step_fixed(dt)
        qb, _ = s.get_state()
    assert np.array_equal(interior(p, qb), np.roll(interior(p, qa), (37, -101), axis=(0, 1)))


@pytest.mark.parametrize("weno", [FIN_WENO_JS, FIN_WENO_Z])
def test_fp32_bulk_vs_fp64(Solver, weno):
    """FP32 reconstruction/splitting/projection with FP64 state: per-step
    relative L-infinity against the FP64 form below 1e-5."""
    p64 = P.riemann_params(n=96, weno=weno)
    q = P.riemann_init(p64)
    p32 = p64.copy()
    p32.precision = FIN_PREC_FP32
    dt = 2e-4
    with Solver(p64) as a, Solver(p32) as b:
        a.set_state(q)
        b.set_state(q)
        for _ in range(5):
            a.step_fixed(dt)
            b.step_fixed(dt)
        qa, _ = a.get_state()
        qb, _ = b.get_state()
    err = rel_linf(interior(p64, qb), interior(p64, qa))
    assert err <= 1e-5, err


def test_oversized_first_dt_is_rejected_and_retried(Solver, oracle):
    """initial_dt above the CFL limit: the first attempt is rejected
    (FinSolveRK.cpp:343-357) and retried with dt*desired_cfl/cfl."""
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    q = oracle.set_bnd(p, P.riemann_init(p))
    rc, qo, to, dto, n = oracle.finsolve(p, q, 0.0, 0.01, 0.004)   # first CFL ~0.6 > max_cfl 0.45
    with Solver(p) as s:
        s.set_state(q)
        dtv, ng = s.FinSolveRK(0.01, [0.0, 0.004, p.max_dt])
        qg, tg = s.get_state()
    assert rc == 0 and ng == n
    assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL_FRAME
    assert abs(dtv[1] - dto) <= 1e-10 * dto


def test_nan_producing_attempt_is_rejected_not_fatal(Solver):
    """A first dt so large that the attempt produces NaNs (CFL ~80): the
    reference's GetCFL skips NaN faces, rejects the step and retries; so does
    the C ABI, which only reports an error if such a step would be accepted."""
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    q = P.riemann_init(p)
    with Solver(p) as s:
        s.set_state(q)
        dtv, ng = s.FinSolveRK(0.01, [0.0, 0.5, p.max_dt])
        qg, tg = s.get_state()
    assert ng > 0 and abs(tg - 0.01) < 1e-12
    assert np.all(np.isfinite(interior(p, qg)))


# ---------------------------------------------------------------------------
# Lax-Wendroff / two-stage multiderivative path
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("path", golden_cases("intr_"))
def test_integrated_flux_golden(Solver, path):
    from finess_b200._abi import FIN_TS_LXW
    g = load_golden(path)
    p = g["p"]
    if p.time_order != 4:
        p.time_stepping_method = FIN_TS_LXW   # MD is built for time_order 4; LxW takes any order
    with Solver(p) as s:
        F, G = s.ConstructIntegratedR(float(g["dt"]), g["q"])
    mb = p.mbc
    E = (slice(mb - 3, mb + p.mx + 3), slice(mb - 3, mb + p.my + 3))
    assert rel_linf(F[E], g["F"][E]) <= TOL_STEP
    assert rel_linf(G[E], g["G"][E]) <= TOL_STEP


@pytest.mark.parametrize("path", golden_cases("finsolvemd_") + golden_cases("finsolvelxw_"))
def test_finsolve_md_lxw_golden(Solver, path):
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        s.set_state(g["q0"], float(g["t0"]))
        dtv, n = s.FinSolveMD(float(g["tend"]), [0.0, float(g["dt0"]), p.max_dt])
        q1, t1 = s.get_state()
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= TOL_FRAME
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dtv[1] - float(g["dt1"])) <= 1e-10 * float(g["dt1"])


@pytest.mark.parametrize("method", ["md", "lxw"])
@pytest.mark.parametrize("kind", ["riemann", "smooth"])
def test_md_lxw_steps_vs_oracle(Solver, oracle, method, kind):
    """Two fixed-dt steps on ragged grids, against the oracle, per step."""
    from finess_b200._abi import FIN_BC_PERIODIC, FIN_TS_LXW, FIN_TS_MD
    rng = np.random.default_rng(21)
    p = P.riemann_params(n=41, weno=FIN_WENO_Z, method=FIN_TS_MD)
    p.my = 35
    if method == "lxw":
        p.time_stepping_method = FIN_TS_LXW
        p.time_order = 3
    if kind == "smooth":
        p.bc_xlow = p.bc_xhigh = p.bc_ylow = p.bc_yhigh = FIN_BC_PERIODIC
        q = P.random_smooth_state(p, rng)
    else:
        q = P.random_riemann_state(p, rng)
    q = oracle.set_bnd(p, q)
    dt = 0.15 / 41 / 3.0
    with Solver(p) as s:
        s.set_state(q)
        qo = q
        for _ in range(2):
            cg = s.step_fixed(dt)
            qo, co = oracle.step_fixed(p, qo, dt)
            qg, _ = s.get_state()
            assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL_STEP
            assert abs(cg - co) <= 1e-14 * co


@pytest.mark.parametrize("path", golden_cases("finsolvelxwmpp_"))
def test_finsolve_lxw_mpp_golden(Solver, path):
    """Lax-Wendroff frames with the MPP limiter (ConstructLFL,
    ApplyMPPLimiter2D, FinSolveLxW.cpp:126-151) against the reference's own
    run; in the near-vacuum case the limiter changes the frame, and the
    device matches the limited frame, not the unlimited one."""
    g = load_golden(path)
    p = g["p"]
    assert p.mpp_limiter == 1
    with Solver(p) as s:
        s.set_state(g["q0"], float(g["t0"]))
        dtv, n = s.FinSolveMD(float(g["tend"]), [0.0, float(g["dt0"]), p.max_dt])
        q1, t1 = s.get_state()
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= TOL_FRAME
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dtv[1] - float(g["dt1"])) <= 1e-10 * float(g["dt1"])
    if "rarefaction" in path:
        # without the limiter the reference's frame breaks down (NaN); with
        # it, density and pressure stay positive, here as there
        assert not np.all(np.isfinite(interior(p, g["q1_unlimited"])))
        qi = interior(p, q1)
        rho = qi[..., 0]
        pr = (p.gamma - 1) * (qi[..., 4] - 0.5 * (qi[..., 1] ** 2 + qi[..., 2] ** 2) / rho)
        assert rho.min() > 0 and pr.min() > 0


def test_lxw_mpp_live_reference(Solver):
    """One MPP Lax-Wendroff frame on a random four-quadrant state against the
    reference's FinSolveLxW run live (where oracle/_ref was built)."""
    from oracle import RefLib
    if not RefLib.available():
        pytest.skip("oracle/_ref/libfinref.so not built")
    from finess_b200._abi import FIN_TS_LXW, FIN_TS_MD
    ref = RefLib()
    p = P.riemann_params(n=33, weno=FIN_WENO_Z, method=FIN_TS_MD, time_stepping_method=FIN_TS_LXW, time_order=3,
                         mpp_limiter=1)
    p.my = 29
    q0 = ref.set_bnd(p, P.random_riemann_state(p, np.random.default_rng(77)))
    rc, q1, t1, dt1 = ref.finsolve(p, q0, 0.0, 0.03, 1e-3)
    assert rc == 0
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        dtv, n = s.FinSolveMD(0.03, [0.0, 1e-3, p.max_dt])
        q2, t2 = s.get_state()
    assert rel_linf(interior(p, q2), interior(p, q1)) <= TOL_FRAME
    assert abs(t2 - t1) <= 1e-14 * abs(t1)
    assert abs(dtv[1] - dt1) <= 1e-10 * dt1


@pytest.mark.parametrize("path", golden_cases("finsolverk1_") + golden_cases("finsolverk2_") +
                         golden_cases("finsolverk4_") + golden_cases("finsolverk5_") + golden_cases("finsolvemd5_"))
def test_finsolve_rk_orders_golden(Solver, path):
    """FinSolveRK frames with time_order 1, 2, 4 (ten-stage SSP) and 5
    (eight stages, whose UpdateSoln leaves Qnew's time at the last step's
    start), and FinSolveMD frames with time_order 5 (the three-coefficient
    ConstructIntegratedR), against the reference's own run."""
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        s.set_state(g["q0"], float(g["t0"]))
        dtv, n = s.FinSolveRK(float(g["tend"]), [0.0, float(g["dt0"]), p.max_dt])
        q1, t1 = s.get_state()
    assert n > 0
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= TOL_FRAME
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dtv[1] - float(g["dt1"])) <= 1e-10 * float(g["dt1"])


@pytest.mark.parametrize("path", golden_cases("hiorder_constructl"))
def test_construct_l_space_orders_golden(Solver, path):
    """ConstructL of the other spatial orders (LLF, JS7/9/11, Z7/9, FD7/9,
    the generic FP64 face kernel) against the reference's own output."""
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        L, smax = s.ConstructL(g["q"])
    assert rel_linf(interior(p, L), interior(p, g["L"])) <= TOL_STEP
    assert rel_linf(smax, g["smax"]) <= 1e-14


@pytest.mark.parametrize("path", golden_cases("hiorder_finsolverk"))
def test_finsolve_rk_space_orders_golden(Solver, path):
    """SSP-RK3 frames of the other spatial orders.  Bar: 1e-11, or ten times
    the reference's own sensitivity where that is larger.  The sensitivity
    (stored with each fixture) is how far the reference's frame moves when
    every value of its initial state moves by one ulp.  The smoothness
    indicators of orders 9 and 11 cancel terms with coefficients up to
    ~4e8, so on near-flat states the weights carry roundoff and those
    frames move by up to ~1e-7 from one ulp of input.  An implementation
    that is not bit-identical differs by a few times that.  The LLF and FD
    frames (sensitivity ~1e-15) keep 1e-11."""
    g = load_golden(path)
    p = g["p"]
    with Solver(p) as s:
        s.set_state(g["q0"], float(g["t0"]))
        dtv, n = s.FinSolveRK(float(g["tend"]), [0.0, float(g["dt0"]), p.max_dt])
        q1, t1 = s.get_state()
    tol = max(TOL_FRAME, 10.0 * float(g["sens"]))
    assert n > 0
    assert rel_linf(interior(p, q1), interior(p, g["q1"])) <= tol
    assert abs(t1 - float(g["t1"])) <= 1e-14 * abs(float(g["t1"]))
    assert abs(dtv[1] - float(g["dt1"])) <= max(1e-10, tol) * float(g["dt1"])


@pytest.mark.parametrize("so,weno", [(3, FIN_WENO_JS), (11, FIN_WENO_Z), (11, FIN_WENO_FD), (13, FIN_WENO_JS)])
def test_unbuilt_space_orders_are_refused(Solver, so, weno):
    """GetWenoReconstruct (lib/WenoReconstruct.cpp:40-71) throws for these."""
    p = P.riemann_params(n=16, weno=weno, space_order=so, mbc=7)
    with pytest.raises(Exception, match="not implemented"):
        Solver(p)


def test_space_order_needs_mbc(Solver):
    p = P.riemann_params(n=16, weno=FIN_WENO_JS, space_order=9, mbc=4)
    with pytest.raises(Exception, match="mbc"):
        Solver(p)
