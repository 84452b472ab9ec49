"""Plain FP64 CUDA path against the reference's own compiled code at the full
sizes of the benchmark configurations (the other parity tests stop at
128^2).  The reference runs live on the host (oracle/_ref/libfinref.so and
libfinref_mhd.so, OpenMP over all host threads); skipped where it was not
built.

* isentropic vortex, 200^2, WENO5-JS, SSP-RK3 at CFL 0.4 to t = 10 (one
  period): the whole adaptive run, frame at 1e-11 relative L-infinity, the
  same number of accepted steps and the same final time;
* four-quadrant Riemann problem, 4096^2, WENO5-Z, transmissive: one
  ConstructL and one fixed-dt SSP-RK3 step at 1e-12, from a state evolved on
  the GPU to t = 0.02 (so the waves, not only the initial jumps, are tested);
* shock / entropy-wave interaction, 8192 x 1024, WENO5-JS, transmissive in
  x and periodic in y: one ConstructL and one SSP-RK3 step at 1e-12;
* ideal MHD Orszag-Tang, 2048^2, WENO5-JS, periodic, from the reference's own
  QinitFunc: one ConstructL (with the A3 Hamilton-Jacobi right-hand side) and
  one SSP-RK3 step with constrained transport at 1e-12 (ConstructL: at 1e-12
  or the reference's own one-ulp sensitivity at this size, whichever is
  larger).

Each test records its measured error: with FIN_PARITY_REPORT set to a file
path, one JSON line per measurement is appended there.
"""
import json
import os

import numpy as np

import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_WENO_JS, FIN_WENO_Z

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_FRAME = 1e-11


def _report(case, **vals):
    line = {"case": case, **vals}
    print(json.dumps(line))
    path = os.environ.get("FIN_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(line) + "\n")


def _first_dt(p, a1, a2):
    return p.desired_cfl * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / max(a1, a2)


def test_vortex200_whole_run_to_t10(reflib):
    from finess_b200.solver import Solver
    p = P.vortex_params(n=200, weno=FIN_WENO_JS)
    q0 = reflib.set_bnd(p, P.vortex_exact(p))
    a1, a2 = reflib.global_wave_spd(p, q0)
    dt0 = _first_dt(p, a1, a2)
    rc, qr, tr, dtr = reflib.finsolve(p, q0, 0.0, 10.0, dt0)
    nr = reflib.last_steps
    assert rc == 0
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        dtv, ng = s.FinSolveRK(10.0, [0.0, dt0, p.max_dt])
        qg, tg = s.get_state()
    err = rel_linf(interior(p, qg), interior(p, qr))
    _report("vortex200_js_rk3_t10", steps_gpu=ng, steps_ref=nr, rel_linf=err, t_gpu=tg, t_ref=tr,
            dt_rel=abs(dtv[1] - dtr) / dtr)
    assert ng == nr
    assert abs(tg - tr) <= 1e-14 * tr
    assert err <= TOL_FRAME
    assert abs(dtv[1] - dtr) <= 1e-10 * dtr


def _construct_l_and_step(reflib, p, q, case):
    """One ConstructL and one fixed-dt SSP-RK3 step of both implementations
    from the same ghosted state q (ghosts filled by the reference)."""
    from finess_b200.solver import Solver
    q = reflib.set_bnd(p, q)
    Lr, smr = reflib.construct_l(p, q)
    a1, a2 = reflib.global_wave_spd(p, q)
    dt = 0.5 * _first_dt(p, a1, a2)
    rc, q1r, t1r, _ = reflib.finsolve(p, q, 0.0, dt, dt)
    assert rc == 0 and reflib.last_steps == 1
    with Solver(p) as s:
        Lg, smg = s.ConstructL(q)
        s.set_state(q, 0.0)
        s.step_fixed(dt)
        q1g, t1g = s.get_state()
    eL = rel_linf(interior(p, Lg), interior(p, Lr))
    es = rel_linf(smg, smr)
    eq = rel_linf(interior(p, q1g), interior(p, q1r))
    _report(case, grid=f"{p.mx}x{p.my}", construct_l_rel_linf=eL, smax_rel_linf=es, step_rel_linf=eq, dt=dt)
    assert eL <= TOL_STEP
    assert es <= 1e-14
    assert eq <= TOL_STEP
    assert abs(t1g - t1r) <= 1e-14 * t1r


def test_riemann4096_construct_l_and_step(reflib):
    from finess_b200.solver import Solver
    p = P.riemann_params(n=4096, weno=FIN_WENO_Z)
    q0 = P.riemann_init(p)
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        a1, a2 = s.GlobalWaveSpd(q0)
        s.FinSolveRK(0.02, [0.0, _first_dt(p, a1, a2), p.max_dt])
        q, _ = s.get_state()
    _construct_l_and_step(reflib, p, q, "riemann4096_z_t0.02")


def test_shock_entropy8192x1024_construct_l_and_step(reflib):
    p = P.shock_entropy_params(nx=8192, ny=1024, weno=FIN_WENO_JS)
    _construct_l_and_step(reflib, p, P.shock_entropy_init(p), "shock_entropy8192x1024_js_t0")


def test_orszag_tang2048_construct_l_and_step():
    from oracle import MhdRefLib
    if not MhdRefLib.available():
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    from finess_b200.mhd import MhdSolver, first_dt
    ref = MhdRefLib()
    p = P.orszag_tang_params(n=2048, weno=FIN_WENO_JS)
    q, aux = ref.qinit(p)
    q, aux = ref.set_bnd(p, q, aux)
    Lr, smr = ref.construct_l(p, q, aux)
    Lar = ref.construct_hj_l(p, q, aux)
    dt = 0.5 * first_dt(p, q)
    rc, q1r, a1r, t1r, _ = ref.finsolve(p, q, aux, 0.0, dt, dt)
    assert rc == 0
    with MhdSolver(p) as s:
        Lg, smg = s.ConstructL(q, aux)
        Lag = s.ConstructHJ_L(q, aux)
        s.set_state(q, aux, 0.0)
        s.step_fixed(dt)
        q1g, a1g, t1g = s.get_state()
    eL = rel_linf(interior(p, Lg), interior(p, Lr))
    ea = rel_linf(interior(p, Lag), interior(p, Lar))
    eq = rel_linf(interior(p, q1g), interior(p, q1r))
    eaux = rel_linf(interior(p, a1g), interior(p, a1r))
    # The reference's own sensitivity at this size: its ConstructL of the
    # state with every interior value moved by one ulp (up or down at
    # random).  The initial density is uniform, so rho's right-hand side is
    # rounding noise and the 8 x 8 projections meet degenerate states on
    # whole grid lines; one ulp of input moves the reference's L by ~2e-12.
    rng = np.random.default_rng(1)
    qp = q.copy()
    I = qp[p.mbc:p.mbc + p.mx, p.mbc:p.mbc + p.my]
    I[...] = np.where(rng.random(I.shape) < 0.5, np.nextafter(I, np.inf), np.nextafter(I, -np.inf))
    qp, auxp = ref.set_bnd(p, qp, aux)
    Lp, _ = ref.construct_l(p, qp, auxp)
    sens = rel_linf(interior(p, Lp), interior(p, Lr))
    _report("orszag_tang2048_js", construct_l_rel_linf=eL, reference_one_ulp_sensitivity=sens, hj_rel_linf=ea,
            smax_rel_linf=rel_linf(smg, smr), step_rel_linf=eq, step_aux_rel_linf=eaux, dt=dt)
    assert eL <= max(TOL_STEP, sens)
    assert ea <= TOL_STEP
    assert rel_linf(smg, smr) <= TOL_STEP
    assert eq <= TOL_STEP and eaux <= TOL_STEP
