"""Generates the golden fixtures in this directory by running the reference's
own sources (oracle/_ref/libfinref.so and libfinref_mhd.so, built by
``make -C oracle ref ref_mhd`` from the reference checkout) on small seeded
inputs.

The reference repository stores no golden vectors for this path, so these
files pin its behaviour: each .npz holds the inputs (ghosted q after the BC
remap, parameters) and the reference's outputs.  Re-run with
``python tests/golden/make_golden.py`` after ``make -C oracle ref ref_mhd`` (``... mhd`` or
``... mpp``, ``... rk`` or ``... space`` rewrites only the MHD, the MPP-limiter, the other
Runge-Kutta orders' or the other spatial orders' fixtures).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import MhdRefLib, RefLib  # noqa: E402
from finess_b200 import problems as P  # noqa: E402
from finess_b200._abi import (FIN_BC_TRANSMISSIVE, FIN_TS_LXW, FIN_TS_MD, FIN_TS_RK, FIN_WENO_FD,  # noqa: E402
                              FIN_WENO_JS, FIN_WENO_Z)


def params_json(p):
    return json.dumps(p.as_dict())


def construct_l_cases():
    rng = np.random.default_rng(20261203)
    cases = []
    for weno, wname in ((FIN_WENO_JS, "js"), (FIN_WENO_Z, "z"), (FIN_WENO_FD, "fd")):
        p = P.vortex_params(n=20, weno=weno)
        p.my = 14
        cases.append((f"constructl_{wname}_smooth_periodic", p, P.random_smooth_state(p, rng)))
        p = P.riemann_params(n=18, weno=weno)
        p.my = 22
        cases.append((f"constructl_{wname}_riemann_transmissive", p, P.random_riemann_state(p, rng)))
    # mixed boundaries and the local (non-global) LLF alpha
    p = P.shock_entropy_params(nx=24, ny=12, weno=FIN_WENO_JS)
    cases.append(("constructl_js_shock_entropy_mixed", p, P.shock_entropy_init(p)))
    p = P.riemann_params(n=16, weno=FIN_WENO_Z, global_alpha=0)
    cases.append(("constructl_z_riemann_local_alpha", p, P.riemann_init(p)))
    return cases


def main():
    ref = RefLib()
    # ConstructIntegratedR, 1-state, with (time_order 4) and without
    # (time_order 2) the Hessian terms.
    rng = np.random.default_rng(99)
    for to, kind in ((4, "riemann"), (2, "riemann"), (4, "smooth")):
        p = P.riemann_params(n=16, weno=FIN_WENO_Z, method=FIN_TS_MD, time_order=to)
        p.my = 13
        if kind == "smooth":
            from finess_b200._abi import FIN_BC_PERIODIC
            p.bc_xlow = p.bc_xhigh = p.bc_ylow = p.bc_yhigh = FIN_BC_PERIODIC
            q = P.random_smooth_state(p, rng)
        else:
            q = P.random_riemann_state(p, rng)
        q = ref.set_bnd(p, q)
        F, G = ref.construct_integrated_r(p, 0.004, q)
        name = f"intr_t{to}_{kind}"
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q=q, F=F, G=G, dt=0.004)
        print("wrote", name)
    for name, p, q in construct_l_cases():
        q = ref.set_bnd(p, q)
        L, smax = ref.construct_l(p, q)
        a1, a2 = ref.global_wave_spd(p, q)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q=q, L=L, smax=smax,
                            alpha=np.array([a1, a2]))
        print("wrote", name)

    # Whole FinSolveRK frames (adaptive dt, accept/reject) on small grids.
    runs = []
    p = P.vortex_params(n=24, weno=FIN_WENO_JS)
    runs.append(("finsolverk_js_vortex24", p, P.vortex_exact(p), 0.0, 0.5, 0.05))
    p = P.riemann_params(n=32, weno=FIN_WENO_Z)
    runs.append(("finsolverk_z_riemann32", p, P.riemann_init(p), 0.0, 0.05, 1e-3))
    # a large initial dt forces step rejections (FinSolveRK.cpp:343-357)
    p = P.riemann_params(n=20, weno=FIN_WENO_JS)
    runs.append(("finsolverk_js_riemann20_reject", p, P.riemann_init(p), 0.0, 0.03, 0.05))
    # Two-stage multiderivative (FinSolveMD, time_order 4) and single-stage
    # Lax-Wendroff (FinSolveLxW) frames; both need mbc = 5.
    p = P.riemann_params(n=24, weno=FIN_WENO_Z, method=FIN_TS_MD)
    p.my = 20
    runs.append(("finsolvemd_z_riemann24", p, P.riemann_init(p), 0.0, 0.02, 1e-3))
    p = P.vortex_params(n=20, weno=FIN_WENO_JS, mbc=5, time_stepping_method=FIN_TS_MD, time_order=4)
    runs.append(("finsolvemd_js_vortex20", p, P.vortex_exact(p), 0.0, 0.3, 0.05))
    p = P.riemann_params(n=22, weno=FIN_WENO_JS, method=FIN_TS_MD, time_stepping_method=FIN_TS_LXW,
                         time_order=3)
    runs.append(("finsolvelxw_js_riemann22", p, P.riemann_init(p), 0.0, 0.02, 1e-3))
    for name, p, q0, t0, tend, dt in runs:
        q0 = ref.set_bnd(p, q0)
        rc, q1, t1, dt1 = ref.finsolve(p, q0, t0, tend, dt)
        assert rc == 0
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q0=q0, q1=q1,
                            t0=t0, t1=t1, tend=tend, dt0=dt, dt1=dt1)
        print("wrote", name, t1, dt1)
    mhd_main()


def mhd_main():
    """Ideal MHD (apps/2d/mhd/lib with the Orszag-Tang case): ConstructL with
    the MHD callbacks, ConstructHJ_L_Order1, AfterStep's constrained
    transport, and whole FinSolveRK frames."""
    ref = MhdRefLib()
    rng = np.random.default_rng(20261204)
    cases = []
    p = P.orszag_tang_params(n=24, weno=FIN_WENO_JS)
    cases.append(("mhd_constructl_js_ot24_local", p, ref.qinit(p)))
    p = P.orszag_tang_params(n=20, weno=FIN_WENO_Z, global_alpha=1)
    p.my = 18
    p.yhigh = 2.0
    cases.append(("mhd_constructl_z_random20x18_global", p, P.mhd_random_state(p, rng)))
    for name, p, (q, aux) in cases:
        q, aux = ref.set_bnd(p, q, aux)
        L, smax = ref.construct_l(p, q, aux)
        La = ref.construct_hj_l(p, q, aux)
        qct = ref.after_step(p, q, aux)
        a1, a2 = ref.global_wave_spd(p, q, aux)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q=q, aux=aux, L=L,
                            smax=smax, Laux=La, qct=qct, alpha=np.array([a1, a2]))
        print("wrote", name)
    runs = []
    p = P.orszag_tang_params(n=24, weno=FIN_WENO_JS)
    runs.append(("mhd_finsolverk_js_ot24", p, 0.0, 0.08, 1e-3))
    # a large initial dt forces step rejections (FinSolveRK.cpp:343-357 of the MHD app)
    p = P.orszag_tang_params(n=20, weno=FIN_WENO_Z)
    runs.append(("mhd_finsolverk_z_ot20_reject", p, 0.0, 0.05, 0.2))
    for name, p, t0, tend, dt in runs:
        q0, aux0 = ref.set_bnd(p, *ref.qinit(p))
        rc, q1, aux1, t1, dt1 = ref.finsolve(p, q0, aux0, t0, tend, dt)
        assert rc == 0
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q0=q0, aux0=aux0, q1=q1,
                            aux1=aux1, t0=t0, t1=t1, tend=tend, dt0=dt, dt1=dt1)
        print("wrote", name, t1, dt1)


def mpp_main():
    """Lax-Wendroff frames with the MPP limiter (FinSolveLxW.cpp:126-151:
    ConstructLxWL's fluxes, ConstructLFL, ApplyMPPLimiter2D): the
    four-quadrant Riemann problem and a near-vacuum double rarefaction."""
    ref = RefLib()
    runs = []
    p = P.riemann_params(n=22, weno=FIN_WENO_JS, method=FIN_TS_MD, time_stepping_method=FIN_TS_LXW,
                         time_order=3, mpp_limiter=1)
    runs.append(("finsolvelxwmpp_js_riemann22", p, P.riemann_init(p), 0.0, 0.02, 1e-3))
    p = P.riemann_params(n=26, weno=FIN_WENO_Z, method=FIN_TS_MD, time_stepping_method=FIN_TS_LXW,
                         time_order=3, mpp_limiter=1)
    p.my = 12
    # strong enough that the unlimited method breaks down (NaN) by t = 0.05
    runs.append(("finsolvelxwmpp_z_rarefaction26", p, P.double_rarefaction_init(p, speed=3.0, pr=0.2), 0.0, 0.05,
                 1e-3))
    for name, p, q0, t0, tend, dt in runs:
        q0 = ref.set_bnd(p, q0)
        rc, q1, t1, dt1 = ref.finsolve(p, q0, t0, tend, dt)
        assert rc == 0
        p_off = p.copy()
        p_off.mpp_limiter = 0
        _, q_off, _, _ = ref.finsolve(p_off, q0, t0, tend, dt)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q0=q0, q1=q1,
                            t0=t0, t1=t1, tend=tend, dt0=dt, dt1=dt1, q1_unlimited=q_off)
        mb = p.mbc
        gap = np.abs(q1 - q_off)[mb:mb + p.mx, mb:mb + p.my].max()
        print("wrote", name, t1, dt1, "limiter changed the interior by", float(gap))


def rk_orders_main():
    """FinSolveRK frames of the other Runge-Kutta orders (FinSolveRK.cpp:
    117-299): forward Euler, SSP-RK2, the ten-stage SSP-RK4 and the
    eight-stage fifth-order method."""
    ref = RefLib()
    runs = []
    for order, weno, wname in ((1, FIN_WENO_JS, "js"), (2, FIN_WENO_Z, "z"), (4, FIN_WENO_JS, "js"),
                               (5, FIN_WENO_Z, "z")):
        p = P.riemann_params(n=24, weno=weno, time_order=order)
        p.my = 20
        runs.append((f"finsolverk{order}_{wname}_riemann24", p, P.riemann_init(p), 0.0, 0.03, 1e-3))
        p = P.vortex_params(n=20, weno=weno, time_order=order, global_alpha=1)
        runs.append((f"finsolverk{order}_{wname}_vortex20", p, P.vortex_exact(p), 0.0, 0.3, 0.05))
    # the fifth-order two-stage multiderivative method (FinSolveMD.cpp:172-226)
    p = P.riemann_params(n=24, weno=FIN_WENO_Z, method=FIN_TS_MD, time_order=5)
    p.my = 20
    runs.append(("finsolvemd5_z_riemann24", p, P.riemann_init(p), 0.0, 0.02, 1e-3))
    p = P.vortex_params(n=20, weno=FIN_WENO_JS, mbc=5, time_stepping_method=FIN_TS_MD, time_order=5)
    runs.append(("finsolvemd5_js_vortex20", p, P.vortex_exact(p), 0.0, 0.3, 0.05))
    for name, p, q0, t0, tend, dt in runs:
        q0 = ref.set_bnd(p, q0)
        rc, q1, t1, dt1 = ref.finsolve(p, q0, t0, tend, dt)
        assert rc == 0
        np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q0=q0, q1=q1,
                            t0=t0, t1=t1, tend=tend, dt0=dt, dt1=dt1)
        print("wrote", name, t1, dt1)


SPACE_ORDERS = ((1, FIN_WENO_JS, "js"), (7, FIN_WENO_JS, "js"), (7, FIN_WENO_Z, "z"), (7, FIN_WENO_FD, "fd"),
                (9, FIN_WENO_JS, "js"), (9, FIN_WENO_Z, "z"), (9, FIN_WENO_FD, "fd"), (11, FIN_WENO_JS, "js"))


def space_orders_main():
    """ConstructL and FinSolveRK (SSP-RK3) of the other spatial orders that
    GetWenoReconstruct accepts (lib/WenoReconstruct.cpp:40-71): LLF (order 1),
    JS7/9/11, Z7/9 and FD7/9, each with mbc = r = (order + 1) / 2 (order 1
    keeps mbc 3)."""
    ref = RefLib()
    rng = np.random.default_rng(7911)
    for so, weno, wname in SPACE_ORDERS:
        mbc = max(3, (so + 1) // 2)
        cases = []
        p = P.vortex_params(n=22, weno=weno, space_order=so, mbc=mbc)
        p.my = 16
        cases.append((f"hiorder_constructl{so}_{wname}_smooth_periodic", p, P.random_smooth_state(p, rng)))
        p = P.riemann_params(n=18, weno=weno, space_order=so, mbc=mbc, global_alpha=0)
        p.my = 24
        cases.append((f"hiorder_constructl{so}_{wname}_riemann_local_alpha", p, P.random_riemann_state(p, rng)))
        for name, p, q in cases:
            q = ref.set_bnd(p, q)
            L, smax = ref.construct_l(p, q)
            a1, a2 = ref.global_wave_spd(p, q)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q=q, L=L, smax=smax,
                                alpha=np.array([a1, a2]))
            print("wrote", name)
        runs = []
        p = P.riemann_params(n=24, weno=weno, space_order=so, mbc=mbc)
        p.my = 20
        # linear weights oscillate at the shocks and the reference's own run
        # loses positivity by t = 0.01 (FD7) / 0.015 (FD9): stop before that
        tend = 0.005 if weno == FIN_WENO_FD else 0.03
        runs.append((f"hiorder_finsolverk{so}_{wname}_riemann24", p, P.riemann_init(p), 0.0, tend, 1e-3))
        p = P.vortex_params(n=20, weno=weno, space_order=so, mbc=mbc)
        runs.append((f"hiorder_finsolverk{so}_{wname}_vortex20", p, P.vortex_exact(p), 0.0, 0.3, 0.05))
        for name, p, q0, t0, tend, dt in runs:
            q0 = ref.set_bnd(p, q0)
            rc, q1, t1, dt1 = ref.finsolve(p, q0, t0, tend, dt)
            assert rc == 0
            # FinSolveRK fills no ghost cells after the last update, so with
            # mbc > 3 the outer layers of its frame are left-over heap data:
            # store the frame with its ghosts refilled (tests compare interiors)
            q1 = ref.set_bnd(p, q1)
            assert np.isfinite(q1).all(), name
            # The reference's own sensitivity: how far its frame moves when
            # every value of q0 moves by one ulp (largest of three seeded
            # perturbations).  The high-order smoothness indicators cancel
            # terms with coefficients up to ~4e8, so near-flat states put
            # roundoff into the weights and the orders 9 and 11 frames move
            # by up to ~1e-7.
            sens = 0.0
            prng = np.random.default_rng(1234)
            for _ in range(3):
                up = prng.random(q0.shape) < 0.5
                qp = ref.set_bnd(p, np.where(up, np.nextafter(q0, np.inf), np.nextafter(q0, -np.inf)))
                rcp_, qp1, _, _ = ref.finsolve(p, qp, t0, tend, dt)
                assert rcp_ == 0
                m = mbc
                a, b = qp1[m:m + p.mx, m:m + p.my], q1[m:m + p.mx, m:m + p.my]
                sens = max(sens, float(np.abs(a - b).max() / np.abs(b).max()))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), params=params_json(p), q0=q0, q1=q1,
                                t0=t0, t1=t1, tend=tend, dt0=dt, dt1=dt1, sens=sens)
            print("wrote", name, t1, dt1, "sensitivity", sens)


if __name__ == "__main__":
    if sys.argv[1:] == ["space"]:
        space_orders_main()
    elif sys.argv[1:] == ["mhd"]:
        mhd_main()
    elif sys.argv[1:] == ["mpp"]:
        mpp_main()
    elif sys.argv[1:] == ["rk"]:
        rk_orders_main()
    else:
        main()
