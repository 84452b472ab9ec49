"""The application callback surface on the device (fin_physics.cuh,
fin_physics_host.h): physics policies an application writes, built into the
application's own library (tests/apps/phys_app.cu -> libfin_phys_app.so),
against the generic restatement of ConstructL / SSP-RK3
(oracle/generic_oracle.py, pinned to the reference's fixtures on the CPU).

* a third physics, linear advection-acoustics (meqn 3), through the same
  template: ConstructL and three SSP-RK3 steps for WENO-JS, Z and FD, on
  ragged grids, periodic and transmissive, with the hooks of lib/2d/hooks.h;
* the library's Euler callbacks as a policy through the same template,
  against the golden fixtures, the C restatement and the specialised kernel.

Bar: 1e-12 relative L-infinity per evaluation or step (the plain method's)."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, golden_cases, interior, load_golden, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_BC_PERIODIC, FIN_BC_TRANSMISSIVE, FIN_OK, FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z, \
    FinParams

pytestmark = pytest.mark.gpu
TOL = 1e-12
APP_SO = os.path.join(ROOT, "tests", "apps", "libfin_phys_app.so")
ACOUSTICS = (4.0, 1.5, 0.4, -0.25)   # K, rho0, ax, ay
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def app():
    lib = C.CDLL(APP_SO)     # built by __graft_entry__.build(); fails loudly when missing
    vp = C.c_void_p
    lib.app_create.argtypes = [C.c_int, C.POINTER(FinParams), C.c_void_p, C.POINTER(vp)]
    lib.app_destroy.argtypes = [vp]
    lib.app_set_state.argtypes = [vp, _dp, C.c_double]
    lib.app_get_state.argtypes = [vp, _dp, C.POINTER(C.c_double)]
    lib.app_construct_l.argtypes = [vp, _dp, _dp, C.c_void_p]
    lib.app_global_wave_spd.argtypes = [vp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.app_step_fixed.argtypes = [vp, C.c_double, C.POINTER(C.c_double)]
    for n in ("app_create", "app_destroy", "app_set_state", "app_get_state", "app_construct_l",
              "app_global_wave_spd", "app_step_fixed"):
        getattr(lib, n).restype = C.c_int
    return lib


class App:
    def __init__(self, lib, kind, p, prm=()):
        self.lib, self.p = lib, p.copy()
        a = np.ascontiguousarray(prm, dtype=np.float64)
        h = C.c_void_p()
        rc = lib.app_create(kind, C.byref(self.p), a.ctypes.data_as(C.c_void_p) if a.size else None, C.byref(h))
        assert rc == FIN_OK, rc
        self.h = h

    def close(self):
        self.lib.app_destroy(self.h)

    def construct_l(self, q):
        L = np.zeros_like(q)
        sm = np.zeros((self.p.mx + 1 + 2 * self.p.mbc, self.p.my + 1 + 2 * self.p.mbc, 2))
        assert self.lib.app_construct_l(self.h, np.ascontiguousarray(q), L, sm.ctypes.data_as(C.c_void_p)) == FIN_OK
        return L, sm

    def steps(self, q, dt, n):
        assert self.lib.app_set_state(self.h, np.ascontiguousarray(q), 0.0) == FIN_OK
        cfl = C.c_double()
        cfls = []
        for _ in range(n):
            assert self.lib.app_step_fixed(self.h, dt, C.byref(cfl)) == FIN_OK
            cfls.append(cfl.value)
        out = np.zeros_like(q)
        t = C.c_double()
        assert self.lib.app_get_state(self.h, out, C.byref(t)) == FIN_OK
        return out, cfls, t.value


def _acoustics_case(weno, periodic, seed):
    p = P.vortex_params(n=37, weno=weno)
    p.my, p.meqn = 29, 3
    p.xlow, p.xhigh, p.ylow, p.yhigh = -1.0, 2.0, 0.0, 2.5
    bc = FIN_BC_PERIODIC if periodic else FIN_BC_TRANSMISSIVE
    p.bc_xlow = p.bc_xhigh = p.bc_ylow = p.bc_yhigh = bc
    x, y = P.cell_centres(p)
    rng = np.random.default_rng(seed)
    q = np.zeros(x.shape + (3,))
    q[..., 0] = 1.0 + 0.3 * np.exp(-8 * ((x - 0.4) ** 2 + (y - 1.1) ** 2)) + 0.05 * rng.standard_normal(x.shape)
    q[..., 1] = 0.2 * np.sin(2 * np.pi * x / 3.0)
    q[..., 2] = np.where(x + y > 1.7, 0.3, -0.1)     # a jump, so the nonlinear weights work
    return p, q


@pytest.mark.parametrize("weno", [FIN_WENO_JS, FIN_WENO_Z, FIN_WENO_FD])
@pytest.mark.parametrize("periodic", [True, False])
def test_third_physics_construct_l(app, weno, periodic):
    import generic_oracle as G
    p, q = _acoustics_case(weno, periodic, seed=weno + 3 * periodic)
    q = G.set_bnd(p, q)
    ph = G.AdvAcousticsCallbacks(*ACOUSTICS)
    a = App(app, 0, p, ACOUSTICS)
    try:
        L, sm = a.construct_l(q)
    finally:
        a.close()
    Lo, smo = G.construct_l(ph, p, q)
    assert rel_linf(interior(p, L), interior(p, Lo)) <= TOL
    assert rel_linf(sm, smo) <= 1e-15


@pytest.mark.parametrize("weno", [FIN_WENO_JS, FIN_WENO_Z])
@pytest.mark.parametrize("hooks", [False, True])
def test_third_physics_rk3_steps_with_hooks(app, weno, hooks):
    import generic_oracle as G
    p, q = _acoustics_case(weno, True, seed=11)
    q = G.set_bnd(p, q)
    ph = G.AdvAcousticsCallbacks(*ACOUSTICS)
    h0, h1 = 1e-3, 0.999
    prm = ACOUSTICS + ((h0, h1) if hooks else ())
    bs = af = None
    if hooks:
        def bs(a):
            a = a.copy()
            a[..., 0] = a[..., 0] + h0      # BeforeStep: p += h0
            return a

        def af(a):
            a = a.copy()
            a[..., 1] = a[..., 1] * h1      # AfterStep: u *= h1
            return a
    dt = 0.3 * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / 2.5
    a = App(app, 1 if hooks else 0, p, prm)
    try:
        qg, cfls, t = a.steps(q, dt, 3)
    finally:
        a.close()
    qo = q
    for k in range(3):
        qo, cfl = G.rk3_step(ph, p, qo, dt, bs, af)
        assert abs(cfls[k] - cfl) <= 1e-14 * cfl
    assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL
    assert t == pytest.approx(3 * dt, rel=1e-15)


@pytest.mark.parametrize("path", golden_cases("constructl_"))
def test_euler_policy_through_the_template(app, path):
    g = load_golden(path)
    p = g["p"]
    a = App(app, 2, p)
    try:
        L, sm = a.construct_l(g["q"])
    finally:
        a.close()
    assert rel_linf(interior(p, L), interior(p, g["L"])) <= TOL
    assert rel_linf(sm, g["smax"]) <= 1e-14


def test_euler_policy_steps_equal_the_specialised_kernel(app, oracle):
    from finess_b200.solver import Solver
    rng = np.random.default_rng(21)
    p = P.riemann_params(n=41, weno=FIN_WENO_Z)
    p.my = 35
    q = oracle.set_bnd(p, P.random_riemann_state(p, rng))
    dt = 0.2 * (1.0 / 41) / 4.0
    a = App(app, 2, p)
    try:
        qg, cfls, _ = a.steps(q, dt, 3)
    finally:
        a.close()
    with Solver(p) as s:
        s.set_state(q)
        for _ in range(3):
            s.step_fixed(dt)
        qs, _ = s.get_state()
    qo = q
    for _ in range(3):
        qo, _ = oracle.step_fixed(p, qo, dt)
    assert rel_linf(interior(p, qg), interior(p, qo)) <= TOL
    assert rel_linf(interior(p, qg), interior(p, qs)) <= TOL


def test_reciprocal_error_bounds(app):
    """fin_device.cuh's rcp (Newton-Raphson refinement of rcp.approx, two
    steps in FP64): within 1 ulp of the correctly rounded 1/x, and equal to
    CUDA's __ddiv_rn(1, x) for most x, over normal magnitudes 2^-1000 ..
    2^1000 of both signs; x = 0 and subnormal x give NaN and results below
    the normal range flush to 0, as its comment states (no use divides by
    such values: a zero or subnormal density is already a failed state).
    FP32: rcp.approx alone, within 1 ulp of 1/x."""
    f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    f32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    app.app_rcp_probe.argtypes = [f64, f64, f64, f32, C.c_int]
    app.app_rcp_probe.restype = C.c_int
    rng = np.random.default_rng(8)
    e = rng.uniform(-1000, 1000, 200000)
    x = np.ldexp(rng.uniform(1.0, 2.0, e.size), e.astype(np.int64)) * rng.choice([-1.0, 1.0], e.size)
    x = np.concatenate([x, [1.0, 3.0, 0.1, 1.4, 1e-300, 7e300, 2.0 ** -1022, 2.0 ** 1021 * 1.5]])
    edge = np.array([0.0, 1e-310, -2.0 ** -1070, 2.0 ** 1023])
    allx = np.ascontiguousarray(np.concatenate([x, edge]))
    n = allx.size
    r64, d64, r32 = np.zeros(n), np.zeros(n), np.zeros(n, dtype=np.float32)
    assert app.app_rcp_probe(allx, r64, d64, r32, n) == FIN_OK
    exact = 1.0 / x
    k = x.size
    ulp_err = np.abs(r64[:k] - exact) / np.spacing(np.abs(exact))
    assert np.max(ulp_err) <= 1.0
    assert np.array_equal(d64[:k], exact)                      # CUDA's division is correctly rounded
    assert np.mean(r64[:k] == exact) > 0.99
    assert np.isnan(r64[k]) and np.isnan(r64[k + 1]) and np.isnan(r64[k + 2])   # 0 and subnormal x
    assert r64[k + 3] == 0.0                                   # 1/2^1023 is subnormal: flushed
    x32 = x[(np.abs(x) > 1e-30) & (np.abs(x) < 1e30)].astype(np.float32)
    sel = (np.abs(allx[:k]) > 1e-30) & (np.abs(allx[:k]) < 1e30)
    ex32 = (np.float32(1.0) / x32).astype(np.float32)
    err32 = np.abs(r32[:k][sel].astype(np.float64) - ex32) / np.spacing(np.abs(ex32))
    assert np.max(err32) <= 1.0
