"""Initial conditions and parameter sets of the benchmark problems.

Each ``*_params`` function returns a ``FinParams`` for one problem; ``sample``
point-samples its QinitFunc at cell centres ``xlow + (i - 1/2) dx`` over the
whole ghosted grid, as lib/2d/SampleFunction.cpp:62-125 does (called from
lib/2d/RunFinpack.cpp:80), and returns the reference's ghosted (i, j, m)
array.  The Euler state is (rho, rho u, rho v, rho w, E) with w = 0
(apps/2d/euler/test_exact2/QinitFunc.cpp:66-72 is the pattern).
"""
import math

import numpy as np

from ._abi import (FIN_BC_PERIODIC, FIN_BC_TRANSMISSIVE, FIN_PHYS_MHD, FIN_TS_MD, FIN_TS_RK, FIN_WENO_JS,
                   FIN_WENO_Z, default_params)


def cell_centres(p):
    dx = (p.xhigh - p.xlow) / p.mx
    dy = (p.yhigh - p.ylow) / p.my
    i = np.arange(1 - p.mbc, p.mx + p.mbc + 1, dtype=np.float64)
    j = np.arange(1 - p.mbc, p.my + p.mbc + 1, dtype=np.float64)
    xc = p.xlow + (i - 0.5) * dx
    yc = p.ylow + (j - 0.5) * dy
    return np.meshgrid(xc, yc, indexing="ij")


def primitive_to_conserved(gamma, rho, u, v, pr):
    q = np.zeros(rho.shape + (5,))
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = 0.0
    q[..., 4] = pr / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return q


# --------------------------------------------------------------------------
# 1. Isentropic vortex on [0,10]^2, periodic.
# --------------------------------------------------------------------------
def vortex_params(n=200, weno=FIN_WENO_JS, **kw):
    p = default_params(mx=n, my=n, mbc=3, xlow=0.0, xhigh=10.0, ylow=0.0, yhigh=10.0,
                       weno_version=weno, global_alpha=1, desired_cfl=0.4, max_cfl=0.45,
                       time_stepping_method=FIN_TS_RK, time_order=3, gamma=1.4)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def vortex_exact(p, t=0.0, eps=5.0, x=None, y=None):
    """Vortex translated by (t, t) with period 10 (background u = v = 1)."""
    g = p.gamma
    if x is None:
        x, y = cell_centres(p)
    xs = np.mod(x - t - 0.0, 10.0)
    ys = np.mod(y - t - 0.0, 10.0)
    dxv = xs - 5.0
    dyv = ys - 5.0
    r2 = dxv * dxv + dyv * dyv
    ex = np.exp((1.0 - r2) / 2.0)
    du = -eps / (2.0 * math.pi) * ex * dyv
    dv = eps / (2.0 * math.pi) * ex * dxv
    T = 1.0 - (g - 1.0) * eps * eps / (8.0 * g * math.pi * math.pi) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (g - 1.0))
    pr = rho ** g
    return primitive_to_conserved(g, rho, 1.0 + du, 1.0 + dv, pr)


# --------------------------------------------------------------------------
# 2. Four-quadrant Riemann problem on [0,1]^2, transmissive, interface (0.8, 0.8).
# --------------------------------------------------------------------------
RIEMANN_STATES = {  # (rho, u, v, p)
    "ur": (1.5, 0.0, 0.0, 1.5),
    "ul": (0.5323, 1.206, 0.0, 0.3),
    "ll": (0.138, 1.206, 1.206, 0.029),
    "lr": (0.5323, 0.0, 1.206, 0.3),
}


def riemann_params(n=4096, weno=FIN_WENO_Z, method=FIN_TS_RK, **kw):
    mbc = 5 if method == FIN_TS_MD else 3
    p = default_params(mx=n, my=n, mbc=mbc, xlow=0.0, xhigh=1.0, ylow=0.0, yhigh=1.0,
                       weno_version=weno, global_alpha=1, desired_cfl=0.4, max_cfl=0.45,
                       time_stepping_method=method, time_order=4 if method == FIN_TS_MD else 3,
                       gamma=1.4)
    p.bc_xlow = p.bc_xhigh = p.bc_ylow = p.bc_yhigh = FIN_BC_TRANSMISSIVE
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def riemann_init(p, xc0=0.8, yc0=0.8, states=None):
    s = RIEMANN_STATES if states is None else states
    x, y = cell_centres(p)
    rho = np.empty_like(x); u = np.empty_like(x); v = np.empty_like(x); pr = np.empty_like(x)
    quads = {
        "ur": (x >= xc0) & (y >= yc0), "ul": (x < xc0) & (y >= yc0),
        "ll": (x < xc0) & (y < yc0), "lr": (x >= xc0) & (y < yc0),
    }
    for k, mask in quads.items():
        r_, u_, v_, p_ = s[k]
        rho[mask], u[mask], v[mask], pr[mask] = r_, u_, v_, p_
    return primitive_to_conserved(p.gamma, rho, u, v, pr)


def double_rarefaction_init(p, speed=2.0, rho=1.0, pr=0.4):
    """Near-vacuum test for the positivity limiter: two rarefactions moving
    apart from x = 0.5 (u = -speed left, +speed right), a weak transverse
    wave in v, constant rho and p."""
    x, y = cell_centres(p)
    u = np.where(x < 0.5 * (p.xlow + p.xhigh), -speed, speed)
    v = 0.1 * np.sin(2.0 * math.pi * (y - p.ylow) / (p.yhigh - p.ylow))
    return primitive_to_conserved(p.gamma, np.full_like(x, rho), u, v, np.full_like(x, pr))


# --------------------------------------------------------------------------
# 3. Shock / entropy-wave interaction on [-5,5]x[0,1], periodic in y.
# --------------------------------------------------------------------------
def shock_entropy_params(nx=8192, ny=1024, weno=FIN_WENO_JS, **kw):
    p = default_params(mx=nx, my=ny, mbc=3, xlow=-5.0, xhigh=5.0, ylow=0.0, yhigh=1.0,
                       weno_version=weno, global_alpha=1, desired_cfl=0.4, max_cfl=0.45,
                       time_stepping_method=FIN_TS_RK, time_order=3, gamma=1.4)
    p.bc_xlow = p.bc_xhigh = FIN_BC_TRANSMISSIVE
    p.bc_ylow = p.bc_yhigh = FIN_BC_PERIODIC
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def shock_entropy_init(p):
    x, y = cell_centres(p)
    left = x < -4.0
    rho = np.where(left, 3.857143, 1.0 + 0.2 * np.sin(5.0 * x) + 0.1 * np.sin(2.0 * math.pi * y))
    u = np.where(left, 2.629369, 0.0)
    v = np.zeros_like(x)
    pr = np.where(left, 10.33333, 1.0)
    return primitive_to_conserved(p.gamma, rho, u, v, pr)


# --------------------------------------------------------------------------
# 5. Ideal MHD Orszag-Tang vortex on [0,2pi]^2, periodic (apps/2d/mhd/orszag_tang).
# --------------------------------------------------------------------------
def orszag_tang_params(n=2048, weno=FIN_WENO_JS, **kw):
    """apps/2d/mhd/orszag_tang/parameters.ini (meqn 8, maux 1, mbc 7,
    gamma 5/3, domain [0, 6.2831853071795865]^2, global_alpha default false)
    with SSP-RK3 at CFL 0.4 (max 0.45) and n x n cells."""
    p = default_params(mx=n, my=n, mbc=7, meqn=8, maux=1, xlow=0.0, xhigh=6.2831853071795865, ylow=0.0,
                       yhigh=6.2831853071795865, weno_version=weno, global_alpha=0, desired_cfl=0.4,
                       max_cfl=0.45, time_stepping_method=FIN_TS_RK, time_order=3, gamma=1.6666666666666667,
                       physics=FIN_PHYS_MHD, constrained_transport=1, initial_dt=0.001)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def orszag_tang_init(p):
    """(q, aux): QinitFunc (apps/2d/mhd/orszag_tang/QinitFunc.cpp:10-52) at
    the cell centres, rho = gamma^2, p = gamma, u = (-sin y, sin x, 0),
    B = (-sin y, sin 2x, 0); aux = A3 = 0.5 cos 2x + cos y (AfterQinit.cpp:
    10-35, whose curl is B).  Ghost cells hold the periodic images."""
    x, y = cell_centres(p)
    g = p.gamma
    rho = np.full_like(x, g * g)
    u1, u2 = -np.sin(y), np.sin(x)
    B1, B2 = -np.sin(y), np.sin(2.0 * x)
    q = np.zeros(x.shape + (8,))
    q[..., 0] = rho
    q[..., 1] = rho * u1
    q[..., 2] = rho * u2
    q[..., 4] = g / (g - 1.0) + 0.5 * rho * (u1 * u1 + u2 * u2) + 0.5 * (B1 * B1 + B2 * B2)
    q[..., 5] = B1
    q[..., 6] = B2
    aux = (0.5 * np.cos(2.0 * x) + np.cos(y))[..., None]
    return q, aux


def mhd_random_state(p, rng, amp=0.3):
    """A smooth periodic MHD state with every component nonzero (u3, B3
    included) and (q, aux) consistent: B1, B2 the 4th-order central curl of
    the periodic potential aux, as constrained transport leaves them."""
    x, y = cell_centres(p)
    Lx, Ly = p.xhigh - p.xlow, p.yhigh - p.ylow
    kx, ky = 2.0 * math.pi / Lx, 2.0 * math.pi / Ly
    ph = rng.uniform(0, 2 * math.pi, size=10)
    rho = 1.0 + amp * np.sin(kx * x + ph[0]) * np.cos(ky * y + ph[1])
    u1 = 0.4 + amp * np.sin(kx * x + ph[2] + ky * y)
    u2 = -0.3 + amp * np.cos(ky * y + ph[3] - kx * x)
    u3 = 0.2 * np.sin(kx * x + ph[4])
    pr = 1.0 + amp * np.cos(kx * x + ph[5]) * np.sin(ky * y + ph[6])
    A = 0.6 * np.cos(kx * x + ph[7]) + 0.5 * np.sin(ky * y + ph[8]) + 0.2 * np.sin(kx * x + ky * y + ph[9])
    dx, dy = Lx / p.mx, Ly / p.my
    B1 = (np.roll(A, 2, 1) - 8 * np.roll(A, 1, 1) + 8 * np.roll(A, -1, 1) - np.roll(A, -2, 1)) / (12 * dy)
    B2 = -(np.roll(A, 2, 0) - 8 * np.roll(A, 1, 0) + 8 * np.roll(A, -1, 0) - np.roll(A, -2, 0)) / (12 * dx)
    B3 = 0.3 + 0.1 * np.cos(ky * y + ph[0])
    g = p.gamma
    q = np.zeros(x.shape + (8,))
    q[..., 0] = rho
    q[..., 1], q[..., 2], q[..., 3] = rho * u1, rho * u2, rho * u3
    q[..., 4] = pr / (g - 1.0) + 0.5 * rho * (u1 * u1 + u2 * u2 + u3 * u3) + 0.5 * (B1 * B1 + B2 * B2 + B3 * B3)
    q[..., 5], q[..., 6], q[..., 7] = B1, B2, B3
    return q, A[..., None]


# --------------------------------------------------------------------------
# Random smooth and random Riemann states for parity tests.
# --------------------------------------------------------------------------
def random_smooth_state(p, rng, amp=0.2):
    x, y = cell_centres(p)
    Lx, Ly = p.xhigh - p.xlow, p.yhigh - p.ylow
    kx = 2.0 * math.pi / Lx
    ky = 2.0 * math.pi / Ly
    ph = rng.uniform(0, 2 * math.pi, size=8)
    rho = 1.0 + amp * np.sin(kx * x + ph[0]) * np.cos(ky * y + ph[1])
    u = 0.5 + amp * np.sin(kx * x + ph[2] + ky * y)
    v = -0.3 + amp * np.cos(ky * y + ph[3] - kx * x)
    pr = 1.0 + amp * np.cos(kx * x + ph[4]) * np.sin(ky * y + ph[5])
    return primitive_to_conserved(p.gamma, rho, u, v, pr)


def random_riemann_state(p, rng):
    states = {}
    for k in RIEMANN_STATES:
        states[k] = (rng.uniform(0.1, 2.0), rng.uniform(-1.5, 1.5), rng.uniform(-1.5, 1.5),
                     rng.uniform(0.02, 2.0))
    xc0 = p.xlow + (p.xhigh - p.xlow) * rng.uniform(0.3, 0.7)
    yc0 = p.ylow + (p.yhigh - p.ylow) * rng.uniform(0.3, 0.7)
    return riemann_init(p, xc0, yc0, states)


def density_errors(p, q, qref):
    """Density L1 (area-normalised: sum|diff| dx dy / area, as
    apps/2d/euler/test_exact2/run_error.py:52 with its area 100) and Linf,
    interior cells only."""
    mb = p.mbc
    a = q[mb:mb + p.mx, mb:mb + p.my, 0]
    b = qref[mb:mb + p.mx, mb:mb + p.my, 0]
    d = np.abs(a - b)
    dx = (p.xhigh - p.xlow) / p.mx
    dy = (p.yhigh - p.ylow) / p.my
    area = (p.xhigh - p.xlow) * (p.yhigh - p.ylow)
    return float(d.sum() * dx * dy / area), float(d.max())
