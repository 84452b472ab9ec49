"""CPU restatement of lib/2d's ConstructL, GlobalWaveSpd, UpdateSoln and the
SSP-RK3 stage sequence of FinSolveRK for a physics given as Python callbacks
(the application callbacks of lib/2d/ConstructL.h:8-23, vectorised over
points).  TEST INFRASTRUCTURE ONLY: the checker of the device callback
surface (finess_b200/csrc/fin_physics.cuh, fin_physics_host.h).

Every function follows the reference's operation order:
* ``weno5``: lib/WenoReconstruct.cpp (JS5 :90-141, Z5 :385-438, FD5
  :580-616): smoothness indicators :121-123, candidates :126-128, weights
  :131-137 (numpy's power is the C library's pow);
* ``construct_l``: lib/2d/ConstructL.cpp:62-208 (x faces), :214-358 (y
  faces), :390-401 (L);
* ``global_wave_spd``: lib/2d/GlobalWaveSpd.cpp:52-78;
* ``rk3_step``: lib/2d/FinSolveRK.cpp:158-211 with SetBndValues, the hooks
  (hooks.h) and UpdateSoln.cpp:29-35.

A physics object provides M (meqn) and, on arrays whose last axis is the
component:
    flux(x, y, Q) -> (f, g)
    wave_speed(nx, ny, x, y, Ql, Qr) -> (s1, s2)
    face(ixy, Qavg) -> F; left(F, V) -> W; right(F, W) -> V
``EulerCallbacks`` restates the reference's Euler callbacks in their own
formula order (apps/2d/euler/lib/{FluxFunc,SetWaveSpd,ProjectLeftEig,
ProjectRightEig}.cpp); it pins this restatement against the reference's
golden ConstructL fixtures.
"""
import numpy as np

FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z = 0, 1, 2
FIN_BC_PERIODIC = 0


def Max(a, b):
    """dog_math.h's Max(a, b) = a > b ? a : b, element-wise."""
    return np.where(a > b, a, b)


def Min(a, b):
    return np.where(a < b, a, b)


def weno5(u, version, eps, pw):
    """u: sequence of the 5 stencil arrays u_{i-2} .. u_{i+2}."""
    uim2, uim1, ui, uip1, uip2 = u
    t = uim2 - 2 * uim1 + ui
    b0 = (13. / 12.) * (t * t)
    t = uim2 - 4 * uim1 + 3 * ui
    b0 = b0 + 0.25 * (t * t)
    t = uim1 - 2 * ui + uip1
    b1 = (13. / 12.) * (t * t)
    t = uim1 - uip1
    b1 = b1 + 0.25 * (t * t)
    t = ui - 2 * uip1 + uip2
    b2 = (13. / 12.) * (t * t)
    t = 3 * ui - 4 * uip1 + uip2
    b2 = b2 + 0.25 * (t * t)
    c0 = (1. / 3.) * uim2 - (7. / 6.) * uim1 + (11. / 6.) * ui
    c1 = (-1. / 6.) * uim1 + (5. / 6.) * ui + (1. / 3.) * uip1
    c2 = (1. / 3.) * ui + (5. / 6.) * uip1 - (1. / 6.) * uip2
    if version == FIN_WENO_FD:
        return 0.1 * c0 + 0.6 * c1 + 0.3 * c2
    if version == FIN_WENO_JS:
        o0 = 0.1 * np.power(eps + b0, -pw)
        o1 = 0.6 * np.power(eps + b1, -pw)
        o2 = 0.3 * np.power(eps + b2, -pw)
    else:
        tau5 = np.abs(b0 - b2)
        o0 = 0.1 * (1. + np.power(tau5 / (eps + b0), pw))
        o1 = 0.6 * (1. + np.power(tau5 / (eps + b1), pw))
        o2 = 0.3 * (1. + np.power(tau5 / (eps + b2), pw))
    os_ = o0 + o1 + o2
    return (o0 * c0 + o1 * c1 + o2 * c2) / os_


def set_bnd(p, q):
    """Periodic or zeroth-order extrapolation ghost cells of every side (the
    two SetBndValues of the Euler applications), corners included."""
    q = q.copy()
    mb, mx, my = p.mbc, p.mx, p.my
    ii = np.arange(-mb, mx + mb)
    jj = np.arange(-mb, my + mb)

    def remap(k, n, lo, hi):
        k = k.copy()
        low, high = k < 0, k >= n
        k[low] = (k[low] % n) if lo == FIN_BC_PERIODIC else 0
        k[high] = (k[high] % n) if hi == FIN_BC_PERIODIC else n - 1
        return k

    ri = remap(ii, mx, p.bc_xlow, p.bc_xhigh) + mb
    rj = remap(jj, my, p.bc_ylow, p.bc_yhigh) + mb
    return q[np.ix_(ri, rj)]


def global_wave_spd(phys, p, q):
    mb = p.mbc
    Q = q[mb:mb + p.mx, mb:mb + p.my]
    dx, dy = (p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my
    i = np.arange(1, p.mx + 1, dtype=np.float64)[:, None]
    j = np.arange(1, p.my + 1, dtype=np.float64)[None, :]
    x = p.xlow + i * dx - 0.5 * dx + 0 * j
    y = p.ylow + j * dy - 0.5 * dy + 0 * i
    a1 = a2 = 0.0
    s1, s2 = phys.wave_speed(1.0, 0.0, x, y, Q, Q)
    sx = Max(np.abs(s1), np.abs(s2))
    s1, s2 = phys.wave_speed(0.0, 1.0, x, y, Q, Q)
    sy = Max(np.abs(s1), np.abs(s2))
    # the serial loop's Max(alpha, v) keeps alpha when v is NaN
    a1 = float(np.max(sx[~np.isnan(sx)], initial=0.0))
    a2 = float(np.max(sy[~np.isnan(sy)], initial=0.0))
    return a1, a2


def _face_fluxes(phys, p, q, ixy, alpha_g):
    """Fhat (ixy 1: faces i = 1..mx+1, j = 1..my) or Ghat (ixy 2: i = 1..mx,
    j = 1..my+1) and the face speeds alpha."""
    mb, mx, my = p.mbc, p.mx, p.my
    dx, dy = (p.xhigh - p.xlow) / mx, (p.yhigh - p.ylow) / my
    if ixy == 1:
        fi = np.arange(1, mx + 2)[:, None]
        fj = np.arange(1, my + 1)[None, :]
    else:
        fi = np.arange(1, mx + 1)[:, None]
        fj = np.arange(1, my + 2)[None, :]
    pts = []
    for s in range(1, 7):                       # is = i-1+s-r, r = 3 (ConstructL.cpp:96)
        if ixy == 1:
            ci, cj = fi - 1 + s - 3, fj + 0 * fi
        else:
            ci, cj = fi + 0 * fj, fj - 1 + s - 3
        xi = p.xlow + ci.astype(np.float64) * dx - 0.5 * dx
        yi = p.ylow + cj.astype(np.float64) * dy - 0.5 * dy
        Q = q[ci - 1 + mb, cj - 1 + mb]
        f, g = phys.flux(xi, yi, Q)
        pts.append((Q, f if ixy == 1 else g))
    Ql, Qr = pts[2][0], pts[3][0]
    Qavg = 0.5 * (Qr + Ql)
    xe = p.xlow + (fi + 0 * fj).astype(np.float64) * dx - 0.5 * dx
    ye = p.ylow + (fj + 0 * fi).astype(np.float64) * dy - 0.5 * dy
    nx, ny = (1.0, 0.0) if ixy == 1 else (0.0, 1.0)
    s1, s2 = phys.wave_speed(nx, ny, xe, ye, Ql, Qr)
    alpha = Max(alpha_g, Max(np.abs(s1), np.abs(s2)))
    la = p.alpha_scaling * alpha
    F = phys.face(ixy, Qavg)
    W = [phys.left(F, Q) for Q, _ in pts]
    G = [phys.left(F, f) for _, f in pts]
    gp = [0.5 * (G[s] + la[..., None] * W[s]) for s in range(5)]
    gm = [0.5 * (G[5 - s] - la[..., None] * W[5 - s]) for s in range(5)]
    ghat = np.empty_like(Qavg)
    for m in range(phys.M):
        ghat[..., m] = (weno5([g[..., m] for g in gp], p.weno_version, p.epsilon, p.power_param)
                        + weno5([g[..., m] for g in gm], p.weno_version, p.epsilon, p.power_param))
    return phys.right(F, ghat), alpha


def construct_l(phys, p, q):
    """L (ghosted array, interior set, ghosts 0) and smax (ghosted (mx+1,
    my+1, 2), zero-initialised, max-accumulated) of a state whose ghosts
    are already set."""
    mb, mx, my = p.mbc, p.mx, p.my
    dx, dy = (p.xhigh - p.xlow) / mx, (p.yhigh - p.ylow) / my
    a1, a2 = global_wave_spd(phys, p, q) if p.global_alpha else (0.0, 0.0)
    Fh, ax = _face_fluxes(phys, p, q, 1, a1)
    Gh, ay = _face_fluxes(phys, p, q, 2, a2)
    L = np.zeros_like(q)
    tmp = -(Fh[1:, :] - Fh[:-1, :]) / dx
    tmp = tmp - (Gh[:, 1:] - Gh[:, :-1]) / dy
    L[mb:mb + mx, mb:mb + my] = tmp
    smax = np.zeros((mx + 1 + 2 * mb, my + 1 + 2 * mb, 2))
    smax[mb:mb + mx + 1, mb:mb + my, 0] = Max(smax[mb:mb + mx + 1, mb:mb + my, 0], ax)
    smax[mb:mb + mx, mb:mb + my + 1, 1] = Max(smax[mb:mb + mx, mb:mb + my + 1, 1], ay)
    return L, smax


def rk3_step(phys, p, q, dt, before_step=None, after_step=None):
    """One SSP-RK3 step of exactly dt (FinSolveRK.cpp:158-211): SetBndValues,
    BeforeStep, ConstructL, UpdateSoln, AfterStep per stage (the hooks act on
    whole ghosted arrays); returns (q^{n+1}, CFL of GetCFL.cpp:31-73)."""
    mb, mx, my = p.mbc, p.mx, p.my
    dx, dy = (p.xhigh - p.xlow) / mx, (p.yhigh - p.ylow) / my
    bs = before_step or (lambda a: a)
    af = after_step or (lambda a: a)
    smax = np.zeros((mx + 1 + 2 * mb, my + 1 + 2 * mb, 2))
    qnew = set_bnd(p, q)
    qnew = bs(qnew)
    L, s = construct_l(phys, p, qnew)
    smax = Max(smax, s)
    qstar = 1.0 * qnew + (1.0 * dt) * L           # 0 * Qstar dropped
    qstar = af(qstar)
    qstar = bs(set_bnd(p, qstar))
    L, s = construct_l(phys, p, qstar)
    smax = Max(smax, s)
    qstar = 0.75 * qnew + 0.25 * qstar + (0.25 * dt) * L
    qstar = af(qstar)
    qstar = bs(set_bnd(p, qstar))
    L, s = construct_l(phys, p, qstar)
    smax = Max(smax, s)
    qnew = (2.0e0 / 3.0e0) * qstar + (1.0e0 / 3.0e0) * qnew + ((2.0e0 / 3.0e0) * dt) * L
    qnew = af(qnew)
    S = smax[mb:mb + mx, mb:mb + my]
    cfl = max(-100.0, float(np.max(dt * S[..., 0] / dx)), float(np.max(dt * S[..., 1] / dy)))
    return set_bnd(p, qnew), cfl


class EulerCallbacks:
    """apps/2d/euler/lib's callbacks, in their formula order."""
    M = 5

    def __init__(self, gamma):
        self.gamma = gamma

    def flux(self, x, y, Q):                              # FluxFunc.cpp:18-43
        g_ = self.gamma
        rho = Q[..., 0]
        u1, u2, u3 = Q[..., 1] / rho, Q[..., 2] / rho, Q[..., 3] / rho
        energy = Q[..., 4]
        press = (g_ - 1.0e0) * (energy - 0.5e0 * rho * (u1 * u1 + u2 * u2 + u3 * u3))
        f = np.stack([rho * u1, rho * u1 * u1 + press, rho * u1 * u2, rho * u1 * u3, u1 * (energy + press)], -1)
        g = np.stack([rho * u2, rho * u2 * u1, rho * u2 * u2 + press, rho * u2 * u3, u2 * (energy + press)], -1)
        return f, g

    def wave_speed(self, nx, ny, x, y, Ql, Qr):           # SetWaveSpd.cpp:11-69
        g_ = self.gamma

        def prim(Q):
            rho = Q[..., 0]
            u1, u2, u3 = Q[..., 1] / rho, Q[..., 2] / rho, Q[..., 3] / rho
            pr = (g_ - 1.0e0) * (Q[..., 4] - 0.5e0 * rho * (u1 * u1 + u2 * u2 + u3 * u3))
            return rho, u1, u2, u3, pr

        rl, u1l, u2l, u3l, pl = prim(Ql)
        rr, u1r, u2r, u3r, pr_ = prim(Qr)
        rho = 0.5e0 * (rl + rr)
        u1 = 0.5e0 * (u1l + u1r)
        u2 = 0.5e0 * (u2l + u2r)
        press = 0.5e0 * (pl + pr_)
        nmag = np.sqrt(nx ** 2 + ny ** 2)
        cl = nmag * np.sqrt(np.abs(g_ * pl / rl))
        cr = nmag * np.sqrt(np.abs(g_ * pr_ / rr))
        c = nmag * np.sqrt(np.abs(g_ * press / rho))
        un = nx * u1 + ny * u2
        unl = nx * u1l + ny * u2l
        unr = nx * u1r + ny * u2r
        return Min(unl - cl, un - c), Max(unr + cr, un + c)

    def face(self, ixy, Qa):                              # ProjectLeftEig.cpp:20-44
        g_ = self.gamma
        mu, mv = (1, 2) if ixy == 1 else (2, 1)
        rho = Qa[..., 0]
        u1, u2, u3 = Qa[..., mu] / rho, Qa[..., mv] / rho, Qa[..., 3] / rho
        energy = Qa[..., 4]
        umag2 = u1 * u1 + u2 * u2 + u3 * u3
        press = (g_ - 1.0e0) * (energy - 0.5e0 * rho * umag2)
        return {"mu": mu, "mv": mv, "u1": u1, "u2": u2, "u3": u3, "umag2": umag2, "H": (energy + press) / rho,
                "cl": np.sqrt(g_ * press / rho), "cr": np.sqrt(np.abs(g_ * press / rho))}

    def left(self, F, Q):                                 # ProjectLeftEig.cpp:47-66
        mu, mv = F["mu"], F["mv"]
        u1, u2, u3, umag2, H, c = F["u1"], F["u2"], F["u3"], F["umag2"], F["H"], F["cl"]
        q1, qmu, qmv, qmw, q5 = Q[..., 0], Q[..., mu], Q[..., mv], Q[..., 3], Q[..., 4]
        W = np.empty_like(Q)
        W[..., 0] = ((umag2 / 2.0 - H - u1 * c) * qmu + (umag2 / 2.0 * (c - u1) + H * u1) * q1
                     + c * (q5 - u2 * qmv - u3 * qmw)) / (c * (2.0 * H - umag2))
        W[..., mu] = 2.0 * ((H - umag2) * q1 + u1 * qmu + u2 * qmv + u3 * qmw - q5) / (2.0 * H - umag2)
        W[..., mv] = qmv - u2 * q1
        W[..., 3] = qmw - u3 * q1
        W[..., 4] = ((H - umag2 / 2.0 - u1 * c) * qmu + (umag2 / 2.0 * (c + u1) - H * u1) * q1
                     + c * (q5 - u2 * qmv - u3 * qmw)) / (c * (2.0 * H - umag2))
        return W

    def right(self, F, W):                                # ProjectRightEig.cpp:46-62
        mu, mv = F["mu"], F["mv"]
        u1, u2, u3, umag2, H, c = F["u1"], F["u2"], F["u3"], F["umag2"], F["H"], F["cr"]
        w1, wmu, wmv, wmw, w5 = W[..., 0], W[..., mu], W[..., mv], W[..., 3], W[..., 4]
        Q = np.empty_like(W)
        Q[..., 0] = w1 + wmu + w5
        Q[..., mu] = (u1 - c) * w1 + u1 * wmu + (u1 + c) * w5
        Q[..., mv] = u2 * (w1 + wmu + w5) + wmv
        Q[..., 3] = u3 * (w1 + wmu + w5) + wmw
        Q[..., 4] = (H - u1 * c) * w1 + umag2 / 2.0 * wmu + u2 * wmv + u3 * wmw + (H + u1 * c) * w5
        return Q


class AdvAcousticsCallbacks:
    """The linear advection-acoustics physics of tests/apps/phys_app.cu."""
    M = 3

    def __init__(self, K, rho0, ax, ay):
        self.K, self.rho0, self.ax, self.ay = K, rho0, ax, ay
        self.c = np.sqrt(K / rho0)

    def flux(self, x, y, Q):
        p_, u, v = Q[..., 0], Q[..., 1], Q[..., 2]
        f = np.stack([self.ax * p_ + self.K * u, self.ax * u + p_ / self.rho0, self.ax * v], -1)
        g = np.stack([self.ay * p_ + self.K * v, self.ay * u, self.ay * v + p_ / self.rho0], -1)
        return f, g

    def wave_speed(self, nx, ny, x, y, Ql, Qr):
        an = self.ax * nx + self.ay * ny
        s1 = an - self.c + 0 * Ql[..., 0]
        s2 = an + self.c + 0 * Ql[..., 0]
        return s1, s2

    def face(self, ixy, Qa):
        return (ixy, self.rho0 * self.c)

    def left(self, F, V):
        ixy, Z = F
        n, t = (1, 2) if ixy == 1 else (2, 1)
        W = np.empty_like(V)
        W[..., 0] = -V[..., 0] / (2.0 * Z) + 0.5 * V[..., n]
        W[..., 1] = V[..., t]
        W[..., 2] = V[..., 0] / (2.0 * Z) + 0.5 * V[..., n]
        return W

    def right(self, F, W):
        ixy, Z = F
        n, t = (1, 2) if ixy == 1 else (2, 1)
        V = np.empty_like(W)
        V[..., 0] = -Z * W[..., 0] + Z * W[..., 2]
        V[..., n] = W[..., 0] + W[..., 2]
        V[..., t] = W[..., 1]
        return V
