"""Initial states for the block: Orszag-Tang vortex, Fishbone-Moncrief torus,
advected entropy wave. Arrays come back in the device layout (NPR planes of
primitives, 3 planes of face field, ghost zones left for the ghost fill).

Torus: init_torus (init_torus.c:84-511) with lfish_calc (init_torus.c:501),
the BL -> KS -> code-coordinate velocity transform of coord_transform
(init.c:3218-3290) and a single poloidal loop A_phi ~ max(rho/rho_max - 0.2, 0)
normalised to a minimum plasma beta (init_mag.c:6-468). The 4 % pressure
perturbation uses a seeded generator instead of the time-seeded ranc
(ranc.c:36-40), so runs are reproducible.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .api import (B1, B2, B3, CENT, FACE1, FACE2, KTOT, NPR, RHO, U1, U2, U3, UU, Geometry, build_geometry,
                  ks_grid, pad64)


@dataclass
class Problem:
    n1: int
    n2: int
    n3: int
    ng: int
    ksize: int
    gsize: int
    dx: tuple              # (dx1, dx2, dx3)
    gam: float
    cour: float
    bc: tuple
    poles: tuple
    ct_upwind: bool
    geo: Geometry
    p: np.ndarray          # NPR * ksize
    ps: np.ndarray         # 3 * ksize
    coords: str = "ks"
    spin: float = 0.0
    startx: tuple = (0.0, 0.0, 0.0, 0.0)

    @property
    def g(self):
        g1 = self.n1 + 2 * self.ng
        g2 = self.n2 + 2 * self.ng
        g3 = self.n3 + 2 * self.ng if self.n3 > 1 else 1
        return g1, g2, g3

    def view(self, a):
        g1, g2, g3 = self.g
        k = a.size // self.ksize
        return a.reshape(k, self.ksize)[:, :g1 * g2 * g3].reshape(k, g1, g2, g3)

    def active(self, a):
        v = self.view(a)
        g = self.ng
        g3 = g if self.n3 > 1 else 0
        return v[:, g:g + self.n1, g:g + self.n2, g3:g3 + self.n3]

    def block_kwargs(self):
        return dict(n1=self.n1, n2=self.n2, n3=self.n3, dx=self.dx, gam=self.gam, cour=self.cour,
                    bc=self.bc, poles=self.poles, ct_upwind=self.ct_upwind, ng=self.ng)


def _alloc(n1, n2, n3, ng):
    g1, g2 = n1 + 2 * ng, n2 + 2 * ng
    g3 = n3 + 2 * ng if n3 > 1 else 1
    ks = pad64(g1 * g2 * g3)
    return ks, np.zeros(NPR * ks), np.zeros(3 * ks)


def _geo_plane(geo, gsize, g1, g2, name, comp, loc):
    a = getattr(geo, name)
    k = comp * 5 + loc if name in ("gcov", "gcon") else loc
    return a[k * gsize: k * gsize + g1 * g2].reshape(g1, g2)


# ----------------------------------------------------------------- OT vortex
def orszag_tang(n: int = 128, gam: float = 5.0 / 3.0, vscale: float = 0.5, cour: float = 0.5) -> Problem:
    """2-D Orszag-Tang vortex on the periodic unit square: rho = 25/(36 pi),
    p = 5/(12 pi), v = vscale (-sin 2pi y, sin 2pi x),
    B = (-sin 2pi y, sin 4pi x)/sqrt(4 pi). The published vortex has |v| up to
    sqrt(2) in units where c does not appear; in this relativistic code the
    velocity pattern is scaled by `vscale` (default 0.5, |v| < 0.71 c)."""
    ng = 3
    ks, p, ps = _alloc(n, n, 1, ng)
    dx = (1.0 / n, 1.0 / n, 1.0)
    geo = build_geometry("cartesian", 0.0, n, n, 1, [0.0, 0.0, 0.0, 0.0], [0.0, *dx], ng)
    g1 = g2 = n + 2 * ng
    ii = np.arange(g1) - ng
    xc = (ii + 0.5) / n
    xf = ii / n
    X, Y = np.meshgrid(xc, xc, indexing="ij")
    Xf, Yc = np.meshgrid(xf, xc, indexing="ij")
    Xc2, Yf = np.meshgrid(xc, xf, indexing="ij")
    rho = 25.0 / (36.0 * np.pi)
    pres = 5.0 / (12.0 * np.pi)
    vx = -vscale * np.sin(2 * np.pi * Y)
    vy = vscale * np.sin(2 * np.pi * X)
    lor = 1.0 / np.sqrt(1.0 - vx * vx - vy * vy)
    s4p = np.sqrt(4.0 * np.pi)
    P = p.reshape(NPR, ks)[:, :g1 * g2].reshape(NPR, g1, g2, 1)
    S = ps.reshape(3, ks)[:, :g1 * g2].reshape(3, g1, g2, 1)
    P[RHO, ..., 0] = rho
    P[UU, ..., 0] = pres / (gam - 1.0)
    P[U1, ..., 0] = lor * vx
    P[U2, ..., 0] = lor * vy
    S[0, ..., 0] = -np.sin(2 * np.pi * Yc) / s4p
    S[1, ..., 0] = np.sin(4 * np.pi * Xc2) / s4p
    P[B1, :-1, :, 0] = 0.5 * (S[0, :-1, :, 0] + S[0, 1:, :, 0])
    P[B2, :, :-1, 0] = 0.5 * (S[1, :, :-1, 0] + S[1, :, 1:, 0])
    P[KTOT, ..., 0] = (gam - 1.0) * P[UU, ..., 0] * rho ** (-gam)
    return Problem(n, n, 1, ng, ks, geo.gsize, dx, gam, cour, ("periodic", "periodic", "periodic"), (0, 0),
                   False, geo, p, ps, coords="cartesian")


# ------------------------------------------------------------ entropy wave
def entropy_wave(n: int, amp: float = 1e-3, v0: float = 0.5, gam: float = 5.0 / 3.0, cour: float = 0.5) -> Problem:
    """Density wave rho = 1 + amp sin(2 pi x) advected at v0 through a uniform
    pressure p = 1 on the periodic unit square (x1 = x, n x 4 zones): after
    t = 1/v0 the exact solution is the initial state."""
    ng = 3
    n2 = 4
    ks, p, ps = _alloc(n, n2, 1, ng)
    dx = (1.0 / n, 1.0 / n2, 1.0)
    geo = build_geometry("cartesian", 0.0, n, n2, 1, [0.0, 0.0, 0.0, 0.0], [0.0, *dx], ng)
    g1, g2 = n + 2 * ng, n2 + 2 * ng
    x = (np.arange(g1) - ng + 0.5) / n
    # cell average of sin over the zone, so the discrete state is exact
    rho = 1.0 + amp * (np.cos(2 * np.pi * (x - 0.5 / n)) - np.cos(2 * np.pi * (x + 0.5 / n))) / (2 * np.pi / n)
    P = p.reshape(NPR, ks)[:, :g1 * g2].reshape(NPR, g1, g2, 1)
    P[RHO] = rho[:, None, None]
    P[UU] = 1.0 / (gam - 1.0)
    P[U1] = v0 / np.sqrt(1.0 - v0 * v0)
    P[KTOT] = (gam - 1.0) * P[UU] * P[RHO] ** (-gam)
    return Problem(n, n2, 1, ng, ks, geo.gsize, dx, gam, cour, ("periodic", "periodic", "periodic"), (0, 0),
                   False, geo, p, ps, coords="cartesian")


# ------------------------------------------------------- linear MHD modes
# 3-D (1,1,1) plane waves on the uniform state rho = 1, u = 1, B = (1, 0, 0):
# frequency and eigenvector (drho, du, du1, du2, du3, dB1, dB2, dB3) per mode
# (init_entwave, init_tests.c:1054-1156). The frequencies are those of
# gamma = 4/3 (the Alfven one is 2 pi sqrt(3) v_A with v_A^2 = (1/3) /
# (rho + gamma u + b^2)); the reference's config.h sets GAMMA = 5/3, for which
# these vectors are not eigenmodes, so linear_mode uses 4/3.
LINEAR_MODES = {
    "entropy": (2. * np.pi / 5., (1., 0., 0., 0., 0., 0., 0., 0.)),
    "slow": (2.35896379113, (0.556500332363, 0.742000443151, -0.282334999306, 0.0367010491491, 0.0367010491491,
                             -0.195509141461, 0.0977545707307, 0.0977545707307)),
    "alfven": (-3.44144232573, (0., 0., 0., -0.339683110243, 0.339683110243, 0., 0.620173672946, -0.620173672946)),
    "fast": (6.92915162882, (0.481846076323, 0.642461435098, -0.0832240462505, -0.224080007379, -0.224080007379,
                             0.406380545676, -0.203190272838, -0.203190272838)),
}


def linear_mode(n: int, mode: str = "fast", amp: float = 1.e-5, gam: float = 4.0 / 3.0, cour: float = 0.4,
                ng: int = 3) -> Problem:
    """Linear MHD eigenmode on the periodic unit cube in Minkowski space, n^3
    zones, wavevector 2 pi (1, 1, 1): primitives rho0 + drho cos(k.X), ... at
    zone centres, the face field at the faces (init_entwave,
    init_tests.c:1253-1289). After one period 2 pi / |omega| (the reference's
    tf) the exact solution is the initial state again."""
    omega, vec = LINEAR_MODES[mode]
    ks, p, ps = _alloc(n, n, n, ng)
    dx = (1.0 / n, 1.0 / n, 1.0 / n)
    geo = build_geometry("cartesian", 0.0, n, n, n, [0.0, 0.0, 0.0, 0.0], [0.0, *dx], ng)
    g = n + 2 * ng
    c = (np.arange(g) - ng + 0.5) / n
    f = (np.arange(g) - ng) / n
    k1 = k2 = k3 = 2.0 * np.pi

    def cosk(x1, x2, x3):
        return amp * np.cos(k1 * x1[:, None, None] + k2 * x2[None, :, None] + k3 * x3[None, None, :])

    P = p.reshape(NPR, ks)[:, :g ** 3].reshape(NPR, g, g, g)
    S = ps.reshape(3, ks)[:, :g ** 3].reshape(3, g, g, g)
    m = cosk(c, c, c)
    base = (1.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0)
    for k in range(8):
        P[k] = base[k] + vec[k] * m
    P[KTOT] = (gam - 1.0) * P[UU] * P[RHO] ** (-gam)
    S[0] = base[5] + vec[5] * cosk(f, c, c)
    S[1] = base[6] + vec[6] * cosk(c, f, c)
    S[2] = base[7] + vec[7] * cosk(c, c, f)
    return Problem(n, n, n, ng, ks, geo.gsize, dx, gam, cour, ("periodic", "periodic", "periodic"), (0, 0), False,
                   geo, p, ps, coords="cartesian")


# ---------------------------------------------------------------- FM torus
def lfish(a, r):
    """Specific angular momentum of the Fishbone-Moncrief torus with pressure
    maximum at r (lfish_calc, init_torus.c:501)."""
    return (((a ** 2 - 2. * a * np.sqrt(r) + r ** 2) *
             ((-2. * a * r * (a ** 2 - 2. * a * np.sqrt(r) + r ** 2)) / np.sqrt(2. * a * np.sqrt(r) + (-3. + r) * r) +
              ((a + (-2. + r) * np.sqrt(r)) * (r ** 3 + a ** 2 * (2. + r))) / np.sqrt(1 + (2. * a) / r ** 1.5 - 3. / r))) /
            (r ** 3 * np.sqrt(2. * a * np.sqrt(r) + (-3. + r) * r) * (a ** 2 + (-2. + r) * r)))


def _theta_of_x2(x2):
    """theta(X2) of the default uniform map (vofx_matthewcoords, coord.c:147)."""
    return np.pi * (x2 + 1.0) / 2.0


def _bsq(P, gcov, gcon):
    """b^2 of cell states (get_state, GPU_phys_mhd.h:672) with metric
    components broadcast over the trailing x3 axis."""
    u1, u2, u3 = P[U1], P[U2], P[U3]
    g = gcov
    qsq = (g[4] * u1 * u1 + g[7] * u2 * u2 + g[9] * u3 * u3 +
           2. * (g[5] * u1 * u2 + g[6] * u1 * u3 + g[8] * u2 * u3))
    gamma = np.sqrt(1. + np.maximum(qsq, 0.0))
    alpha = 1. / np.sqrt(-gcon[0])
    ucon = [gamma / alpha] + [P[U1 + j - 1] - gamma * gcon[j] * alpha * alpha / alpha for j in (1, 2, 3)]

    def lower(v):
        return [g[0] * v[0] + g[1] * v[1] + g[2] * v[2] + g[3] * v[3],
                g[1] * v[0] + g[4] * v[1] + g[5] * v[2] + g[6] * v[3],
                g[2] * v[0] + g[5] * v[1] + g[7] * v[2] + g[8] * v[3],
                g[3] * v[0] + g[6] * v[1] + g[8] * v[2] + g[9] * v[3]]
    ucov = lower(ucon)
    b0 = P[B1] * ucov[1] + P[B2] * ucov[2] + P[B3] * ucov[3]
    bcon = [b0] + [(P[B1 + j - 1] + b0 * ucon[j]) / ucon[0] for j in (1, 2, 3)]
    bcov = lower(bcon)
    return sum(bcon[k] * bcov[k] for k in range(4))


def fm_torus(n1, n2, n3, spin=0.9375, rin=6.0, rmax=12.0, gam=13.0 / 9.0, kappa=1.e-3, beta=100.0,
             rout=None, seed=12345, noise=0.04, rho_atm=1.e-14, u_atm=1.e-16, cour=0.8, ng=3,
             generic=0.0, geometry=None) -> Problem:
    """Magnetised Fishbone-Moncrief torus around a Kerr hole in the reference's
    code coordinates. n3 > 1: transmissive poles; n3 == 1: axisymmetric with
    reflective poles. The atmosphere is the reference's 1e-7*RHOMIN / 1e-7*UUMIN
    (init_torus.c:211-212), also divided by the density maximum. ng: ghost
    layers (3; 2 suits the linear MC reconstruction). generic > 0 removes the
    exact ties of this state (flat atmosphere, equatorial mirror symmetry,
    zero velocities and field outside the torus), at which the limiters and
    upwind switches are not differentiable: seeded relative noise of that size
    on rho, u and the velocities, a power-law atmosphere, and a weak seeded
    field everywhere (vector potential scaled with sqrt(rho)). geometry: the
    metric-table builder, called like api.build_geometry (default: the
    library's hamr_build_geometry)."""
    if rout is None:
        rout = 4.0 * rmax * 2.0
    startx, dx = ks_grid(n1, n2, n3, spin, rout)
    geo = (geometry or build_geometry)("ks", spin, n1, n2, n3, startx, dx, ng)
    ks, p, ps = _alloc(n1, n2, n3, ng)
    g1, g2 = n1 + 2 * ng, n2 + 2 * ng
    g3 = n3 + 2 * ng if n3 > 1 else 1
    gs = geo.gsize
    a = spin
    act1 = slice(ng, ng + n1)
    act2 = slice(ng, ng + n2)
    # zone-centre code coordinates and BL radius / colatitude of active zones
    X1 = startx[1] + (np.arange(n1) + 0.5) * dx[1]
    X2 = startx[2] + (np.arange(n2) + 0.5) * dx[2]
    r = np.exp(X1)[:, None]
    th = _theta_of_x2(X2)[None, :]
    sth, cth = np.sin(th), np.cos(th)
    l = lfish(a, rmax)
    DD = r * r - 2. * r + a * a
    AA = (r * r + a * a) ** 2 - DD * a * a * sth * sth
    SS = r * r + a * a * cth * cth
    thin = np.pi / 2.
    sthin, cthin = np.sin(thin), np.cos(thin)
    DDin = rin * rin - 2. * rin + a * a
    AAin = (rin * rin + a * a) ** 2 - DDin * a * a * sthin * sthin
    SSin = rin * rin + a * a * cthin * cthin
    with np.errstate(invalid="ignore", divide="ignore"):
        lnh = (0.5 * np.log((1. + np.sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * sth * AA * sth))) / (SS * DD / AA))
               - 0.5 * np.sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * AA * sth * sth)) - 2. * a * r * l / AA
               - (0.5 * np.log((1. + np.sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin)))
                               / (SSin * DDin / AAin))
                  - 0.5 * np.sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin))
                  - 2. * a * rin * l / AAin))
    lnh = np.where(r >= rin, lnh, 1.0)
    inside = (lnh >= 0.) & (r >= rin)
    hm1 = np.where(inside, np.exp(np.where(inside, lnh, 0.0)) - 1., 0.)
    ratm, uatm = (rho_atm * (r / rin) ** -1.5, u_atm * (r / rin) ** -2.5) if generic > 0 else (rho_atm, u_atm)
    rho = np.where(inside, (np.maximum(hm1, 0.) * (gam - 1.) / (kappa * gam)) ** (1. / (gam - 1.)), ratm)
    u = np.where(inside, kappa * rho ** gam / (gam - 1.), uatm)
    # BL u^phi of the torus, then u^t from normalisation; u^r = u^theta = 0
    with np.errstate(invalid="ignore", divide="ignore"):
        expm2chi = SS * SS * DD / (AA * AA * sth * sth)
        up1 = np.sqrt((-1. + np.sqrt(1. + 4. * l * l * expm2chi)) / 2.)
        up = 2. * a * r * np.sqrt(1. + up1 * up1) / np.sqrt(AA * SS * DD) + np.sqrt(SS / AA) * up1 / sth
    up = np.where(inside, up, 0.0)
    gtt = -(1. - 2. * r / SS)
    gtp = -2. * a * r * sth * sth / SS
    gpp = (r * r + a * a + 2. * a * a * r * sth * sth / SS) * sth * sth
    BB = 2. * gtp * up
    CC = 1. + gpp * up * up
    with np.errstate(invalid="ignore"):
        ut = (-BB - np.sqrt(BB * BB - 4. * gtt * CC)) / (2. * gtt)
    # KS u^t, u^phi equal the BL ones when u^r = 0; dphi/dX3 = 1, so the code
    # four-velocity is (ut, 0, 0, up); relative velocity u~^i = u^i - u^t g^{0i}/g^{00}
    gcon = [_geo_plane(geo, gs, g1, g2, "gcon", c, CENT)[act1, act2] for c in range(10)]
    gcov = [_geo_plane(geo, gs, g1, g2, "gcov", c, CENT)[act1, act2] for c in range(10)]
    util1 = -ut * gcon[1] / gcon[0]
    util2 = -ut * gcon[2] / gcon[0]
    util3 = up - ut * gcon[3] / gcon[0]
    shape3 = (n1, n2, n3)
    rng = np.random.default_rng(seed)
    rho3 = np.broadcast_to(rho[:, :, None], shape3).copy()
    u3 = np.broadcast_to(u[:, :, None], shape3).copy()
    pert = 1. + noise * (rng.random(shape3) - 0.5)
    u3 = np.where(inside[:, :, None], u3 * pert, u3)
    if not inside.any():
        raise ValueError(f"no bound torus for a={a}, r_in={rin}, r_max={rmax} on this grid")
    rhomax = rho3[np.broadcast_to(inside[:, :, None], shape3)].max()
    rho3 /= rhomax
    u3 /= rhomax
    P = p.reshape(NPR, ks)[:, :g1 * g2 * g3].reshape(NPR, g1, g2, g3)
    act3 = slice(ng, ng + n3) if n3 > 1 else slice(0, 1)
    Pa = P[:, act1, act2, act3]
    Pa[RHO] = rho3
    Pa[UU] = u3
    Pa[U1] = np.where(inside, util1, 0.0)[:, :, None]
    Pa[U2] = np.where(inside, util2, 0.0)[:, :, None]
    Pa[U3] = np.where(inside, util3, 0.0)[:, :, None]
    if generic > 0:
        grng = np.random.default_rng(seed + 1)
        Pa[RHO] *= 1. + generic * grng.standard_normal(shape3)
        Pa[UU] *= 1. + generic * grng.standard_normal(shape3)
        for k in (U1, U2, U3):
            Pa[k] += generic * 1e-2 * grng.standard_normal(shape3)
    Pa[KTOT] = (gam - 1.) * Pa[UU] * Pa[RHO] ** (-gam)
    # single poloidal loop: A_phi at zone corners from the corner-averaged density
    rho2 = rho / rhomax
    rpad = np.pad(rho2, 1, mode="edge")
    rho_av = 0.25 * (rpad[1:, 1:] + rpad[:-1, 1:] + rpad[1:, :-1] + rpad[:-1, :-1])   # (n1+1, n2+1)
    A = np.maximum(rho_av - 0.2, 0.0)
    if generic > 0:
        A = A + generic * A.max() * np.sqrt(np.maximum(rho_av, 0.)) * grng.standard_normal(A.shape)
    gdf1 = _geo_plane(geo, gs, g1, g2, "gdet", 0, FACE1)[ng:ng + n1 + 1, act2]
    gdf2 = _geo_plane(geo, gs, g1, g2, "gdet", 0, FACE2)[act1, ng:ng + n2 + 1]
    gdc = _geo_plane(geo, gs, g1, g2, "gdet", 0, CENT)[act1, act2]
    b1 = (A[:, 1:] - A[:, :-1]) / dx[2] / gdf1          # (n1+1, n2) on x1-faces
    b2 = -(A[1:, :] - A[:-1, :]) / dx[1] / gdf2         # (n1, n2+1) on x2-faces
    Bc1 = 0.5 * (b1[:-1] * gdf1[:-1] + b1[1:] * gdf1[1:]) / gdc
    Bc2 = 0.5 * (b2[:, :-1] * gdf2[:, :-1] + b2[:, 1:] * gdf2[:, 1:]) / gdc
    Pa[B1] = Bc1[:, :, None]
    Pa[B2] = Bc2[:, :, None]
    Pa[B3] = 0.0
    # normalise to the minimum plasma beta p_max / (b^2_max / 2) (init_mag.c:355-357)
    bsq = _bsq(Pa, [c[:, :, None] for c in gcov], [c[:, :, None] for c in gcon])
    pmax = ((gam - 1.) * Pa[UU]).max()
    bsq_max = bsq.max()
    norm = np.sqrt(pmax / (0.5 * bsq_max) / beta) if bsq_max > 0 else 0.0
    Pa[B1] *= norm
    Pa[B2] *= norm
    S = ps.reshape(3, ks)[:, :g1 * g2 * g3].reshape(3, g1, g2, g3)
    S[0, ng:ng + n1 + 1, act2, act3] = (b1 * norm)[:, :, None]
    S[1, act1, ng:ng + n2 + 1, act3] = (b2 * norm)[:, :, None]
    bc = ("outflow", "pole_trans", "periodic") if n3 > 1 else ("outflow", "pole_refl", "periodic")
    return Problem(n1, n2, n3, ng, ks, gs, (dx[1], dx[2], dx[3]), gam, cour, bc, (1, 1), True, geo, p, ps,
                   coords="ks", spin=spin, startx=tuple(startx))


def torus_ensemble(count=64, nmin=32, nmax=96, seed=2024, spin_max=0.99, rmax_range=(10.0, 16.0),
                   rin=6.0, **kw):
    """Seeded ensemble of magnetised FM tori of uneven sizes: per member, each
    of n1, n2, n3 drawn uniformly from [nmin, nmax] (n3 even, for the
    transmissive poles), spin a ~ U[0, spin_max], r_max ~ U[rmax_range], inner
    edge r_in, outer boundary 8 r_max; draws that admit no bound torus are
    redrawn. Returns (problems, draws)."""
    rng = np.random.default_rng(seed)
    out, draws = [], []
    while len(out) < count:
        n1, n2, n3 = (int(x) for x in rng.integers(nmin, nmax + 1, size=3))
        n3 += n3 % 2
        a = float(rng.uniform(0.0, spin_max))
        rmax = float(rng.uniform(*rmax_range))
        try:
            out.append(fm_torus(n1, n2, n3, spin=a, rin=rin, rmax=rmax, rout=8.0 * rmax,
                                seed=int(rng.integers(1 << 30)), **kw))
        except ValueError:
            continue   # (a, r_max) admits no bound torus with this inner edge: draw again
        draws.append(dict(n=(n1, n2, n3), spin=a, rmax=rmax))
    return out, draws
