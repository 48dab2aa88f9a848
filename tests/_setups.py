"""Seeded synthetic blocks for the parity tests.

States are smooth, magnetised and sub-relativistic, with a divergence-free
staggered field built as the discrete curl of an edge vector potential, so
every branch of the step (PPM clamps, HLL upwinding, EMF upwind selection,
Newton inversion) is exercised. ``stress`` adds cells that make the primary
inversion fail, to walk the entropy fallbacks.
"""
import dataclasses
import numpy as np

from oracle import oracle as O


def mks_grid(n1, n2, n3, spin, rout):
    """startx / dx of the reference's log-r, uniform-theta grid
    (set_gridparam / set_points, coord.c:327-461)."""
    rin = 0.9 * (1.0 + np.sqrt(1.0 - spin * spin))
    frac = 1.0 - 2.0 / n2 if n3 > 1 else 1.0   # transmissive poles leave one cell
    startx = [0.0, np.log(rin), -1.0 + (1.0 - frac), 0.0]
    dx = [0.0, (np.log(rout) - np.log(rin)) / n1, 2.0 * frac / n2, 2.0 * np.pi / n3]
    return startx, dx


def fill_synthetic(blk: O.Block, geo: O.Geometry, dx, seed=1, bamp=0.02, stress=False):
    rng = np.random.default_rng(seed)
    P = blk.view("p")
    g1, g2, g3 = blk.g1, blk.g2, blk.g3
    I, J, Z = np.meshgrid(np.arange(g1), np.arange(g2), np.arange(g3), indexing="ij")
    P[O.RHO] = 1.0 + 0.3 * np.sin(0.7 * I) * np.cos(0.9 * J) + 0.05 * rng.random(I.shape)
    P[O.UU] = 0.1 + 0.03 * np.cos(0.5 * I + 0.3 * Z) + 0.01 * rng.random(I.shape)
    P[O.U1] = 0.05 * np.sin(0.3 * J + 0.2 * Z) + 0.01 * rng.random(I.shape)
    P[O.U2] = 0.02 * np.cos(0.4 * I) + 0.005 * rng.random(I.shape)
    P[O.U3] = 0.1 * np.sin(0.2 * I) + 0.01 * rng.random(I.shape)
    P[O.KTOT] = 0.01 + 0.001 * rng.random(I.shape)
    gs = blk.gsize
    gd = lambda loc: geo.gdet[loc * gs: loc * gs + g1 * g2].reshape(g1, g2)[:, :, None]
    gdf1, gdf2, gdf3, gdc = gd(O.FACE1), gd(O.FACE2), gd(O.FACE3), gd(O.CENT)
    # edge vector potential on a (g1+1, g2+1, g3+1) lattice
    a = np.arange(g1 + 1)[:, None, None]
    b = np.arange(g2 + 1)[None, :, None]
    c = np.arange(g3 + 1)[None, None, :]
    A3 = bamp * np.sin(0.5 * a) * np.cos(0.6 * b) + 0.0 * c
    A1 = bamp * 0.5 * np.cos(0.4 * b + 0.3 * c) + 0.0 * a
    A2 = bamp * 0.5 * np.sin(0.35 * a + 0.25 * c) + 0.0 * b
    d1, d2, d3 = dx[1], dx[2], dx[3]
    three_d = g3 > 1
    s1 = (A3[:g1, 1:, :g3] - A3[:g1, :g2, :g3]) / d2
    s2 = -(A3[1:, :g2, :g3] - A3[:g1, :g2, :g3]) / d1
    s3 = np.zeros((g1, g2, g3))
    if three_d:
        s1 = s1 - (A2[:g1, :g2, 1:] - A2[:g1, :g2, :g3]) / d3
        s2 = s2 + (A1[:g1, :g2, 1:] - A1[:g1, :g2, :g3]) / d3
        s3 = (A2[1:, :g2, :g3] - A2[:g1, :g2, :g3]) / d1 - (A1[:g1, 1:, :g3] - A1[:g1, :g2, :g3]) / d2
    PS = blk.view("ps")
    PS[0] = s1 / gdf1
    PS[1] = s2 / gdf2
    PS[2] = s3 / gdf3
    P[O.B1] = 0.0
    P[O.B2] = 0.0
    P[O.B1][:-1] = 0.5 * (s1[:-1] + s1[1:]) / gdc[:-1]
    P[O.B2][:, :-1] = 0.5 * (s2[:, :-1] + s2[:, 1:]) / gdc[:, :-1]
    if three_d:
        P[O.B3][:, :, :-1] = 0.5 * (s3[:, :, :-1] + s3[:, :, 1:]) / gdc
    else:
        P[O.B3] = 0.01 * np.cos(0.3 * I)
    if stress:
        # strongly magnetised, nearly cold pockets: the Noble 2D solve fails there
        sel = np.random.default_rng(3).random(I.shape) < 0.05
        P[O.UU][sel] = 1e-7
        P[O.RHO][sel] = 1e-5


def product_geometry(coords, spin, n1, n2, n3, gsize, startx, dx):
    """The library's host metric builder (hamr_build_geometry), which the ABI
    tests pin bit for bit to the reference's metric code, as oracle tables."""
    from hamr_gamma_wind_b200 import api
    g = api.build_geometry(coords, spin, n1, n2, n3, startx, dx, gsize=gsize)
    return O.Geometry(gsize, g.gcov, g.gcon, g.gdet, g.conn)


def make_setup(variant, spin=0.9375, rout=40.0, seed=1, stress=False, cour=0.8, dims=None,
               geometry="reference"):
    """Reference-variant block with the reference's own geometry tables
    (geometry="product": the library's geometry builder instead; dims =
    ((n1, n2, n3, ..., ksize, gsize), gam) when the reference build is absent)."""
    dims, gam = dims if dims is not None else O.ref_dims(variant)
    n1, n2, n3 = (int(x) for x in dims[:3])
    ksize, gsize = int(dims[7]), int(dims[8])
    blk = O.Block(n1, n2, n3, int(dims[3]), ksize, gsize)
    if variant == "ot":
        startx = [0.0, 0.0, 0.0, 0.0]
        dx = [0.0, 1.0 / n1, 1.0 / n2, 1.0]
        geo = (O.ref_geometry(variant, 0.0, startx, dx) if geometry == "reference"
               else product_geometry("cartesian", 0.0, n1, n2, n3, gsize, startx, dx))
        bc = (O.BC_PERIODIC, O.BC_PERIODIC, O.BC_PERIODIC)
        poles = (0, 0)
    else:
        startx, dx = mks_grid(n1, n2, n3, spin, rout)
        geo = (O.ref_geometry(variant, spin, startx, dx) if geometry == "reference"
               else product_geometry("ks", spin, n1, n2, n3, gsize, startx, dx))
        bc = (O.BC_OUTFLOW, O.BC_POLE_TRANS if n3 > 1 else O.BC_POLE_REFL, O.BC_PERIODIC)
        poles = (1, 1)
    fill_synthetic(blk, geo, dx, seed=seed, stress=stress)
    s = O.Setup(blk, geo, tuple(dx[1:]), gam, cour, poles[0], poles[1], bc,
                ct_upwind=0 if variant == "ot" else 1, recon=1 if variant.endswith("m") else 0,
                riemann={"c": 1, "d": 2}.get(variant[-1], 0))
    O.oracle_bound(s, "p", "ps")
    return s


def clone(s: O.Setup) -> O.Setup:
    return dataclasses.replace(s, blk=s.blk.copy())


def plant_failures(s: O.Setup, frac=0.08, seed=11):
    """Make the inversion fail outright in some zones: a negative internal
    energy there leaves every solver of the fallback chain without a
    physical root. A random fraction of the active zones plus a solid 3 x 3
    (x 3) patch, so that failed zones also border one another."""
    b = s.blk
    P = b.active("p")
    sel = np.random.default_rng(seed).random(P[0].shape) < frac
    i0, j0 = P.shape[1] // 2, P.shape[2] // 2
    z0 = P.shape[3] // 2
    dz = 3 if P.shape[3] > 1 else 1
    sel[i0:i0 + 3, j0:j0 + 3, z0:z0 + dz] = True
    P[O.UU][sel] = -1e-2
    O.oracle_bound(s, "p", "ps")
    return int(sel.sum())
