"""Writes the golden fixtures of tests/test_golden.py from the reference's own
kernel code, built for the host from the reference sources (oracle/Makefile,
`make -C oracle ref REF=<reference source tree>`). Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (numpy .npz, compressed):
  ref_cells.npz   single-cell known answers: PPM edge values (para), fluxes and
                  fast speeds (primtoflux), and the four inversions (Noble 2D,
                  1dvsq2fix1, 1dfix1, Newman) on stressed states, at metric
                  points of the 3-D torus grid
  ref_<v>.npz     per compile-time variant (t3: 3-D torus 16x8x8, t2: 2-D
                  torus 24x24, ot: 2-D Orszag-Tang box 32x32): the half
                  sub-step's outputs and the state after two RK2 steps of the
                  reference kernels on a seeded synthetic block, on the
                  active zones only; plus SHA-256 digests of the metric tables
                  and of the initial state, so the test can confirm it rebuilt
                  exactly the same inputs without the reference present.
  ref_repair.npz  the failed-zone repairs (t3, t2): the reference's CPU
                  fixup_utoprim on seeded random states and flag patterns
                  (two flag densities), and its fixuputoprim kernel after a
                  half sub-step of the reference kernels on a seeded block
                  with planted failed zones; active zones only.

  ref_dump_t2.npz the parameter header, float dump and double restart files the
                  reference's own writers (dump_params, dump_block,
                  rdump_block_write; oracle/ref_dumpio.c) produce for the 2-D
                  variant's block with a seeded generic state (dump_case)
`python tests/golden/make_golden.py repair` writes ref_repair.npz alone,
`... dump` ref_dump_t2.npz alone.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from tests._setups import clone, make_setup, plant_failures  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 13
DT = {"t3": 0.002, "t2": 0.002, "ot": 0.002}


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, np.float64).tobytes())
    return h.hexdigest()


def active(blk, name):
    return blk.active(name).copy()


def variant_fixture(v):
    dims, gam = O.ref_dims(v)
    s = make_setup(v, seed=SEED)
    geo = s.geo
    out = {"dims": np.asarray(dims, np.int64), "gam": gam,
           "geo_sha": digest(geo.gcov, geo.gcon, geo.gdet, geo.conn),
           "in_sha": digest(s.blk.arrays["p"], s.blk.arrays["ps"]), "dt": DT[v]}
    h = clone(s)
    d = O.ref_stage(v, h, 0, 0.5 * DT[v], DT[v], True)
    out["half_ph"] = active(h.blk, "ph")
    out["half_psh"] = active(h.blk, "psh")
    out["half_dtdir"] = np.asarray(d)
    st = clone(s)
    dt = DT[v]
    stage = lambda s_, f, Dt, dd, c: O.ref_stage(v, s_, f, Dt, dd, c)
    bound = lambda s_, a, b: O.oracle_bound(s_, a, b)
    dts = []
    for _ in range(2):
        n = O.step(stage, bound, st, dt)
        dts.append(n)
        dt = min(n, 1.3 * dt)
    out["steps_p"] = active(st.blk, "p")
    out["steps_ps"] = active(st.blk, "ps")
    out["steps_dt"] = np.asarray(dts)
    return out


def cell_fixture():
    rng = np.random.default_rng(SEED)
    L = O.ref("t3")
    _, gam = O.ref_dims("t3")
    s = make_setup("t3", seed=2)
    geo, gs, g2 = s.geo, s.blk.gsize, s.blk.g2
    out = {"gam": gam}
    xs = rng.normal(size=(200, 5)) * rng.choice([1e-3, 1.0, 1e3], size=(200, 1))
    lr = np.zeros((200, 2))
    for n, x in enumerate(xs):
        l1, r1 = np.zeros(1), np.zeros(1)
        L.ref_para(O._ptr(np.ascontiguousarray(x)), O._ptr(l1), O._ptr(r1))
        lr[n] = l1[0], r1[0]
    out["para_x"], out["para_lr"] = xs, lr

    def metric(i, j, loc):
        idx = i * g2 + j
        gcov = np.array([geo.gcov[(c * 5 + loc) * gs + idx] for c in range(10)])
        gcon = np.array([geo.gcon[(c * 5 + loc) * gs + idx] for c in range(10)])
        return gcov, gcon, geo.gdet[loc * gs + idx]

    rows = []
    for _ in range(100):
        i, j, d = int(rng.integers(3, 12)), int(rng.integers(3, 10)), int(rng.integers(0, 4))
        loc = int(rng.choice([O.FACE1, O.FACE2, O.FACE3, O.CENT]))
        gcov, gcon, gdet = metric(i, j, loc)
        pr = np.array([1.0, 0.2, 0.1, 0.01, 0.2, 0.3, 0.02, 0.1, 0.01]) * (1 + 0.2 * rng.random(9))
        f = np.zeros(9)
        v = np.zeros(2)
        L.ref_primtoflux(O._ptr(pr.copy()), O._ptr(gcov), O._ptr(gcon), gdet, d, O._ptr(f), O._ptr(v[:1]),
                         O._ptr(v[1:]))
        rows.append((pr, gcov, gcon, gdet, d, f, v))
    out["ptf_pr"] = np.array([r[0] for r in rows])
    out["ptf_gcov"] = np.array([r[1] for r in rows])
    out["ptf_gcon"] = np.array([r[2] for r in rows])
    out["ptf_gdet"] = np.array([r[3] for r in rows])
    out["ptf_dir"] = np.array([r[4] for r in rows])
    out["ptf_flux"] = np.array([r[5] for r in rows])
    out["ptf_v"] = np.array([r[6] for r in rows])

    for name in ("2d", "1dvsq2fix1", "1dfix1", "nm"):
        keep = []
        trial = 0
        while len(keep) < 80:
            trial += 1
            i, j = int(rng.integers(3, 19)), int(rng.integers(3, 11))
            gcov, gcon, gdet = metric(i, j, O.CENT)
            rho = 10 ** rng.uniform(-6, 0)
            u = rho * 10 ** rng.uniform(-4, 0)
            pr = np.array([rho, u, *(rng.normal(size=3) * 10 ** rng.uniform(-2, 0.5)),
                           *(rng.normal(size=3) * np.sqrt(rho) * 10 ** rng.uniform(-1, 1.5)), 0.0])
            flux = np.zeros(9)
            vv = np.zeros(2)
            O.lib().ho_primtoflux(gam, O._ptr(pr), O._ptr(gcov), O._ptr(gcon), gdet, 0, O._ptr(flux),
                                  O._ptr(vv[:1]), O._ptr(vv[1:]))
            U = flux.copy()
            U[O.UU] += rng.uniform(0, 3.0) * gdet * u
            if trial % 3 == 0:
                U[O.KTOT] *= -1.0
            guess = pr * (1 + 0.01 * rng.normal(size=9))
            if name == "nm":
                O.utoprim("nm", gam, U, gcov, gcon, gdet, guess)
                if O.lib().ho_utoprim_nm_max_index() > 2:
                    continue  # outside the reference's 3-slot pressure history
            r, p = O.ref_utoprim("t3", name, U, gcov, gcon, gdet, guess)
            keep.append((U, gcov, gcon, gdet, guess, r, p))
        out[f"inv_{name}_U"] = np.array([k[0] for k in keep])
        out[f"inv_{name}_gcov"] = np.array([k[1] for k in keep])
        out[f"inv_{name}_gcon"] = np.array([k[2] for k in keep])
        out[f"inv_{name}_gdet"] = np.array([k[3] for k in keep])
        out[f"inv_{name}_guess"] = np.array([k[4] for k in keep])
        out[f"inv_{name}_ret"] = np.array([k[5] for k in keep])
        out[f"inv_{name}_prim"] = np.array([k[6] for k in keep])
    return out


REPAIR_DENSITIES = (0.35, 0.7)


def flag_pattern_setup(dims, gam, density, seed):
    """Seeded random primitives over the whole ghosted block and random
    nonzero flags on a fraction `density` of the active zones (fixup_utoprim
    reads no metric)."""
    n1, n2, n3, ng = (int(x) for x in dims[:4])
    blk = O.Block(n1, n2, n3, ng, int(dims[7]), int(dims[8]))
    rng = np.random.default_rng(seed)
    blk.arrays["p"][:] = rng.random(blk.arrays["p"].size)
    act = blk.active("pflag", 1)[0]
    act[...] = np.where(rng.random(act.shape) < density, rng.integers(1, 7, act.shape), 0)
    geo = O.Geometry.empty(int(dims[8]))
    return O.Setup(blk, geo, (1.0, 1.0, 1.0), gam, 0.8, 0, 0, (0, 0, 0))


def repair_fixture():
    out = {}
    for v in ("t3", "t2"):
        dims, gam = O.ref_dims(v)
        out[f"{v}_dims"], out[f"{v}_gam"] = np.asarray(dims, np.int64), gam
        for k, dens in enumerate(REPAIR_DENSITIES):
            s = flag_pattern_setup(dims, gam, dens, SEED + k)
            out[f"{v}_nb{k}_in_sha"] = digest(s.blk.arrays["p"], s.blk.arrays["pflag"])
            O.ref_fixup_utoprim(v, s, "p")
            out[f"{v}_nb{k}_p"] = active(s.blk, "p")[:5]   # RHO..U3: the planes the repair sets
            out[f"{v}_nb{k}_fi4"] = s.blk.active("failimage")[4].copy()
            assert not s.blk.pflag.any()
        s = make_setup(v, seed=7)
        plant_failures(s, frac=0.08, seed=11)
        out[f"{v}_reset_in_sha"] = digest(s.blk.arrays["p"], s.blk.arrays["ps"])
        O.ref_stage(v, s, 0, 0.0005, 0.001)
        O.ref_fixuputoprim(v, s, "ph")
        out[f"{v}_reset_ph"] = active(s.blk, "ph")[:5]
        out[f"{v}_reset_pflag"] = s.blk.active("pflag", 1)[0].copy()
        assert (out[f"{v}_reset_pflag"] != 0).any()
    return out


def dump_case(v):
    """The block of variant v with a generic state (torus, seeded 1e-3 relative
    perturbation of every entry, ghosts included) and run parameters for the
    dump and restart comparison; returns (problem, Params, prm_d, prm_i)."""
    from hamr_gamma_wind_b200 import dumpio, problems
    dims, _ = O.ref_dims(v) if O.ref_available(v) else (DUMP_DIMS[v], None)
    n1, n2, n3 = (int(x) for x in dims[:3])
    pb = problems.fm_torus(n1, n2, n3, rout=40.0)
    rng = np.random.default_rng(3)
    pb.p[:] *= 1.0 + 1e-3 * rng.standard_normal(pb.p.shape)
    pb.ps[:] *= 1.0 + 1e-3 * rng.standard_normal(pb.ps.shape)
    prm = dumpio.params_for(pb, t=12.5, nstep=40, dt=0.01, spin=0.9375, rin=1.2, rout=40.0, tf=2000.0)
    prm.dump_cnt, prm.rdump_cnt, prm.lim = 3, 7, 1
    prm_d = [prm.t, prm.dt, prm.DTd, prm.DTl, prm.startx1, prm.startx2, prm.startx3, prm.dx1, prm.dx2, prm.dx3,
             prm.tf, prm.a, prm.gam, prm.cour, prm.Rin, prm.Rout, prm.R0]
    prm_i = [prm.nstep, prm.dump_cnt, prm.rdump_cnt, prm.failed, prm.lim, prm.dump_cnt_reduced]
    return pb, prm, prm_d, prm_i


DUMP_DIMS = {"t3": (16, 8, 8), "t2": (24, 24, 1)}


def dump_fixture(v):
    """The reference writers' files (dump_params, dump_block,
    rdump_block_write) for dump_case(v), as byte arrays, and a digest of the
    inputs."""
    import tempfile
    pb, prm, prm_d, prm_i = dump_case(v)
    d = tempfile.mkdtemp()
    paths = [os.path.join(d, f) for f in ("parameters", "new_dump0", "rdump0")]
    O.ref_dump_files(v, pb.p, pb.ps, pb.ksize, pb.geo, prm_d, prm_i, *paths)
    out = {k: np.frombuffer(open(pth, "rb").read(), np.uint8) for k, pth in zip(("params", "dump", "rdump"), paths)}
    out["inputs"] = np.array(digest(pb.p, pb.ps, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet))
    return out


def main():
    if sys.argv[1:] == ["repair"]:
        np.savez_compressed(os.path.join(HERE, "ref_repair.npz"), **repair_fixture())
        return
    if sys.argv[1:] == ["dump"]:
        np.savez_compressed(os.path.join(HERE, "ref_dump_t2.npz"), **dump_fixture("t2"))
        return
    for v in ("t3", "t2", "ot"):
        if not O.ref_available(v):
            raise SystemExit(f"reference host build {v} missing: run `make -C oracle ref REF=<reference source tree>` first")
        np.savez_compressed(os.path.join(HERE, f"ref_{v}.npz"), **variant_fixture(v))
    np.savez_compressed(os.path.join(HERE, "ref_cells.npz"), **cell_fixture())
    np.savez_compressed(os.path.join(HERE, "ref_repair.npz"), **repair_fixture())
    np.savez_compressed(os.path.join(HERE, "ref_dump_t2.npz"), **dump_fixture("t2"))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
