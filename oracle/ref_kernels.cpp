/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Host build of the reference's own CUDA kernel bodies. GPU_program1.cu and the
 * GPU_*.h headers it includes are compiled as host C++ (see ref_shim/hostcuda.h)
 * against a configured copy of the reference's config.h, and the functions below
 * walk each kernel's launch grid thread by thread, in the order the reference's
 * host code launches them for one uniform block:
 *
 *   advance_GPU (step_ch.c:997-1335) for a block with AMR_TIMELEVEL == 1:
 *     GPU_fluxcalc2D(dir = 3, 2, 1)      GPU_main.cu:560   fluxcalcprep + fluxcalc2D2
 *     fluxcalc_GPU (host min of dtij)     GPU_main.cu:1091
 *     GPU_fix_flux (reflective poles)     GPU_main.cu:1126  step_ch.c:1209
 *     GPU_consttransport1/2               GPU_main.cu:1365,1393
 *     E_average (transmissive poles)      const_trans.c:268-503 (restated below:
 *                                         its MPI pack/unpack is host glue)
 *     GPU_consttransport3                 GPU_main.cu:1535
 *     GPU_fixup                           GPU_main.cu:1740
 *
 * Buffers follow the reference's device layout: cell arrays are NPR planes of
 * ksize doubles, index (i*G2 + j)*G3 + z (GPU_program1.cu:90-94); metric tables
 * are axisymmetric (i*G2 + j) planes (GPU_main.cu:139-300).
 *
 * Output of this file is only used by tests to pin oracle/hamr_oracle.c.
 */
#include "hostcuda.h"
struct hc_dim3 threadIdx, blockIdx, blockDim;
#include "GPU_program1.cu"

/* Walks a 1-D launch of nblocks x nthreads. Threads of a block run one after
 * another in DESCENDING thread order: fluxcalc2D2's shared-memory tree
 * reduction (GPU_program1.cu:1056-1067) then sees exactly the values it would
 * see with the barriers, because thread t only reads slots t+i that belong to
 * threads which have already finished every level above i. */
template <typename F>
static void run_grid(long nthreads_total, int bs, F body) {
    long nb = (nthreads_total + bs - 1) / bs;
    blockDim.x = bs; blockDim.y = blockDim.z = 1;
    for (long b = 0; b < nb; b++) {
        blockIdx.x = (unsigned)b;
        for (int t = bs - 1; t >= 0; t--) {
            threadIdx.x = (unsigned)t;
            body();
        }
    }
}

static const int G1 = BS_1 + 2 * N1G, G2 = BS_2 + 2 * N2G, G3 = BS_3 + 2 * N3G;
static const long KSIZE = (long)G1 * G2 * G3 + (LOCAL_WORK_SIZE - ((long)G1 * G2 * G3) % LOCAL_WORK_SIZE);
static const long GSIZE = (long)G1 * G2 + (LOCAL_WORK_SIZE - ((long)G1 * G2) % LOCAL_WORK_SIZE);

extern "C" {

/* dims[0..8] = BS_1, BS_2, BS_3, N1G, N2G, N3G, NPR, ksize, gsize; gam = GAMMA */
void ref_dims(long *dims, double *gam) {
    dims[0] = BS_1; dims[1] = BS_2; dims[2] = BS_3;
    dims[3] = N1G; dims[4] = N2G; dims[5] = N3G;
    dims[6] = NPR; dims[7] = KSIZE; dims[8] = GSIZE;
    *gam = GAMMA;
}

/* Directional CFL restriction: min over work-group minima in (1e-6, 1e9), as the
 * host loop of fluxcalc_GPU (GPU_main.cu:1103-1121). */
static double host_dt_min(const double *dtij, long ngroups) {
    double ndt = 1.e9;
    for (long y = 0; y < ngroups; y++)
        if (dtij[y] < ndt && dtij[y] < 1.e9 && dtij[y] > 1.e-6) ndt = dtij[y];
    return ndt;
}

/*
 * One RK2 sub-step (full = 0: half step writing ph/psh, full = 1: full step
 * writing p/ps) exactly as advance_GPU launches it for one block.
 *   Dt      sub-step length (0.5*dt or dt)
 *   dt      the step's dt (E_average scales by it, GPU_boundcomE.cu:58)
 *   pole1/2 POLE_1/POLE_2 of GPU_main.cu:566-567
 *   calc_dt nonzero: also return the directional CFL limits in dtdir[1..3]
 * work arrays (all ksize-planar, zero-initialised by the caller):
 *   F1,F2,F3,dq1,dq2 : NPR planes; E_cent, emf : 4 planes; storage2: NPR planes
 */
/* HLLC builds (FRAME_TRANSFORM): the orthonormal face frames, in the device
 * layout get_trans reads (GPU_hllc.h:878-900), are supplied by the caller
 * (set_Mud, hllc.c:20-164, is host code bound to the reference's globals). */
static const double *g_mud = nullptr, *g_mudinv = nullptr;
void ref_set_mud(const double *mud, const double *mudinv) {
    g_mud = mud;
    g_mudinv = mudinv;
}
long ref_mud_plane(void) { return (long)(BS_2 + 2 * N2G) * (BS_1 + 2 * N1G) + FIX_MEM2; }
int ref_nsolver(void) { return NSOLVER; }

void ref_stage(int full, double Dt, double dt, double cour,
               double dx1, double dx2, double dx3, int pole1, int pole2,
               double *p, double *ph, double *ps, double *psh, double *storage2,
               double *F1, double *F2, double *F3, double *dq1, double *dq2,
               double *E_cent, double *emf, int *pflag, int *failimage,
               const double *gcov, const double *gcon, const double *gdet,
               const double *conn, const double *radius,
               int calc_dt, double *dtdir) {
    double *pin = full ? ph : p;
    double *psin = full ? psh : ps;
    double *Fd[4] = {0, F1, F2, F3};
    double dxd[4] = {0, dx1, dx2, dx3};
    int dirs[3] = {3, 2, 1};
    for (int di = 0; di < 3; di++) {
        int dir = dirs[di];
        if (dir == 3 && !(N3G > 0)) { dtdir[3] = 1e9; continue; }
        long nprep = (long)(BS_1 + 2 * D1) * (BS_2 + 2 * D2) * (BS_3 + 2 * D3);
        run_grid(nprep, LOCAL_WORK_SIZE, [&] {
            fluxcalcprep(Fd[dir], dq1, dq2, pin, dir, MC, 0, NULL, pole1, pole2);
        });
        long nface = (long)(BS_1 + 2 * D1 - (dir == 1)) * (BS_2 + 2 * D2 - (dir == 2)) * (BS_3 + 2 * D3 - (dir == 3));
        long ngroups = ((LOCAL_WORK_SIZE - nface % LOCAL_WORK_SIZE) + nface) / LOCAL_WORK_SIZE;
        double *dtij = (double *)calloc(ngroups, sizeof(double));
        run_grid(ngroups * LOCAL_WORK_SIZE, LOCAL_WORK_SIZE, [&] {
#if (FRAME_TRANSFORM)
            fluxcalc2D_FT(Fd[dir], dq1, dq2, pin, psin, gcov, gcon, gdet, g_mud, g_mudinv, MC, dir, cour, dtij,
                          pole1, pole2, dxd[dir], calc_dt ? 1 : 0, full);
#else
            fluxcalc2D2(Fd[dir], dq1, dq2, pin, psin, gcov, gcon, gdet, MC, dir, cour, dtij,
                        pole1, pole2, dxd[dir], calc_dt ? 1 : 0, full);
#endif
        });
        if (calc_dt) dtdir[dir] = host_dt_min(dtij, ngroups);
        free(dtij);
    }
#if (BOUND_TYPE2 == REFLECTIVE)
    {
        long nfix = (long)(BS_1 + 2 * N1G) * (BS_3 + 2 * N3G) + (long)(BS_2 + 2 * N2G) * (BS_3 + 2 * N3G);
        int nbr1 = pole1 ? -1 : 0, nbr3 = pole2 ? -1 : 0;
        /* inner/outer radial neighbours absent: no-inflow flux fix (INFLOW == 0) */
        run_grid(nfix, LOCAL_WORK_SIZE, [&] { fix_flux(F1, F2, F3, nbr1, -1, nbr3, -1); });
    }
#endif
    long n1 = (long)(BS_1 + 2 * D1) * (BS_2 + 2 * D2) * (BS_3 + 2 * D3);
    run_grid(n1, LOCAL_WORK_SIZE, [&] { consttransport1(pin, E_cent, gcov, gcon, gdet); });
    long n2 = (long)(BS_1 + D1) * (BS_2 + D2) * (BS_3 + D3);
    run_grid(n2, LOCAL_WORK_SIZE, [&] {
        consttransport2(emf, E_cent, F1, F2, F3, pin, gcov, gcon, gdet, pole1, pole2);
    });
#if (BOUND_TYPE2 == TRANSMISSIVE)
    /* E_average (const_trans.c:268) for a block that holds every phi cell:
     * read_E_avg (const_trans.c:460) packs dt*E1 (packsend2E, GPU_program2.cu:1807)
     * over active i + upper ghosts and active z, averages over z, and
     * write_E_avg (const_trans.c:504) unpacks with calc_corr == 4
     * (GPU_program2.cu:2231): E1 = avg / dt, E3 = 0 on the polar edge. */
    for (int side = 0; side < 2; side++) {
        if ((side == 0 && !pole1) || (side == 1 && !pole2)) continue;
        int jp = side == 0 ? N2G : BS_2 + N2G;
        for (int i = N1G; i < BS_1 + 2 * N1G; i++) {
            double avg = 0.;
            for (int z = N3G; z < BS_3 + N3G; z++) avg += dt * emf[1 * KSIZE + ((long)i * G2 + jp) * G3 + z];
            avg /= (double)(BS_3);
            double avg_new = avg / ((double)1);
            for (int z = N3G; z < BS_3 + 2 * N3G; z++) {
                emf[1 * KSIZE + ((long)i * G2 + jp) * G3 + z] = avg_new / dt;
                emf[3 * KSIZE + ((long)i * G2 + jp) * G3 + z] = 0.;
            }
        }
    }
#endif
    run_grid(n2, LOCAL_WORK_SIZE, [&] {
        consttransport3(dx1, dx2, dx3, gdet, ps, full ? ps : psh, emf, Dt, pole1, pole2);
    });
    long n4 = (long)BS_1 * BS_2 * BS_3;
    run_grid(n4, LOCAL_WORK_SIZE, [&] {
        fixup(p, full ? ph : p, full ? p : ph, storage2, full ? ps : psh, F1, F2, F3, dq1, radius,
              pflag, failimage, gcov, gcon, gdet, conn, dx1, dx2, dx3, Dt, full, pole1, pole2, 0.0);
    });
}

/* Reference polar ghost fill for transmissive poles, boundprim2_trans
 * (GPU_bounds.h:510), NB_3 == 1 path of bound_prim (bounds.c:108-113). */
void ref_bound_pole_trans(double *pv, double *ps, const double *gdet, int pole1, int pole2) {
    long n = 2L * (BS_1 + 2 * N1G) * (BS_3 + 2 * N3G);
    run_grid(n, LOCAL_WORK_SIZE, [&] { boundprim2_trans(pv, gdet, pole1 ? 1 : 0, pole2 ? 1 : 0, ps); });
}

/* Single-cell entry points of the reference's inversion chain, for pinning the
 * restated Newton solvers on sampled states. U is NPR conserved values. */
int ref_utoprim_2d(double *U, const double *gcov10, const double *gcon10, double gdet, double *prim) {
    double gc[10], gn[10];
    for (int k = 0; k < 10; k++) { gc[k] = gcov10[k]; gn[k] = gcon10[k]; }
    return Utoprim_2d(U, gc, gn, gdet, prim, NEWT_TOL, 0);
}
int ref_utoprim_1dvsq2fix1(double *U, const double *gcov10, const double *gcon10, double gdet, double *prim) {
    double gc[10], gn[10];
    for (int k = 0; k < 10; k++) { gc[k] = gcov10[k]; gn[k] = gcon10[k]; }
    return Utoprim_1dvsq2fix1(U, gc, gn, gdet, prim, NEWT_TOL, 0, FULL_ENTROPY);
}
int ref_utoprim_1dfix1(double *U, const double *gcov10, const double *gcon10, double gdet, double *prim) {
    double gc[10], gn[10];
    for (int k = 0; k < 10; k++) { gc[k] = gcov10[k]; gn[k] = gcon10[k]; }
    return Utoprim_1dfix1(U, gc, gn, gdet, prim, NEWT_TOL, 0, FULL_ENTROPY);
}
int ref_utoprim_nm(double *U, const double *gcov10, const double *gcon10, double gdet, double *prim) {
    double gc[10], gn[10];
    for (int k = 0; k < 10; k++) { gc[k] = gcov10[k]; gn[k] = gcon10[k]; }
    return Utoprim_NM(U, gc, gn, gdet, prim, NEWT_TOL, 0);
}

/* primtoflux (GPU_phys_mhd.h:432) for one state at one geometry point. */
void ref_primtoflux(double *pr, const double *gcov10, const double *gcon10, double gdet, int dir,
                    double *flux, double *vmax, double *vmin) {
    struct of_geom geom;
    for (int k = 0; k < 10; k++) { geom.gcov[k] = gcov10[k]; geom.gcon[k] = gcon10[k]; }
    geom.g = gdet;
    struct of_state q;
    get_state(pr, &geom, &q);
    primtoflux(pr, &q, dir, &geom, flux, vmax, vmin);
}

/* para (GPU_interp.h:60) on one 5-point stencil. */
void ref_para(const double *x, double *l, double *r) { para(x[0], x[1], x[2], x[3], x[4], l, r); }

/* fixuputoprim (GPU_fixup.h:735-852) over the active zones: zones with
 * pflag != 0 are reset to the floor state with zero velocity and passed
 * through fixup_cell (a no-op as compiled: its floor body is #if 0). Its
 * call sits commented out after GPU_fixup in advance_GPU (step_ch.c:1281). */
void ref_fixuputoprim(double *pv, const double *radius, const double *gcov, const double *gcon,
                      const double *gdet, int *pflag, int *failimage) {
    long n4 = (long)BS_1 * BS_2 * BS_3;
    run_grid(n4, LOCAL_WORK_SIZE, [&] { fixuputoprim(pv, radius, gcov, gcon, gdet, pflag, failimage); });
}

} /* extern "C" */
