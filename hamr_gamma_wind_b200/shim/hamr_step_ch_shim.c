/*
 * Drop-in shim for the reference's host code: the per-block device step of
 * H-AMR (set_arrays_GPU + GPU_write_metric + GPU_write, then GPU_step_ch /
 * advance_GPU, then GPU_read) routed to this library's C ABI
 * (include/hamr_b200.h) for uniform blocks. It is compiled inside the
 * reference's tree, against its decs.h / config.h, in place of those calls:
 *
 *   hamr_shim_attach(n)   after set_grid() and the initial data, per block:
 *                         replaces set_arrays_GPU (GPU_mem.h:41), GPU_write_metric
 *                         (GPU_main.cu:139) and GPU_write (GPU_main.cu:309)
 *   hamr_shim_step_ch()   replaces GPU_step_ch (step_ch.c:916): 2 x
 *                         AMR_MAXTIMELEVEL sub-steps with the dt refresh every
 *                         AMR_MAXTIMELEVEL steps (step_ch.c:954-975)
 *   hamr_shim_read(n)     replaces GPU_read (GPU_main.cu:2646) before dumps
 *   hamr_shim_detach(n)   frees the block's context
 *
 * The host state stays the reference's: p[nl[n]][index_3D(n, i, j, z)][k] and
 * ps[...][k] (decs.h:58,66) are packed into the library's structure-of-arrays
 * layout (the packing of GPU_write, GPU_main.cu:357-380) and back. The metric
 * comes from the host staging tables GPU_write_metric fills (gcov_GPU, gcon_GPU,
 * gdet_GPU, conn_GPU, decs.h:141-146), which are in the device layout already.
 * Only uniform blocks (no AMR level jumps, one time level): the library steps
 * one block on one GPU.
 */
#include <stdlib.h>

#include "decs.h"
#include "hamr_b200.h"

static hamr_ctx *shim_ctx[NB_LOCAL];
static double *shim_p[NB_LOCAL], *shim_ps[NB_LOCAL];
static long shim_ks[NB_LOCAL];

#define SHIM_G1 (BS_1 + 2 * N1G)
#define SHIM_G2 (BS_2 + 2 * N2G)
#define SHIM_G3 (BS_3 + 2 * N3G)

/* SoA index of cell (i, j, z) of block n (GPU_main.cu:359) */
static long shim_cell(int n, int i, int j, int z) {
    return ((long)(i - N1_GPU_offset[n] + N1G) * SHIM_G2 + (j - N2_GPU_offset[n] + N2G)) * SHIM_G3 +
           (z - N3_GPU_offset[n] + N3G);
}

static void shim_pack(int n) {
    const long ks = shim_ks[nl[n]];
    for (int i = N1_GPU_offset[n] - N1G; i < N1_GPU_offset[n] + BS_1 + N1G; i++)
        for (int j = N2_GPU_offset[n] - N2G; j < N2_GPU_offset[n] + BS_2 + N2G; j++)
            for (int z = N3_GPU_offset[n] - N3G; z < N3_GPU_offset[n] + BS_3 + N3G; z++) {
                const long c = shim_cell(n, i, j, z);
                for (int k = 0; k < NPR; k++) shim_p[nl[n]][k * ks + c] = p[nl[n]][index_3D(n, i, j, z)][k];
                for (int k = 1; k < NDIM; k++) shim_ps[nl[n]][(k - 1) * ks + c] = ps[nl[n]][index_3D(n, i, j, z)][k];
            }
}

static void shim_unpack(int n) {
    const long ks = shim_ks[nl[n]];
    for (int i = N1_GPU_offset[n] - N1G; i < N1_GPU_offset[n] + BS_1 + N1G; i++)
        for (int j = N2_GPU_offset[n] - N2G; j < N2_GPU_offset[n] + BS_2 + N2G; j++)
            for (int z = N3_GPU_offset[n] - N3G; z < N3_GPU_offset[n] + BS_3 + N3G; z++) {
                const long c = shim_cell(n, i, j, z);
                for (int k = 0; k < NPR; k++) p[nl[n]][index_3D(n, i, j, z)][k] = shim_p[nl[n]][k * ks + c];
                for (int k = 1; k < NDIM; k++) ps[nl[n]][index_3D(n, i, j, z)][k] = shim_ps[nl[n]][(k - 1) * ks + c];
            }
}

int hamr_shim_attach(int n) {
    hamr_params prm = {0};
    prm.n1 = BS_1; prm.n2 = BS_2; prm.n3 = BS_3; prm.ng = NG;
    prm.dx1 = dx[nl[n]][1]; prm.dx2 = dx[nl[n]][2]; prm.dx3 = dx[nl[n]][3];
    prm.gam = gam; prm.cour = cour;
    prm.pole1 = block[n][AMR_NBR1] < 0 || block[n][AMR_POLE] == 1 || block[n][AMR_POLE] == 3;
    prm.pole2 = block[n][AMR_NBR3] < 0 || block[n][AMR_POLE] == 2 || block[n][AMR_POLE] == 3;
    prm.bc1 = HAMR_BC_OUTFLOW;
    prm.bc2 = (BOUND_TYPE2 == TRANSMISSIVE) ? HAMR_BC_POLE_TRANS : HAMR_BC_POLE_REFL;
    prm.bc3 = HAMR_BC_PERIODIC;
    prm.ct_upwind = !(CARTESIAN || RESISTIVE);
    prm.precision = HAMR_FP64;
    prm.recon = PPM ? HAMR_RECON_PPM : HAMR_RECON_MC;               /* PPM = 0 builds: MC, NG = 2 */
    prm.riemann = HLLD ? HAMR_RIEMANN_HLLD : (HLLC ? HAMR_RIEMANN_HLLC : HAMR_RIEMANN_HLL);
    prm.inversion = NEWMAN ? HAMR_INV_NM : HAMR_INV_2D;
    prm.floors = 0;   /* the shipped step: fixup_cell's floor body is compiled out */
    prm.repair = 0;   /* and the GPU_fixuputoprim / fixup_utoprim calls are commented out */
    int rc = hamr_ctx_create(&prm, &shim_ctx[nl[n]]);
    if (rc) return rc;
    long ks = 0, gs = 0;
    hamr_strides(shim_ctx[nl[n]], &ks, &gs);
    shim_ks[nl[n]] = ks;
    shim_p[nl[n]] = (double *)malloc(sizeof(double) * NPR * ks);
    shim_ps[nl[n]] = (double *)malloc(sizeof(double) * 3 * ks);
    if (!shim_p[nl[n]] || !shim_ps[nl[n]]) return HAMR_E_NOMEM;
    rc = hamr_set_geometry(shim_ctx[nl[n]], gcov_GPU[nl[n]], gcon_GPU[nl[n]], gdet_GPU[nl[n]], conn_GPU[nl[n]]);
    if (rc) return rc;
    shim_pack(n);
    rc = hamr_upload(shim_ctx[nl[n]], shim_p[nl[n]], shim_ps[nl[n]]);
    return rc ? rc : hamr_bound(shim_ctx[nl[n]]);
}

/* GPU_step_ch for the active blocks: AMR_MAXTIMELEVEL RK2 steps each, the
 * step size refreshed from the CFL limit every AMR_MAXTIMELEVEL steps; the
 * smallest new step size over the blocks becomes dt */
int hamr_shim_step_ch(void) {
    double dt_new = 1.e30;
    for (int m = 0; m < n_active; m++) {
        const int n = n_ord[m];
        double d = dt;
        const int rc = hamr_advance(shim_ctx[nl[n]], AMR_MAXTIMELEVEL, AMR_MAXTIMELEVEL, &d);
        if (rc) return rc;
        if (d < dt_new) dt_new = d;
    }
    t += (double)AMR_MAXTIMELEVEL * dt;
    dt = dt_new;
    nstep += 2 * AMR_MAXTIMELEVEL;
    return HAMR_OK;
}

int hamr_shim_read(int n) {
    const int rc = hamr_download(shim_ctx[nl[n]], shim_p[nl[n]], shim_ps[nl[n]]);
    if (!rc) shim_unpack(n);
    return rc;
}

void hamr_shim_detach(int n) {
    hamr_ctx_destroy(shim_ctx[nl[n]]);
    free(shim_p[nl[n]]);
    free(shim_ps[nl[n]]);
    shim_ctx[nl[n]] = NULL;
    shim_p[nl[n]] = shim_ps[nl[n]] = NULL;
}
