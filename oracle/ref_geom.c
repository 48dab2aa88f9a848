/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Host harness around the reference's own metric.c / coord.c / lu.c: fills the
 * metric tables of one uniform block the way set_grid (main.c:380-455) does,
 * and packs them in the device layout of GPU_write_metric (GPU_main.cu:139-300):
 *   gcov/gcon : 10 symmetric components x 5 grid locations planes of gsize
 *   gdet      : 5 planes
 *   conn      : 10 symmetric (lower) pairs x 4 (upper index) planes, CENT only
 * Tests compare the product's host geometry builder with these tables.
 */
#include "include.h"
#include "decs.h"

/* Globals that coord.c / metric.c / lu.c read (declared in decs.h:94-97,
 * 825-929). One block, n = 0, at refinement level 0. */
double (*restrict conn[NB_LOCAL])[NDIM][NDIM][NDIM];
double (*restrict gcon[NB_LOCAL])[NPG][NDIM][NDIM];
double (*restrict gcov[NB_LOCAL])[NPG][NDIM][NDIM];
double (*restrict gdet[NB_LOCAL])[NPG];
double (*restrict Mud[NB_LOCAL])[NDIM][NDIM][NDIM];
double (*restrict Mud_inv[NB_LOCAL])[NDIM][NDIM][NDIM];
double a, gam;
double Rin, Rout, R0, fractheta, x1br, rbr, npow2, cpow2, x1max;
double cour;
double dV, dx[NB_LOCAL][NPR], startx[NPR];
double dt, bdt[NB_LOCAL][4];
int failed, lim;
static int ref_block_storage[1][NV];
int (*block)[NV] = ref_block_storage;
int n_ord[NB_LOCAL], nl[NB], n_old[NB], n_ord_total[NB], n_ord_RM[NB_LOCAL], n_ord_total_RM[NB];
int N1_GPU_offset[NB], N2_GPU_offset[NB], N3_GPU_offset[NB];

static int ref_geom_failures;
void fail(int fail_type) { (void)fail_type; ref_geom_failures++; }

int index_2D(int n, int i, int j, int z) {
    (void)z;
    return ((i - N1_GPU_offset[n]) + N1G) * (BS_2 + 2 * N2G) + ((j - N2_GPU_offset[n]) + N2G);
}

static const int RG1 = BS_1 + 2 * N1G, RG2 = BS_2 + 2 * N2G;
static long ref_gsize(void) {
    long n = (long)RG1 * RG2;
    return n + (LOCAL_WORK_SIZE - n % LOCAL_WORK_SIZE);
}

/* Symmetric component order of the device tables (GPU_metric.h:36-90). */
static const int SYM_I[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
static const int SYM_J[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};

static void put_metric(double *gcov_out, double *gcon_out, double *gdet_out, long gsize, long idx,
                       int loc, double gc[NDIM][NDIM], double gn[NDIM][NDIM], double g) {
    for (int s = 0; s < 10; s++) {
        gcov_out[(long)(s * NPG + loc) * gsize + idx] = gc[SYM_I[s]][SYM_J[s]];
        gcon_out[(long)(s * NPG + loc) * gsize + idx] = gn[SYM_I[s]][SYM_J[s]];
    }
    gdet_out[(long)loc * gsize + idx] = g;
}

/*
 * spin a, coordinate origin startx[1..3] and spacing dx[1..3] as set by
 * set_gridparam / set_points (coord.c:327-461). Returns the number of fail()
 * calls the reference made (0 when every table entry is regular).
 */
int ref_geometry(double spin, const double *sx, const double *dxs,
                 double *gcov_out, double *gcon_out, double *gdet_out, double *conn_out) {
    long gsize = ref_gsize();
    a = spin;
    nl[0] = 0;
    for (int k = 0; k < NV; k++) block[0][k] = 0;
    N1_GPU_offset[0] = N2_GPU_offset[0] = N3_GPU_offset[0] = 0;
    for (int d = 1; d < 4; d++) { startx[d] = sx[d]; dx[0][d] = dxs[d]; }
    ref_geom_failures = 0;
    for (int i = -N1G; i < BS_1 + N1G; i++) {
        for (int j = -N2G; j < BS_2 + N2G; j++) {
            long idx = (long)(i + N1G) * RG2 + (j + N2G);
            double X[NDIM], gc[NDIM][NDIM], gn[NDIM][NDIM], g;
            struct of_geom geom;
            double cn[NDIM][NDIM][NDIM];
            X[0] = 0.;
            /* zone centre + connection */
            coord(0, i, j, 0, CENT, X);
            gcov_func(X, gc);
            g = gdet_func(gc);
            gcon_func(gc, gn);
            put_metric(gcov_out, gcon_out, gdet_out, gsize, idx, CENT, gc, gn, g);
            for (int r = 0; r < NDIM; r++)
                for (int c = 0; c < NDIM; c++) { geom.gcov[r][c] = gc[r][c]; geom.gcon[r][c] = gn[r][c]; }
            geom.g = g;
            conn_func(X, &geom, cn);
            for (int s = 0; s < 10; s++)
                for (int l = 0; l < NDIM; l++)
                    conn_out[(long)(s * NDIM + l) * gsize + idx] = cn[l][SYM_I[s]][SYM_J[s]];
            /* r-face, phi-face, theta-face */
            coord(0, i, j, 0, FACE1, X);
            gcov_func(X, gc); g = gdet_func(gc); gcon_func(gc, gn);
            put_metric(gcov_out, gcon_out, gdet_out, gsize, idx, FACE1, gc, gn, g);
            coord(0, i, j, 0, FACE3, X);
            gcov_func(X, gc); g = gdet_func(gc); gcon_func(gc, gn);
            put_metric(gcov_out, gcon_out, gdet_out, gsize, idx, FACE3, gc, gn, g);
            coord(0, i, j, 0, FACE2, X);
            gcov_func(X, gc); g = gdet_func(gc); gcon_func(gc, gn);
            put_metric(gcov_out, gcon_out, gdet_out, gsize, idx, FACE2, gc, gn, g);
        }
    }
    return ref_geom_failures;
}

/* bl_coord (coord.c:111): code coordinates -> (r, theta, phi) */
void ref_bl_coord(const double *X, double *rthph) {
    double Xc[NDIM] = {X[0], X[1], X[2], X[3]};
    bl_coord(Xc, &rthph[0], &rthph[1], &rthph[2]);
}
