/*
 * Test infrastructure (oracle) -- never product code.
 *
 * CPU restatement of H-AMR's single-block RK2 sub-step (the `advance_GPU`
 * pipeline, step_ch.c:997-1335) in plain C99 with runtime grid sizes. Only the
 * tests, the smoke check and the bench's CPU-baseline leg call it; the CUDA
 * product never links it.
 *
 * Layout (identical to the reference device layout and to the product):
 *   cell arrays   plane k of ksize doubles, cell (i, j, z) at (i*G2 + j)*G3 + z,
 *                 G1 = n1 + 2*ng, G2 = n2 + 2*ng, G3 = n3 + 2*ng (G3 = 1, no
 *                 ghosts, when n3 == 1)           GPU_program1.cu:90-94
 *   face B (ps)   3 planes, plane d-1 holds B^d on the lower d-face
 *   metric        gcov/gcon: plane (s*5 + loc), gdet: plane loc, conn: plane
 *                 (s*4 + l), all indexed (i*G2 + j)   GPU_main.cu:139-300
 */
#ifndef HAMR_ORACLE_H
#define HAMR_ORACLE_H

#define HO_NPR 9

enum { HO_BC_PERIODIC = 0, HO_BC_OUTFLOW = 1, HO_BC_POLE_TRANS = 2, HO_BC_POLE_REFL = 3 };

typedef struct {
    int n1, n2, n3;      /* active cells */
    int ng;              /* ghost layers (3 for PPM) */
    long ksize, gsize;   /* plane strides: cell arrays, metric tables */
    double dx1, dx2, dx3;
    double gam;          /* adiabatic index */
    double cour;         /* Courant factor */
    int pole1, pole2;    /* lower/upper x2 edge is a polar axis (GPU_main.cu:566) */
    int bc1, bc2, bc3;   /* HO_BC_* per direction */
    int inversion;       /* 0: Noble 2D (default); 1: Newman-Hamlin */
    int ct_upwind;       /* 1: upwinded edge-EMF corrections; 0: plain average of
                            the four face EMFs (the reference's CARTESIAN build,
                            GPU_const_trans.h:187-211) */
    int recon;           /* 0: PPM (para, PPM builds); 1: MC-limited linear
                            (slope_lim with factor 2, PPM = 0 builds) */
    int riemann;         /* 0: HLL; 1: HLLC in the orthonormal face frame
                            (HLLC builds, FRAME_TRANSFORM); 2: HLLD there, with
                            its HLLC and HLL fallbacks (HLLD builds) */
    int halo;            /* sides interior to a decomposed domain, whose ghosts
                            come from a neighbouring block: bit 0 the lower x1
                            side, bit 1 the upper, bits 2, 3 the lower and upper
                            x2 sides (no pole there: pole1/pole2 0); no physical
                            fill and no radial mass-flux fix there (the
                            reference fills them by its block exchange,
                            boundcomP.c) */
    int floors;          /* 1: drift-frame floors after the inversion (fixup_cell,
                            GPU_fixup.h:1025-1800, compiled out in the reference) */
    int repair;          /* zones whose inversion failed (pflag != 0):
                            1 reset to the floor state (fixuputoprim, GPU_fixup.h:735-852);
                            2 interpolated from good neighbours (fixup_utoprim,
                            fixup.c:764-827); 0 left as the solver left them */
} ho_grid;

typedef struct {
    const double *gcov, *gcon, *gdet, *conn;
} ho_geom;

typedef struct {
    double *p, *ph, *ps, *psh;   /* primitives and face B at t^n / half step */
    double *U;                   /* conserved U(p^n), NPR planes (storage2) */
    double *F1, *F2, *F3;        /* face fluxes, NPR planes each */
    double *E_cent, *emf;        /* 4 planes each (index 1..3 used) */
    int *pflag, *failimage;      /* failimage: 5 planes of ksize ints */
} ho_state;

/* One sub-step: full == 0 advances (p, ps) by Dt into (ph, psh), caching U(p);
 * full == 1 advances the cached U by Dt with fluxes of (ph, psh) into (p, ps).
 * dt is the step's dt (pole EMF averaging scales by it). With calc_dt != 0 the
 * directional CFL limits are returned in dtdir[1..3]. */
void ho_stage(const ho_grid *g, const ho_geom *m, ho_state *s, int full,
              double Dt, double dt, int calc_dt, double *dtdir);

/* Ghost fill of (pv, ps) for the boundary types in g (direction 1, then 3, then 2). */
void ho_bound(const ho_grid *g, const ho_geom *m, double *pv, double *ps);
/* Ghost fill of one direction (1, 2 or 3) on the physical sides; ho_bound is
 * x1, x3, x2 in that order. A domain decomposed along x1 exchanges the x1
 * halos between the x1 and x3 fills; one decomposed along x2 exchanges the x2
 * halos after the x2 fill. */
void ho_bound_dim(const ho_grid *g, const ho_geom *m, double *pv, double *ps, int dim);

/* Single-cell pieces (pinned one by one against the reference). */
void ho_para(const double *x, double *l, double *r);
double ho_slope_lim(double y1, double y2, double y3);
void ho_set_mud(const double *gcov10, const double *gcon10, int dir, double Mud[4][4], double Mi[4][4]);
void ho_primtoflux(double gam, const double *pr, const double *gcov10, const double *gcon10,
                   double gdet, int dir, double *flux, double *vmax, double *vmin);
int ho_utoprim_2d(double gam, double *U, const double *gcov10, const double *gcon10, double gdet, double *prim);
int ho_utoprim_1dvsq2fix1(double gam, double *U, const double *gcov10, const double *gcon10, double gdet, double *prim);
int ho_utoprim_1dfix1(double gam, double *U, const double *gcov10, const double *gcon10, double gdet, double *prim);
int ho_utoprim_nm(double gam, double *U, const double *gcov10, const double *gcon10, double gdet, double *prim);
int ho_utoprim_nm_max_index(void);

/* Floors of one zone (centre metric); returns 4 when the Lorentz factor
 * cannot be formed, else 0. */
int ho_fixup_cell(double gam, double *pf, const double *gcov10, const double *gcon10, double gdet);
/* Neighbour repair of the failed active zones of pv in (i, j, z) order,
 * clearing their flags (fixup_utoprim, fixup.c:764-827). */
void ho_fixup_utoprim(const ho_grid *g, double *pv, int *pflag, int *failimage);

/* Diagnostics */
double ho_divb_max(const ho_grid *g, const ho_geom *m, const double *ps);

/* host metric tables of one block (hamr_oracle_geom.c; set_grid, main.c:380-455):
 * coords 0 Kerr-Schild in the reference's code coordinates, 1 Minkowski;
 * 0, -1 bad argument, -5 a singular metric */
int ho_build_geometry(int coords, double spin, int n1, int n2, int n3, int ng, long gsize, const double *startx,
                      const double *dx, double *gcov, double *gcon, double *gdet, double *conn);
/* Boyer-Lindquist (r, theta, phi) of a code-coordinate point (bl_coord, coord.c:111) */
int ho_bl_coord(int coords, double spin, const double *X, double *rthph);
/* OpenMP threads a parallel loop of the oracle uses (1 without OpenMP) */
int ho_num_threads(void);
/* bit-level check of the library's division by a reciprocal (div_rcp) */
long ho_div_rcp_mismatches(const double *a, long n, const double *b, long m);
long ho_div_rcp_mismatches_g(const double *a, long n, const double *b, long m, int guard);

#endif
