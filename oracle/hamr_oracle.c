/*
 * Test infrastructure (oracle) -- never product code.
 *
 * CPU restatement of the reference's single-block RK2 sub-step. Each routine
 * cites the reference routine it follows; expressions keep the reference's
 * operand order so that, with -ffp-contract=off, results agree with the host
 * build of the reference kernels bit for bit (tests/test_oracle_pin.py).
 * Runtime sizes replace the reference's compile-time BS_* / N*G, and the
 * adiabatic index is a runtime value instead of the GAMMA macro.
 */
#include "hamr_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4, B1 = 5, B2 = 6, B3 = 7, KTOT = 8 };
enum { FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3, FACE3 = 4 };
#define NPR HO_NPR
#define SMALL 1.e-20
#define NEWT_TOL 1.0e-10
#define MIN_NEWT_TOL 1.0e-10
#define MAX_NEWT_ITER 30
#define EXTRA_NEWT_ITER 2
#define W_TOO_BIG 1.e20
#define UTSQ_TOO_BIG 1.e20
#define FAIL_VAL 1.e30
#define GAMMAMAX 80.
#define MY_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define MY_MAX(a, b) (((a) > (b)) ? (a) : (b))

typedef struct { double gcov[10], gcon[10], g; } geo;
typedef struct { double ucon[4], ucov[4], bcon[4], bcov[4]; } cstate;

/* ------------------------------------------------------------------ grid -- */
typedef struct {
    int n1, n2, n3, ng1, ng2, ng3, G1, G2, G3;
    int d1, d2, d3;
    long ks, gs;
} dims;

static dims mkdims(const ho_grid *g) {
    dims d;
    d.n1 = g->n1; d.n2 = g->n2; d.n3 = g->n3;
    d.d1 = g->n1 > 1; d.d2 = g->n2 > 1; d.d3 = g->n3 > 1;
    d.ng1 = d.d1 ? g->ng : 0; d.ng2 = d.d2 ? g->ng : 0; d.ng3 = d.d3 ? g->ng : 0;
    d.G1 = g->n1 + 2 * d.ng1; d.G2 = g->n2 + 2 * d.ng2; d.G3 = g->n3 + 2 * d.ng3;
    d.ks = g->ksize; d.gs = g->gsize;
    return d;
}
static inline long cix(const dims *d, int i, int j, int z) { return ((long)i * d->G2 + j) * d->G3 + z; }
static inline long gix(const dims *d, int i, int j) { return (long)i * d->G2 + j; }

/* get_geometry (GPU_metric.h:36-90) */
static void load_geo(const dims *d, const ho_geom *m, int i, int j, int loc, geo *o) {
    long idx = gix(d, i, j);
    for (int s = 0; s < 10; s++) {
        o->gcon[s] = m->gcon[(long)(s * 5 + loc) * d->gs + idx];
        o->gcov[s] = m->gcov[(long)(s * 5 + loc) * d->gs + idx];
    }
    o->g = m->gdet[(long)loc * d->gs + idx];
}

/* ------------------------------------------------------- metric algebra -- */
/* lower / raise (GPU_metric.h:3-34) */
static void lower4(const double *ucon, const double *gcov, double *ucov) {
    ucov[0] = gcov[0] * ucon[0] + gcov[1] * ucon[1] + gcov[2] * ucon[2] + gcov[3] * ucon[3];
    ucov[1] = gcov[1] * ucon[0] + gcov[4] * ucon[1] + gcov[5] * ucon[2] + gcov[6] * ucon[3];
    ucov[2] = gcov[2] * ucon[0] + gcov[5] * ucon[1] + gcov[7] * ucon[2] + gcov[8] * ucon[3];
    ucov[3] = gcov[3] * ucon[0] + gcov[6] * ucon[1] + gcov[8] * ucon[2] + gcov[9] * ucon[3];
}
static void raise4(const double *ucov, const double *gcon, double *ucon) {
    ucon[0] = gcon[0] * ucov[0] + gcon[1] * ucov[1] + gcon[2] * ucov[2] + gcon[3] * ucov[3];
    ucon[1] = gcon[1] * ucov[0] + gcon[4] * ucov[1] + gcon[5] * ucov[2] + gcon[6] * ucov[3];
    ucon[2] = gcon[2] * ucov[0] + gcon[5] * ucov[1] + gcon[7] * ucov[2] + gcon[8] * ucov[3];
    ucon[3] = gcon[3] * ucov[0] + gcon[6] * ucov[1] + gcon[8] * ucov[2] + gcon[9] * ucov[3];
}
static inline double dot4(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* gamma_calc (GPU_phys_mhd.h:740-761): Lorentz factor w.r.t. the normal observer */
static int gamma_calc(const double *pr, const geo *gm, double *gamma) {
    const double *g = gm->gcov;
    double qsq = g[4] * pr[U1] * pr[U1] + g[7] * pr[U2] * pr[U2] + g[9] * pr[U3] * pr[U3]
               + 2. * (g[5] * pr[U1] * pr[U2] + g[6] * pr[U1] * pr[U3] + g[8] * pr[U2] * pr[U3]);
    if (qsq < 0.) {
        if (fabs(qsq) > 1.E-10) { *gamma = 1.; return 1; }
        qsq = 1.E-10;
    }
    *gamma = sqrt(1. + qsq);
    return 0;
}

/* ucon_calc (GPU_phys_mhd.h:694-717) */
static void ucon_calc(const double *pr, const geo *gm, double *ucon) {
    double alpha = 1. / sqrt(-gm->gcon[0]);
    double beta[4], gamma;
    for (int j = 1; j < 4; j++) beta[j] = gm->gcon[j] * alpha * alpha;
    gamma_calc(pr, gm, &gamma);
    ucon[0] = gamma / alpha;
    for (int j = 1; j < 4; j++) ucon[j] = pr[U1 + j - 1] - gamma * beta[j] / alpha;
}

/* bcon_calc (GPU_phys_mhd.h:719-732) */
static void bcon_calc(const double *pr, const double *ucon, const double *ucov, double *bcon) {
    bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
    for (int j = 1; j < 4; j++) bcon[j] = (pr[B1 - 1 + j] + bcon[0] * ucon[j]) / ucon[0];
}

/* get_state (GPU_phys_mhd.h:672-690) */
static void get_state(const double *pr, const geo *gm, cstate *q) {
    ucon_calc(pr, gm, q->ucon);
    lower4(q->ucon, gm->gcov, q->ucov);
    bcon_calc(pr, q->ucon, q->ucov, q->bcon);
    lower4(q->bcon, gm->gcov, q->bcov);
}

/* calc_entropy (GPU_phys_mhd.h:631-670), ideal gas, K = P rho^-gamma */
static inline double calc_entropy(double gam, const double *pr) {
    double P = (gam - 1.0) * pr[UU];
    return P * pow(pr[RHO], -gam);
}

/* primtoflux with fast magnetosonic speeds (GPU_phys_mhd.h:432-628) */
static void primtoflux(double gam, const double *pr, const cstate *q, int dir, const geo *gm,
                       double *flux, double *vmax, double *vmin) {
    double mhd[4];
    double u = pr[UU];
    double P = (gam - 1.) * u;
    double w = pr[RHO] + P + u;
    double bsq = dot4(q->bcon, q->bcov);
    double eta = w + bsq;
    double ptot = P + 0.5 * bsq;
    flux[RHO] = pr[RHO] * q->ucon[dir];
    for (int j = 0; j < 4; j++)
        mhd[j] = eta * q->ucon[dir] * q->ucov[j] + ptot * (dir == j ? 1. : 0.) - q->bcon[dir] * q->bcov[j];
    flux[UU] = mhd[0] + flux[RHO];
    flux[U1] = mhd[1];
    flux[U2] = mhd[2];
    flux[U3] = mhd[3];
    flux[B1] = q->bcon[1] * q->ucon[dir] - q->bcon[dir] * q->ucon[1];
    flux[B2] = q->bcon[2] * q->ucon[dir] - q->bcon[dir] * q->ucon[2];
    flux[B3] = q->bcon[3] * q->ucon[dir] - q->bcon[dir] * q->ucon[3];
    flux[KTOT] = flux[RHO] * calc_entropy(gam, pr);
    for (int k = 0; k < NPR; k++) flux[k] *= gm->g;
    if (dir != 0) {
        double Acon_0, Acon_js;
        if (dir == 1) { Acon_0 = gm->gcon[1]; Acon_js = gm->gcon[4]; }
        else if (dir == 2) { Acon_0 = gm->gcon[2]; Acon_js = gm->gcon[7]; }
        else { Acon_0 = gm->gcon[3]; Acon_js = gm->gcon[9]; }
        double cs2 = gam * (gam - 1.) * pr[UU] / w;
        double va2 = bsq / eta;
        double cms2 = cs2 + va2 - cs2 * va2;
        if (cms2 < 0.) cms2 = SMALL;
        if (cms2 > 1.) cms2 = 1.;
        double Asq = Acon_js, Bsq = gm->gcon[0];
        double Au = q->ucon[dir], Bu = q->ucon[0], AB = Acon_0;
        double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
        double A = Bu2 - (Bsq + Bu2) * cms2;
        double B = 2. * (AuBu - (AB + AuBu) * cms2);
        double C = Au2 - (Asq + Au2) * cms2;
        double discr = B * B - 4. * A * C;
        if ((discr < 0.0) && (discr > -1.e-10)) discr = 0.0;
        else if (discr < -1.e-10) discr = 0.;
        discr = sqrt(discr);
        double vp = -(-B + discr) / (2. * A);
        double vm = -(-B - discr) / (2. * A);
        *vmax = MY_MAX(vp, vm);
        *vmin = MY_MIN(vp, vm);
    }
}

/* ------------------------------------------------------- reconstruction -- */
/* para: Colella-Woodward PPM with MC-2 slopes and monotonicity clamps
 * (GPU_interp.h:60-111) */
void ho_para(const double *x, double *lout, double *rout) {
    double y[5], dq[5];
    for (int i = 0; i < 5; i++) y[i] = x[i];
    dq[0] = dq[4] = 0.;
    for (int i = 1; i < 4; i++) {
        double Dqm = 2. * (y[i] - y[i - 1]);
        double Dqp = 2. * (y[i + 1] - y[i]);
        double Dqc = 0.5 * (y[i + 1] - y[i - 1]);
        double aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
        double s = Dqm * Dqp;
        Dqm = MY_MIN(aDqm, aDqp);
        if (aDqc < Dqm) {
            if (Dqc > 0.) dq[i] = (aDqc) * (double)(s > 0.);
            else dq[i] = (-aDqc) * (double)(s > 0.);
        } else {
            if (Dqc > 0.) dq[i] = (Dqm) * (double)(s > 0.);
            else dq[i] = (-Dqm) * (double)(s > 0.);
        }
    }
    double l = 0.5 * (y[2] + y[1]) - (dq[2] - dq[1]) / 6.0;
    double r = 0.5 * (y[3] + y[2]) - (dq[3] - dq[2]) / 6.0;
    double qa = (r - y[2]) * (y[2] - l);
    double qd = (r - l);
    double qe = 6.0 * (y[2] - 0.5 * (l + r));
    if (qa <= 0.) { l = y[2]; r = y[2]; }
    if (qd * (qd - qe) < 0.0) l = 3.0 * y[2] - 2.0 * r;
    else if (qd * (qd + qe) < 0.0) r = 3.0 * y[2] - 2.0 * l;
    *lout = l;
    *rout = r;
}

/* slope_lim: monotonized-central slope with the GPU's steepening factor 2
 * (GPU_interp.h:2-38, the non-NEUTRON_STAR branch); the zone's face values
 * are y -+ slope/2 (fluxcalcprep with PPM = 0, GPU_program1.cu:178-186) */
double ho_slope_lim(double y1, double y2, double y3) {
    double Dqm = (2.0) * (y2 - y1);
    double Dqp = (2.0) * (y3 - y2);
    double Dqc = 0.5 * (y3 - y1);
    double s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    if (fabs(Dqm) < fabs(Dqp) && fabs(Dqm) < fabs(Dqc)) return Dqm;
    if (fabs(Dqp) < fabs(Dqc)) return Dqp;
    return Dqc;
}

void ho_primtoflux(double gam, const double *pr, const double *gcov10, const double *gcon10,
                   double gdet, int dir, double *flux, double *vmax, double *vmin) {
    geo gm;
    cstate q;
    memcpy(gm.gcov, gcov10, sizeof(gm.gcov));
    memcpy(gm.gcon, gcon10, sizeof(gm.gcon));
    gm.g = gdet;
    get_state(pr, &gm, &q);
    primtoflux(gam, pr, &q, dir, &gm, flux, vmax, vmin);
}

/* ----------------------------------------------------------------- HLLC -- */
static int sym(int a, int b) {
    static const int t[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
    return t[a][b];
}

/* Orthonormal frame of a face of direction dir (set_Mud, hllc.c:20-164):
 * Mud[a][b] and its inverse Mi, from the face metric. With (d, e, f) the
 * cyclic order starting at dir, every entry follows the reference's
 * expression for that direction. */
void ho_set_mud(const double *gcov10, const double *gcon10, int dir, double Mud[4][4], double Mi[4][4]) {
    const int d = dir, e = dir % 3 + 1, f = (dir + 1) % 3 + 1;
#define GU(a, b) gcon10[sym(a, b)]
#define GD(a, b) gcov10[sym(a, b)]
    double A = -pow(-GU(0, 0), -0.5);
    double B = pow((GU(0, 0)) * (GU(0, 0) * GU(d, d) - GU(0, d) * GU(0, d)), -0.5);
    double C = pow(GD(f, f), -0.5);
    double D = pow((GD(f, f)) * (GD(e, e) * GD(f, f) - GD(e, f) * GD(e, f)), -0.5);
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) Mud[a][b] = Mi[a][b] = 0.;
    Mud[0][0] = A * GU(0, 0);
    Mud[d][0] = A * GU(0, d);
    Mud[d][d] = B * (GU(0, d) * GU(0, d) - GU(0, 0) * GU(d, d));
    Mud[e][0] = A * GU(0, e);
    Mud[e][d] = B * (GU(0, d) * GU(0, e) - GU(0, 0) * GU(d, e));
    Mud[e][e] = D * GD(f, f);
    Mud[f][0] = A * GU(0, f);
    Mud[f][d] = B * (GU(0, d) * GU(0, f) - GU(0, 0) * GU(d, f));
    Mud[f][e] = -D * GD(e, f);
    Mud[f][f] = C;
    double E = GU(0, d) * GU(d, e) - GU(d, d) * GU(0, e);
    double F = GU(0, d) * GU(0, e) - GU(0, 0) * GU(d, e);
    double G = GU(0, d) * GU(d, f) - GU(d, d) * GU(0, f);
    double H = GU(0, d) * GU(0, f) - GU(0, 0) * GU(d, f);
    Mi[0][0] = -A;
    Mi[d][0] = B * GU(0, d);
    Mi[d][d] = -B * GU(0, 0);
    Mi[e][0] = B * B * E * GU(0, 0) / (D * GD(f, f));
    Mi[e][d] = B * B * F * GU(0, 0) / (D * GD(f, f));
    Mi[e][e] = 1. / (D * GD(f, f));
    Mi[f][0] = (B * B / C) * GU(0, 0) * (G + E * GD(e, f) / GD(f, f));
    Mi[f][d] = (B * B / C) * GU(0, 0) * (H + F * GD(e, f) / GD(f, f));
    Mi[f][e] = (1. / C) * GD(e, f) / GD(f, f);
    Mi[f][f] = 1. / C;
#undef GU
#undef GD
}

/* fluxes in the orthonormal frame (primtoflux_FT, GPU_hllc.h:903-1010) */
static void primtoflux_ft(double gam, const double *pr, const double *ucon, const double *bcon, int dir,
                          double *flux) {
    flux[RHO] = pr[RHO] * ucon[dir];
    double P = (gam - 1.) * pr[UU];
    double w = P + pr[RHO] + pr[UU];
    double bsq = -bcon[0] * bcon[0] + bcon[1] * bcon[1] + bcon[2] * bcon[2] + bcon[3] * bcon[3];
    double eta = w + bsq;
    double ptot = P + 0.5 * bsq;
    flux[UU] = -eta * ucon[dir] * ucon[0] + ptot * (double)(dir == 0) + bcon[dir] * bcon[0];
    for (int j = 1; j < 4; j++) flux[UU + j] = eta * ucon[dir] * ucon[j] + ptot * (double)(dir == j) - bcon[dir] * bcon[j];
    for (int k = B1; k <= B3; k++) flux[k] = bcon[k - 4] * ucon[dir] - bcon[dir] * ucon[k - 4];
    flux[KTOT] = flux[RHO] * P * pow(pr[RHO], -gam);
}

/* fast speeds in the orthonormal frame (vchar_FT, GPU_hllc.h:1012-1111) */
static void vchar_ft(double gam, const double *pr, const double *ucon, const double *bcon, int dir, double *vmax,
                     double *vmin) {
    double bsq = -bcon[0] * bcon[0] + bcon[1] * bcon[1] + bcon[2] * bcon[2] + bcon[3] * bcon[3];
    double EF = pr[RHO] + gam * pr[UU];
    double cs2 = gam * (gam - 1.) * pr[UU] / EF;
    double EE = bsq + EF;
    double va2 = bsq / EE;
    double cms2 = cs2 + va2 - cs2 * va2;
    if (cms2 < 0.) cms2 = SMALL;
    if (cms2 > 1.) cms2 = 1.;
    double Asq = 1., Bsq = -1.;
    double Au = ucon[dir], Bu = ucon[0];
    double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
    double A = Bu2 - (Bsq + Bu2) * cms2;
    double B = 2. * (AuBu - (AuBu) * cms2);
    double C = Au2 - (Asq + Au2) * cms2;
    double discr = B * B - 4. * A * C;
    if ((discr < 0.0) && (discr > -1.e-10)) discr = 0.0;
    else if (discr < -1.e-10) discr = 0.;
    discr = sqrt(discr);
    double vp = -(-B + discr) / (2. * A);
    double vm = -(-B - discr) / (2. * A);
    if (vp > vm) { *vmax = vp; *vmin = vm; }
    else { *vmax = vm; *vmin = vp; }
}

/* HLLC star states, hydrodynamic case (calc_HLLC_hydro, GPU_hllc.h:250-315) */
static void hllc_hydro(int dir, const double *lu, const double *ru, double iv, double cmin, double cmax,
                       double FT[2][NPR], double FH[2][NPR], const double *Fl, const double *Fr, const double *Ul,
                       const double *Ur) {
    const int U_1 = UU + dir, U_2 = UU + dir % 3 + 1, U_3 = UU + (dir + 1) % 3 + 1;
    const int B_1 = B1 + dir - 1, B_2 = B1 + dir % 3, B_3 = B1 + (dir + 1) % 3;
    int fail = 0;
    double A = -FH[1][UU];
    double B = -FH[1][U_1] + FH[0][UU];
    double C = FH[0][U_1];
    double D = B * B - 4. * A * C;
    double vcon = (-B - sqrt(D)) / (2. * A);
    double ptot = -(-FH[1][UU]) * vcon + FH[1][U_1];
    if (!(fabs(ptot) > 0.) || (vcon < cmin) || (vcon > cmax) || !(fabs(vcon) > 0.)) fail = 1;
    if (cmax > iv && vcon <= iv && fail == 0) {
        double s = (cmax - ru[dir] / ru[0]) / (cmax - vcon + SMALL);
        FT[0][RHO] = s * Ur[RHO];
        FT[0][UU] = (cmax * Ur[UU] + Ur[U_1] - ptot * vcon) / (cmax - vcon + SMALL);
        FT[0][U_1] = (-FT[0][UU] + ptot) * vcon;
        FT[0][U_2] = s * Ur[U_2];
        FT[0][U_3] = s * Ur[U_3];
        FT[0][B_1] = FH[0][B_1];
        FT[0][B_2] = s * Ur[B_2];
        FT[0][B_3] = s * Ur[B_3];
        FT[0][KTOT] = s * Ur[KTOT];
        for (int k = 0; k < NPR; k++) FT[1][k] = (Fr[k] + cmax * (FT[0][k] - Ur[k]));
    } else if (cmin < iv && vcon >= iv && fail == 0) {
        double s = (cmin - lu[dir] / lu[0]) / (cmin - vcon + SMALL);
        FT[0][RHO] = s * Ul[RHO];
        FT[0][UU] = (cmin * Ul[UU] + Ul[U_1] - ptot * vcon) / (cmin - vcon + SMALL);
        FT[0][U_1] = (-FT[0][UU] + ptot) * vcon;
        FT[0][U_2] = s * Ul[U_2];
        FT[0][U_3] = s * Ul[U_3];
        FT[0][B_1] = FH[0][B_1];
        FT[0][B_2] = s * Ul[B_2];
        FT[0][B_3] = s * Ul[B_3];
        FT[0][KTOT] = s * Ul[KTOT];
        for (int k = 0; k < NPR; k++) FT[1][k] = (Fl[k] + cmin * (FT[0][k] - Ul[k]));
    } else {
        for (int k = 0; k < NPR; k++) { FT[0][k] = FH[0][k]; FT[1][k] = FH[1][k]; }
    }
}

/* HLLC star states, magnetised case (calc_HLLC, GPU_hllc.h:317-396) */
static void hllc_mhd(int dir, const double *lu, const double *ru, double iv, double cmin, double cmax,
                     double FT[2][NPR], double FH[2][NPR], const double *Fl, const double *Fr, const double *Ul,
                     const double *Ur) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    const int U_1 = UU + G_1, U_2 = UU + G_2, U_3 = UU + G_3;
    const int B_1 = B1 + G_1 - 1, B_2 = B1 + G_2 - 1, B_3 = B1 + G_3 - 1;
    double vcon[4];
    int fail = 0;
    double A = -FH[1][UU] - (FH[0][B_2] * FH[1][B_2] + FH[0][B_3] * FH[1][B_3]);
    double B = -FH[1][U_1] + FH[0][UU] + (FH[0][B_2] * FH[0][B_2] + FH[0][B_3] * FH[0][B_3]) +
               (FH[1][B_2] * FH[1][B_2] + FH[1][B_3] * FH[1][B_3]);
    double C = FH[0][U_1] - (FH[0][B_2] * FH[1][B_2] + FH[0][B_3] * FH[1][B_3]);
    double D = B * B - 4. * A * C;
    vcon[G_1] = (-B - sqrt(D)) / (2. * A);
    vcon[G_2] = (FH[0][B_2] * vcon[G_1] - FH[1][B_2]) / FH[0][B_1];
    vcon[G_3] = (FH[0][B_3] * vcon[G_1] - FH[1][B_3]) / FH[0][B_1];
    double gammasq = 1. / (1. - (vcon[1] * vcon[1] + vcon[2] * vcon[2] + vcon[3] * vcon[3]));
    double vB = (vcon[1] * FH[0][B1] + vcon[2] * FH[0][B2] + vcon[3] * FH[0][B3]);
    double ptot = -(-FH[1][UU] - FH[0][B_1] * (vB)) * vcon[dir] + FH[1][U_1] + pow(FH[0][B_1], 2.0) / gammasq;
    if (!(fabs(ptot) > 0.) || (vcon[G_1] < cmin) || (vcon[G_1] > cmax) || !(fabs(vcon[G_1]) > 0.)) fail = 1;
    if (cmax > iv && vcon[dir] <= iv && fail == 0) {
        FT[0][RHO] = (cmax - ru[dir] / ru[0]) / (cmax - vcon[dir] + SMALL) * Ur[RHO];
        FT[0][UU] = (cmax * Ur[UU] + Ur[U_1] - ptot * vcon[dir] + vB * FH[0][B_1]) / (cmax - vcon[dir] + SMALL);
        FT[0][U_1] = (-FT[0][UU] + ptot) * vcon[dir] - vB * FH[0][B_1];
        FT[0][U_2] = (-FH[0][B_1] * (FH[0][B_2] / (gammasq) + vB * vcon[G_2]) + cmax * Ur[U_2] - Fr[U_2]) /
                     (cmax - vcon[dir] + SMALL);
        FT[0][U_3] = (-FH[0][B_1] * (FH[0][B_3] / (gammasq) + vB * vcon[G_3]) + cmax * Ur[U_3] - Fr[U_3]) /
                     (cmax - vcon[dir] + SMALL);
        FT[0][B_1] = FH[0][B_1];
        FT[0][B_2] = FH[0][B_2];
        FT[0][B_3] = FH[0][B_3];
        FT[0][KTOT] = (cmax - ru[dir] / ru[0]) / (cmax - vcon[dir] + SMALL) * Ur[KTOT];
        for (int k = 0; k < NPR; k++) FT[1][k] = (Fr[k] + cmax * (FT[0][k] - Ur[k]));
    } else if (cmin < iv && vcon[dir] >= iv && fail == 0) {
        FT[0][RHO] = (cmin - lu[dir] / lu[0]) / (cmin - vcon[dir] + SMALL) * Ul[RHO];
        FT[0][UU] = (cmin * Ul[UU] + Ul[U_1] - ptot * vcon[dir] + vB * FH[0][B_1]) / (cmin - vcon[dir] + SMALL);
        FT[0][U_1] = (-FT[0][UU] + ptot) * vcon[dir] - vB * FH[0][B_1];
        FT[0][U_2] = (-FH[0][B_1] * (FH[0][B_2] / (gammasq) + vB * vcon[G_2]) + cmin * Ul[U_2] - Fl[U_2]) /
                     (cmin - vcon[dir] + SMALL);
        FT[0][U_3] = (-FH[0][B_1] * (FH[0][B_3] / (gammasq) + vB * vcon[G_3]) + cmin * Ul[U_3] - Fl[U_3]) /
                     (cmin - vcon[dir] + SMALL);
        FT[0][B_1] = FH[0][B_1];
        FT[0][B_2] = FH[0][B_2];
        FT[0][B_3] = FH[0][B_3];
        FT[0][KTOT] = (cmin - lu[dir] / lu[0]) / (cmin - vcon[dir] + SMALL) * Ul[KTOT];
        for (int k = 0; k < NPR; k++) FT[1][k] = (Fl[k] + cmin * (FT[0][k] - Ul[k]));
    } else {
        for (int k = 0; k < NPR; k++) { FT[0][k] = FH[0][k]; FT[1][k] = FH[1][k]; }
    }
}

/* HLLD (calc_HLLD and its helpers, GPU_hllc.h:398-876; HLLD builds, which
 * the reference's config marks "Does not work yet", config.h:482). Written
 * as there, including two slips that decide its results: G sums the second
 * transverse residual instead of squaring it (GPU_hllc.h:808,822) and the
 * right intermediate speed check adds vcon_ar[3] * vcon_al[3]
 * (GPU_hllc.h:673). pow(10, -k) constants are the correctly rounded
 * literals the host compiler folds them to. */
typedef struct {
    double K_al[4], B_al[4], K_ar[4], B_ar[4], v_al[4], v_ar[4], v_cl[4], v_cr[4], B_c[4];
    double eta_l, eta_r, w_al, w_ar;
} hlld_fan;

/* calc_error_HLLD (GPU_hllc.h:685-876, the live second half): the fan for a
 * total pressure guess, returning the Newton residual */
static double hlld_error(int dir, double ptot, double cmin, double cmax, double BX, const double *R_l,
                         const double *R_r, hlld_fan *f) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    const int U_1 = UU + G_1, U_2 = UU + G_2, U_3 = UU + G_3;
    const int B_1 = B1 + G_1 - 1, B_2 = B1 + G_2 - 1, B_3 = B1 + G_3 - 1;
    double A, C, G, X, Q;
    A = R_l[U_1] + cmin * R_l[UU] + ptot * (1. - cmin * cmin);
    G = R_l[B_2] * R_l[B_2] + R_l[B_3] + R_l[B_3];
    C = R_l[U_2] * R_l[B_2] + R_l[U_3] * R_l[B_3];
    Q = -A - G + (BX * BX) * (1. - cmin * cmin);
    X = BX * (A * cmin * BX + C) - (A + G) * (cmin * ptot - R_l[UU]);
    f->v_al[G_1] = (BX * (A * BX + cmin * C) - (A + G) * (ptot + R_l[U_1])) / (X);
    f->v_al[G_2] = (Q * R_l[U_2] + R_l[B_2] * (C + BX * (cmin * R_l[U_1] + R_l[UU]))) / (X);
    f->v_al[G_3] = (Q * R_l[U_3] + R_l[B_3] * (C + BX * (cmin * R_l[U_1] + R_l[UU]))) / (X);
    f->w_al = ptot + (-R_l[UU] - (f->v_al[G_1] * R_l[U_1] + f->v_al[G_2] * R_l[U_2] + f->v_al[G_3] * R_l[U_3])) /
                     (cmin - f->v_al[G_1] + SMALL);
    A = R_r[U_1] + cmax * R_r[UU] + ptot * (1. - cmax * cmax);
    G = R_r[B_2] * R_r[B_2] + R_r[B_3] + R_r[B_3];
    C = R_r[U_2] * R_r[B_2] + R_r[U_3] * R_r[B_3];
    Q = -A - G + (BX * BX) * (1. - cmax * cmax);
    X = BX * (A * cmax * BX + C) - (A + G) * (cmax * ptot - R_r[UU]);
    f->v_ar[G_1] = (BX * (A * BX + cmax * C) - (A + G) * (ptot + R_r[U_1])) / (X);
    f->v_ar[G_2] = (Q * R_r[U_2] + R_r[B_2] * (C + BX * (cmax * R_r[U_1] + R_r[UU]))) / (X);
    f->v_ar[G_3] = (Q * R_r[U_3] + R_r[B_3] * (C + BX * (cmax * R_r[U_1] + R_r[UU]))) / (X);
    f->w_ar = ptot + (-R_r[UU] - (f->v_ar[G_1] * R_r[U_1] + f->v_ar[G_2] * R_r[U_2] + f->v_ar[G_3] * R_r[U_3])) /
                     (cmax - f->v_ar[G_1] + SMALL);
    /* fields of the outer intermediate states (eq. 21) */
    f->B_al[G_1] = BX;
    f->B_al[G_2] = (R_l[B_2] - f->B_al[G_1] * f->v_al[G_2]) / (cmin - f->v_al[G_1]);
    f->B_al[G_3] = (R_l[B_3] - f->B_al[G_1] * f->v_al[G_3]) / (cmin - f->v_al[G_1]);
    f->B_ar[G_1] = BX;
    f->B_ar[G_2] = (R_r[B_2] - f->B_ar[G_1] * f->v_ar[G_2]) / (cmax - f->v_ar[G_1]);
    f->B_ar[G_3] = (R_r[B_3] - f->B_ar[G_1] * f->v_ar[G_3]) / (cmax - f->v_ar[G_1]);
    /* Alfven-wave K vectors (eq. 43) */
    f->eta_l = -((double)(BX > 0.0) - (double)(BX <= 0.0)) * sqrt(fabs(f->w_al));
    double dl = cmin * ptot - R_l[UU] + BX * f->eta_l;
    f->K_al[G_1] = (R_l[U_1] + ptot + R_l[B_1] * f->eta_l) / dl;
    f->K_al[G_2] = (R_l[U_2] + R_l[B_2] * f->eta_l) / dl;
    f->K_al[G_3] = (R_l[U_3] + R_l[B_3] * f->eta_l) / dl;
    f->eta_r = ((double)(BX > 0.0) - (double)(BX <= 0.0)) * sqrt(fabs(f->w_ar));
    double dr = cmax * ptot - R_r[UU] + BX * f->eta_r;
    f->K_ar[G_1] = (R_r[U_1] + ptot + R_r[B_1] * f->eta_r) / dr;
    f->K_ar[G_2] = (R_r[U_2] + R_r[B_2] * f->eta_r) / dr;
    f->K_ar[G_3] = (R_r[U_3] + R_r[B_3] * f->eta_r) / dr;
    /* field between the Alfven waves and the contact (eq. 45) */
    f->B_c[G_1] = BX;
    for (int t = 0; t < 2; t++) {
        const int Gt = t ? G_3 : G_2;
        f->B_c[Gt] = ((f->B_ar[Gt] * (f->K_ar[G_1] - f->v_ar[dir]) + f->B_ar[dir] * f->v_ar[Gt]) -
                      (f->B_al[Gt] * (f->K_al[G_1] - f->v_al[dir]) + f->B_al[dir] * f->v_al[Gt])) /
                     (f->K_ar[dir] - f->K_al[dir] + 1e-12);
    }
    const double delta_Kx = (f->K_ar[dir] - f->K_al[dir]);
    double B_hat[4];
    B_hat[1] = delta_Kx * f->B_c[1];
    B_hat[2] = delta_Kx * f->B_c[2];
    B_hat[3] = delta_Kx * f->B_c[3];
    const double kl2 = f->K_al[1] * f->K_al[1] + f->K_al[2] * f->K_al[2] + f->K_al[3] * f->K_al[3];
    const double kr2 = f->K_ar[1] * f->K_ar[1] + f->K_ar[2] * f->K_ar[2] + f->K_ar[3] * f->K_ar[3];
    double Y_l = (1. - kl2) / (f->eta_l * delta_Kx - (f->K_al[1] * B_hat[1] + f->K_al[2] * B_hat[2] + f->K_al[3] * B_hat[3]));
    double Y_r = (1. - kr2) / (f->eta_r * delta_Kx - (f->K_ar[1] * B_hat[1] + f->K_ar[2] * B_hat[2] + f->K_ar[3] * B_hat[3]));
    double error = delta_Kx * (1. - f->B_ar[dir] * (Y_r - Y_l));
    /* contact state (eqs. 47, 50-52) */
    const double kbl = f->eta_l - (f->K_al[1] * f->B_c[1] + f->K_al[2] * f->B_c[2] + f->K_al[3] * f->B_c[3]);
    const double kbr = f->eta_r - (f->K_ar[1] * f->B_c[1] + f->K_ar[2] * f->B_c[2] + f->K_ar[3] * f->B_c[3]);
    const int Gs[3] = {G_1, G_2, G_3};
    for (int t = 0; t < 3; t++) {
        const int Gt = Gs[t];
        f->v_cl[Gt] = (f->K_al[Gt] - (f->B_c[Gt] * (1. - kl2)) / kbl);
        f->v_cr[Gt] = (f->K_ar[Gt] - (f->B_c[Gt] * (1. - kr2)) / kbr);
    }
    f->v_cl[dir] = (f->v_cl[dir] + f->v_cr[dir]) * 0.5;
    f->v_cr[dir] = f->v_cl[dir];
    return error;
}

/* calc_HLLD_pres (GPU_hllc.h:425-531): HLLC estimate of the total pressure,
 * then up to 12 secant-Newton steps on hlld_error */
static double hlld_pres(int dir, int *fail_c, int *fail_d, double cmin, double cmax, double FH[2][NPR],
                        const double *R_l, const double *R_r, hlld_fan *f) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    const int U_1 = UU + G_1;
    const int B_1 = B1 + G_1 - 1, B_2 = B1 + G_2 - 1, B_3 = B1 + G_3 - 1;
    double vcon[4];
    double A = -FH[1][UU] - (FH[0][B_2] * FH[1][B_2] + FH[0][B_3] * FH[1][B_3]);
    double B = -FH[1][U_1] + FH[0][UU] + (FH[0][B_2] * FH[0][B_2] + FH[0][B_3] * FH[0][B_3]) +
               (FH[1][B_2] * FH[1][B_2] + FH[1][B_3] * FH[1][B_3]);
    double C = FH[0][U_1] - (FH[0][B_2] * FH[1][B_2] + FH[0][B_3] * FH[1][B_3]);
    double D = B * B - 4. * A * C;
    vcon[G_1] = (-B - sqrt(MY_MAX(0., D))) / (2. * A);
    vcon[G_2] = (FH[0][B_2] * vcon[G_1] - FH[1][B_2]) / FH[0][B_1];
    vcon[G_3] = (FH[0][B_3] * vcon[G_1] - FH[1][B_3]) / FH[0][B_1];
    double gammasq = 1. / (1. - (vcon[1] * vcon[1] + vcon[2] * vcon[2] + vcon[3] * vcon[3]));
    if ((vcon[dir] < cmin) || (vcon[dir] > cmax) || !(fabs(vcon[dir]) > 0.)) *fail_c = 1;
    double v_dot_B = (vcon[1] * FH[0][B1] + vcon[2] * FH[0][B2] + vcon[3] * FH[0][B3]);
    double ptot_HLLC = -(-FH[1][UU] - FH[0][B_1] * (v_dot_B)) * vcon[dir] + FH[1][U_1] + FH[0][B_1] * FH[0][B_1] / gammasq;
    double ptot = ptot_HLLC;
    if (!(fabs(ptot) > 0.)) {
        /* hydrodynamic estimate */
        *fail_c = 1;
        A = 1.;
        B = (-FH[0][UU] - FH[1][U_1]);
        C = -FH[0][U_1] * FH[1][UU] + FH[1][U_1] * FH[0][UU];
        D = B * B - 4. * A * C;
        ptot = (-B + sqrt(MY_MAX(0., D))) / (2. * A);
        if (!(fabs(ptot) > 0.)) {
            *fail_d = 1;
            return -10.;
        }
    }
    double error_1, error_2, ptot_old = ptot, de_dptot, d_ptot = 0.;
    error_1 = hlld_error(dir, ptot, cmin, cmax, FH[0][B_1], R_l, R_r, f);
    for (int n_iter = 0;; n_iter++) {
        error_2 = hlld_error(dir, ptot + 1e-10 * fabs(ptot), cmin, cmax, FH[0][B_1], R_l, R_r, f);
        ptot_old = ptot;
        de_dptot = (error_2 - error_1) / (1e-10 * fabs(ptot));
        d_ptot = error_1 / de_dptot;
        ptot = ptot - d_ptot;
        if (ptot < 0.) ptot = 0.5 * fabs(ptot);
        error_1 = hlld_error(dir, ptot, cmin, cmax, FH[0][B_1], R_l, R_r, f);
        if ((fabs(ptot - ptot_old) <= 1e-8 * fabs(ptot + ptot_old)) || n_iter > 10) break;
    }
    if (!(fabs(ptot) > 0.) || ((fabs(d_ptot) > 1e-8 * fabs(ptot + ptot_old)))) {
        ptot = ptot_HLLC;
        *fail_d = 1;
    }
    return ptot;
}

/* check_HLLD_par (GPU_hllc.h:635-683): contact speed from both sides, the
 * wave fan's ordering and sub-luminal speeds; returns 1 to reject */
static int hlld_check(int dir, double cmin, double cmax, double ptot, hlld_fan *f) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    int fail = 0;
    double vsq;
    f->v_cl[G_1] = (f->v_cl[G_1] + f->v_cr[G_1]) * 0.5;
    f->v_cr[G_1] = f->v_cl[G_1];
    f->v_cl[G_2] = (f->v_cl[G_2] + f->v_cr[G_2]) * 0.5;
    f->v_cr[G_2] = f->v_cl[G_2];
    f->v_cl[G_3] = (f->v_cl[G_3] + f->v_cr[G_3]) * 0.5;
    f->v_cr[G_3] = f->v_cl[G_3];
    if (f->v_cl[G_1] < f->K_al[G_1] || f->v_cl[G_1] < cmin) fail = 1;
    if (f->v_cl[G_1] > f->K_ar[G_1] || f->v_cl[G_1] > cmax) fail = 1;
    vsq = (f->v_cl[1] * f->v_cl[1] + f->v_cl[2] * f->v_cl[2] + f->v_cl[3] * f->v_cl[3]);
    if (!(vsq < 0.999)) fail = 1;
    if (fabs(f->w_al) <= fabs(ptot) || f->v_al[G_1] <= cmin || f->K_al[G_1] <= cmin || f->w_al <= 0.) fail = 1;
    if (fabs(f->w_ar) <= fabs(ptot) || f->v_ar[G_1] >= cmax || f->K_ar[G_1] >= cmax || f->w_ar <= 0.) fail = 1;
    vsq = (f->v_al[1] * f->v_al[1] + f->v_al[2] * f->v_al[2] + f->v_al[3] * f->v_al[3]);
    if (!(vsq < 0.999)) fail = 1;
    vsq = (f->v_ar[1] * f->v_ar[1] + f->v_ar[2] * f->v_ar[2] + f->v_ar[3] * f->v_al[3]);
    if (!(vsq < 0.999)) fail = 1;
    vsq = (f->K_al[1] * f->K_al[1] + f->K_al[2] * f->K_al[2] + f->K_al[3] * f->K_al[3]);
    if (!(vsq < 0.999)) fail = 1;
    vsq = (f->K_ar[1] * f->K_ar[1] + f->K_ar[2] * f->K_ar[2] + f->K_ar[3] * f->K_ar[3]);
    if (!(vsq < 0.999)) fail = 1;
    return fail;
}

/* one outer (a) or inner (c) intermediate state of the fan: X the state's
 * conserved vector, given the residual R and speed S of the outer wave
 * (calc_HLLD_state, GPU_hllc.h:556-613) */
static void hlld_outer(int dir, double S, const double *R, double ptot, const double *v, const double *Bs,
                       double BX, double *X) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    double v_dot_B = v[1] * Bs[1] + v[2] * Bs[2] + v[3] * Bs[3];
    X[RHO] = R[RHO] / (S - v[G_1]);
    X[UU] = (R[UU] - ptot * v[G_1] + v_dot_B * Bs[G_1]) / (S - v[G_1] + SMALL);
    X[UU + G_1] = (-X[UU] + ptot) * v[G_1] - v_dot_B * Bs[G_1];
    X[UU + G_2] = (-X[UU] + ptot) * v[G_2] - v_dot_B * Bs[G_2];
    X[UU + G_3] = (-X[UU] + ptot) * v[G_3] - v_dot_B * Bs[G_3];
    X[B1 + G_1 - 1] = BX;
    X[B1 + G_2 - 1] = Bs[G_2];
    X[B1 + G_3 - 1] = Bs[G_3];
    X[KTOT] = R[KTOT] / (S - v[G_1]);
}

static void hlld_inner(int dir, const double *Xa, double Ka, const double *va, double ptot, const double *vc,
                       const double *Bc, double BX, double *X) {
    const int G_1 = dir, G_2 = dir % 3 + 1, G_3 = (dir + 1) % 3 + 1;
    double v_dot_B = vc[1] * Bc[1] + vc[2] * Bc[2] + vc[3] * Bc[3];
    X[RHO] = Xa[RHO] * (Ka - va[G_1]) / (Ka - vc[G_1]);
    X[UU] = -(-Ka * Xa[UU] - Xa[UU + G_1] + ptot * vc[G_1] - v_dot_B * Xa[B1 + G_1 - 1]) / (Ka - vc[G_1]);
    X[UU + G_1] = (-Xa[UU] + ptot) * vc[G_1] - v_dot_B * Bc[G_1];
    X[UU + G_2] = (-Xa[UU] + ptot) * vc[G_2] - v_dot_B * Bc[G_2];
    X[UU + G_3] = (-Xa[UU] + ptot) * vc[G_3] - v_dot_B * Bc[G_3];
    X[B1 + G_1 - 1] = BX;
    X[B1 + G_2 - 1] = Bc[G_2];
    X[B1 + G_3 - 1] = Bc[G_3];
    X[KTOT] = Xa[KTOT] * (Ka - va[G_1]) / (Ka - vc[G_1]);
}

/* calc_HLLD (GPU_hllc.h:398-423): the HLLD star fluxes where the fan passes
 * every check, else HLLC where its estimate held, else HLL */
static void hlld_mhd(int dir, const double *lu, const double *ru, double iv, double cmin, double cmax,
                     double FT[2][NPR], double FH[2][NPR], const double *Fl, const double *Fr, const double *Ul,
                     const double *Ur) {
    double R_l[NPR], R_r[NPR];
    hlld_fan f;
    int fail_c = 0, fail_d = 0;
    for (int k = 0; k < NPR; k++) R_l[k] = (cmin * Ul[k] - Fl[k]);
    for (int k = 0; k < NPR; k++) R_r[k] = (cmax * Ur[k] - Fr[k]);
    double ptot = hlld_pres(dir, &fail_c, &fail_d, cmin, cmax, FH, R_l, R_r, &f);
    if (fail_d == 0) fail_d = hlld_check(dir, cmin, cmax, ptot, &f);
    if (fail_d == 0) {
        const double BX = FH[0][B1 + dir - 1];
        double X_a[NPR], X_c[NPR];
        /* the fan region holding the face (iv == K_ar exactly is left to
         * HLL: the reference leaves the flux unset there) */
        if ((cmin < iv) && (iv <= f.K_al[dir])) {
            hlld_outer(dir, cmin, R_l, ptot, f.v_al, f.B_al, BX, X_a);
            for (int k = 0; k < NPR; k++) { FT[0][k] = X_a[k]; FT[1][k] = Fl[k] + cmin * (X_a[k] - Ul[k]); }
        } else if ((f.K_al[dir] < iv) && (iv <= f.v_cl[dir])) {
            hlld_outer(dir, cmin, R_l, ptot, f.v_al, f.B_al, BX, X_a);
            hlld_inner(dir, X_a, f.K_al[dir], f.v_al, ptot, f.v_cl, f.B_c, BX, X_c);
            for (int k = 0; k < NPR; k++) {
                FT[0][k] = X_c[k];
                FT[1][k] = Fl[k] + cmin * (X_a[k] - Ul[k]) + f.K_al[dir] * (X_c[k] - X_a[k]);
            }
        } else if ((f.v_cr[dir] <= iv) && (iv < f.K_ar[dir])) {
            hlld_outer(dir, cmax, R_r, ptot, f.v_ar, f.B_ar, BX, X_a);
            hlld_inner(dir, X_a, f.K_ar[dir], f.v_ar, ptot, f.v_cr, f.B_c, BX, X_c);
            for (int k = 0; k < NPR; k++) {
                FT[0][k] = X_c[k];
                FT[1][k] = Fr[k] + cmax * (X_a[k] - Ur[k]) + f.K_ar[dir] * (X_c[k] - X_a[k]);
            }
        } else if ((cmax > iv) && (iv > f.K_ar[dir])) {
            hlld_outer(dir, cmax, R_r, ptot, f.v_ar, f.B_ar, BX, X_a);
            for (int k = 0; k < NPR; k++) { FT[0][k] = X_a[k]; FT[1][k] = Fr[k] + cmax * (X_a[k] - Ur[k]); }
        } else {
            for (int k = 0; k < NPR; k++) { FT[0][k] = FH[0][k]; FT[1][k] = FH[1][k]; }
        }
    } else if (fail_c == 0) {
        hllc_mhd(dir, lu, ru, iv, cmin, cmax, FT, FH, Fl, Fr, Ul, Ur);
    } else {
        for (int k = 0; k < NPR; k++) { FT[0][k] = FH[0][k]; FT[1][k] = FH[1][k]; }
    }
}

/* One face with the HLLC solver in the orthonormal face frame
 * (fluxcalc2D_FT, GPU_hllc.h:3-248): coordinate-frame fast speeds for the
 * time step, states transformed with the frame's inverse, HLL or HLLC star
 * fluxes there (HLLC's hydrodynamic variant where the normal field is
 * negligible), transformed back; pl/pr already carry the normal field.
 * Returns the face's ctop. */
static double hllc_face(double gam, int dir, const double *pl, const double *pr, const geo *gm, double *Fout,
                        int hlld) {
    cstate ql, qr;
    double cmax_l, cmin_l, cmax_r, cmin_r, vd[NPR];
    get_state(pl, gm, &ql);
    get_state(pr, gm, &qr);
    primtoflux(gam, pl, &ql, dir, gm, vd, &cmax_l, &cmin_l);
    primtoflux(gam, pr, &qr, dir, gm, vd, &cmax_r, &cmin_r);
    double cmax1 = fabs(MY_MAX(MY_MAX(0., cmax_l), cmax_r));
    double cmin1 = fabs(MY_MAX(MY_MAX(0., -cmin_l), -cmin_r));
    double ctop = MY_MAX(cmax1, cmin1);
    double Mud[4][4], Mi[4][4];
    ho_set_mud(gm->gcov, gm->gcon, dir, Mud, Mi);
    double lu[4], lb[4], ru[4], rb[4];
    for (int a = 0; a < 4; a++) {
        lu[a] = 0.0; lb[a] = 0.0; ru[a] = 0.0; rb[a] = 0.0;
        for (int b = 0; b < 4; b++) {
            lu[a] += ql.ucon[b] * Mi[a][b];
            lb[a] += ql.bcon[b] * Mi[a][b];
            ru[a] += qr.ucon[b] * Mi[a][b];
            rb[a] += qr.bcon[b] * Mi[a][b];
        }
    }
    double Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR], FT[2][NPR], FH[2][NPR];
    primtoflux_ft(gam, pl, lu, lb, dir, Fl);
    primtoflux_ft(gam, pr, ru, rb, dir, Fr);
    primtoflux_ft(gam, pl, lu, lb, 0, Ul);
    primtoflux_ft(gam, pr, ru, rb, 0, Ur);
    vchar_ft(gam, pl, lu, lb, dir, &cmax_l, &cmin_l);
    vchar_ft(gam, pr, ru, rb, dir, &cmax_r, &cmin_r);
    double cmax = MY_MAX(cmax_r, cmax_l);
    double cmin = MY_MIN(cmin_r, cmin_l);
    const int sdd = dir == 1 ? 4 : (dir == 2 ? 7 : 9);
    double iv = gm->gcon[dir] / (sqrt(gm->gcon[dir] * gm->gcon[dir] - gm->gcon[0] * gm->gcon[sdd]));
    if (cmax <= iv) {
        for (int k = 0; k < NPR; k++) { FT[0][k] = Ur[k]; FT[1][k] = Fr[k]; }
    } else if (cmin >= iv) {
        for (int k = 0; k < NPR; k++) { FT[0][k] = Ul[k]; FT[1][k] = Fl[k]; }
    } else {
        for (int k = 0; k < NPR; k++) FH[0][k] = (Fl[k] - Fr[k] + cmax * Ur[k] - cmin * Ul[k]) / (cmax - cmin + SMALL);
        for (int k = 0; k < NPR; k++)
            FH[1][k] = ((cmax * Fl[k] - cmin * Fr[k] + cmax * cmin * (Ur[k] - Ul[k])) / (cmax - cmin + SMALL));
        int do_hydro = (fabs(FH[0][dir + B1 - 1] * FH[0][dir + B1 - 1] * lu[0] * ru[0]) < pow(10., -10.) * fabs(FH[0][UU]));
        if (do_hydro) hllc_hydro(dir, lu, ru, iv, cmin, cmax, FT, FH, Fl, Fr, Ul, Ur);
        else if (hlld) hlld_mhd(dir, lu, ru, iv, cmin, cmax, FT, FH, Fl, Fr, Ul, Ur);
        else hllc_mhd(dir, lu, ru, iv, cmin, cmax, FT, FH, Fl, Fr, Ul, Ur);
    }
    double F1[NPR];
    for (int j1 = 0; j1 < 4; j1++) {
        F1[j1 + UU] = 0.;
        for (int j2 = 0; j2 < 4; j2++) {
            F1[j1 + UU] += FT[0][j2 + UU] * Mud[dir][0] * Mi[j2][j1];
            F1[j1 + UU] += FT[1][j2 + UU] * Mud[dir][dir] * Mi[j2][j1];
        }
    }
    FT[0][U3] = 0.;
    FT[1][U3] = -FT[0][B1 - 1 + dir];
    for (int j1 = 1; j1 < 4; j1++) {
        F1[j1 + U3] = 0.;
        for (int j2 = 0; j2 < 4; j2++) {
            F1[j1 + U3] += FT[0][j2 + U3] * Mud[dir][0] * Mud[j1][j2];
            F1[j1 + U3] += FT[1][j2 + U3] * Mud[dir][dir] * Mud[j1][j2];
        }
    }
    F1[RHO] = FT[0][RHO] * Mud[dir][0];
    F1[RHO] += FT[1][RHO] * Mud[dir][dir];
    F1[KTOT] = FT[0][KTOT] * Mud[dir][0];
    F1[KTOT] += FT[1][KTOT] * Mud[dir][dir];
    F1[UU] += F1[RHO];
    for (int k = 0; k < NPR; k++) Fout[k] = gm->g * F1[k];
    return ctop;
}

/* ----------------------------------------------------------------- flux -- */
/*
 * Face fluxes in direction dir (fluxcalcprep + fluxcalc2D2, GPU_program1.cu:78-1068,
 * torus branch :791-1055): PPM face states from the two adjacent cells (left =
 * upper edge value of cell - 1, right = lower edge value of cell), normal B
 * from the staggered field, B1 zeroed on polar x2-faces, HLL flux, and the
 * face's CFL limit cour*dx/ctop. Faces cover the normal range [ng, n+ng] and
 * one ghost layer either side transversally.
 */
static void fluxes(const ho_grid *g, const dims *d, const ho_geom *m, const double *pv,
                   const double *ps, int dir, double *F, double *dtmin) {
    int idel = dir == 1, jdel = dir == 2, zdel = dir == 3;
    long stride = idel ? (long)d->G2 * d->G3 : (jdel ? d->G3 : 1);
    int face = dir == 1 ? FACE1 : (dir == 2 ? FACE2 : FACE3);
    double dxd = dir == 1 ? g->dx1 : (dir == 2 ? g->dx2 : g->dx3);
    double factor = g->cour * dxd;
    int i0 = (d->ng1 - 1) * d->d1 + idel, i1 = i0 + (d->n1 + 2 * d->d1 - idel);
    int j0 = (d->ng2 - 1) * d->d2 + jdel, j1 = j0 + (d->n2 + 2 * d->d2 - jdel);
    int z0 = (d->ng3 - 1) * d->d3 + zdel, z1 = z0 + (d->n3 + 2 * d->d3 - zdel);
    double best = 1.e9;
#pragma omp parallel for collapse(2) reduction(min : best) schedule(static)
    for (int i = i0; i < i1; i++)
        for (int j = j0; j < j1; j++)
            for (int z = z0; z < z1; z++) {
                long c = cix(d, i, j, z);
                geo gm;
                load_geo(d, m, i, j, face, &gm);
                double pl[NPR], pr[NPR], lo, hi, x[5];
                for (int k = 0; k < NPR; k++) {
                    const double *pk = pv + (long)k * d->ks;
                    if (g->recon == 1) {
                        double xm = pk[c - stride], temp;
                        temp = 0.5 * ho_slope_lim(pk[c - 2 * stride], xm, pk[c]);
                        pl[k] = xm + temp;              /* dq2 of cell c - 1 */
                        temp = 0.5 * ho_slope_lim(xm, pk[c], pk[c + stride]);
                        pr[k] = pk[c] - temp;           /* dq1 of cell c */
                        continue;
                    }
                    /* upper edge of cell c - 1 */
                    for (int t = 0; t < 5; t++) x[t] = pk[c - stride + (t - 2) * stride];
                    ho_para(x, &lo, &hi);
                    pl[k] = hi;
                    /* lower edge of cell c */
                    for (int t = 0; t < 5; t++) x[t] = pk[c + (t - 2) * stride];
                    ho_para(x, &lo, &hi);
                    pr[k] = lo;
                }
                double bn = ps[(long)(dir - 1) * d->ks + c];
                pl[B1 + dir - 1] = bn;
                pr[B1 + dir - 1] = bn;
                if (dir == 2 && ((j == d->n2 + d->ng2 && g->pole2) || (j == d->ng2 && g->pole1))) {
                    pl[B1] = 0.;
                    pr[B1] = 0.;
                }
                if (g->riemann >= 1) {
                    double Fo[NPR];
                    double ctop = hllc_face(g->gam, dir, pl, pr, &gm, Fo, g->riemann == 2);
                    for (int k = 0; k < NPR; k++) F[(long)k * d->ks + c] = Fo[k];
                    double dtf = factor / ctop;
                    if (dtf < best && dtf > 1.e-6) best = dtf;
                    continue;
                }
                cstate q;
                double t1[NPR], t2[NPR], t3[NPR], t4[NPR];
                double cmax_l, cmin_l, cmax_r, cmin_r;
                get_state(pl, &gm, &q);
                primtoflux(g->gam, pl, &q, dir, &gm, t1, &cmax_l, &cmin_l);
                primtoflux(g->gam, pl, &q, 0, &gm, t2, &cmax_l, &cmin_l);
                get_state(pr, &gm, &q);
                primtoflux(g->gam, pr, &q, dir, &gm, t3, &cmax_r, &cmin_r);
                primtoflux(g->gam, pr, &q, 0, &gm, t4, &cmax_r, &cmin_r);
                double cmax = fabs(MY_MAX(MY_MAX(0., cmax_l), cmax_r));
                double cmin = fabs(MY_MAX(MY_MAX(0., -cmin_l), -cmin_r));
                double ctop = MY_MAX(cmax, cmin);
                for (int k = 0; k < NPR; k++)
                    F[(long)k * d->ks + c] = (cmax * t1[k] + cmin * t3[k] - cmax * cmin * (t4[k] - t2[k])) / (cmax + cmin + SMALL);
                double dtf = factor / ctop;
                if (dtf < best && dtf > 1.e-6) best = dtf;
            }
    *dtmin = best;
}

/* fix_flux (GPU_const_trans.h:3-61) for reflective poles, INFLOW == 0, both
 * radial edges of the block are domain edges */
static void fix_flux(const ho_grid *g, const dims *d, double *F1, double *F2, double *F3) {
    long ks = d->ks;
    for (int i = 0; i < d->G1; i++)
        for (int z = 0; z < d->G3; z++) {
            if (!(i >= d->ng1 - d->d1 && z >= d->ng3 - d->d3 && i < d->n1 + d->ng1 + d->d1 && z < d->n3 + d->ng3 + d->d3)) continue;
            if (g->pole1) {
                F1[B2 * ks + cix(d, i, d->ng2 - 1, z)] = -F1[B2 * ks + cix(d, i, d->ng2, z)];
                if (d->ng3 > 0) F3[B2 * ks + cix(d, i, d->ng2 - 1, z)] = -F3[B2 * ks + cix(d, i, d->ng2, z)];
                for (int k = 0; k < NPR; k++) F2[k * ks + cix(d, i, d->ng2, z)] = 0.;
            }
            if (g->pole2) {
                F1[B2 * ks + cix(d, i, d->n2 + d->ng2, z)] = -F1[B2 * ks + cix(d, i, d->n2 + d->ng2 - 1, z)];
                if (d->ng3 > 0) F3[B2 * ks + cix(d, i, d->n2 + d->ng2, z)] = -F3[B2 * ks + cix(d, i, d->n2 + d->ng2 - 1, z)];
                for (int k = 0; k < NPR; k++) F2[k * ks + cix(d, i, d->n2 + d->ng2, z)] = 0.;
            }
        }
    for (int j = 0; j < d->G2; j++)
        for (int z = 0; z < d->G3; z++) {
            if (!(j >= d->ng2 - d->d2 && z >= d->ng3 - d->d3 && j < d->n2 + d->ng2 + d->d2 && z < d->n3 + d->ng3 + d->d3)) continue;
            long ci = RHO * ks + cix(d, d->ng1, j, z);
            if (!(g->halo & 1) && F1[ci] > 0.) F1[ci] = 0.;
            long co = RHO * ks + cix(d, d->n1 + d->ng1, j, z);
            if (!(g->halo & 2) && F1[co] < 0.) F1[co] = 0.;
        }
}

/* ------------------------------------------------- constrained transport -- */
/* consttransport1 (GPU_const_trans.h:63-119): cell-centre EMF -gdet (u x b) */
static void emf_centre(const dims *d, const ho_geom *m, const double *pv, double *E_cent) {
    long ks = d->ks;
    int i0 = (d->ng1 - d->d1) * d->d1, j0 = (d->ng2 - d->d2) * d->d2, z0 = (d->ng3 - d->d3) * d->d3;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = i0; i < i0 + d->n1 + 2 * d->d1; i++)
        for (int j = j0; j < j0 + d->n2 + 2 * d->d2; j++)
            for (int z = z0; z < z0 + d->n3 + 2 * d->d3; z++) {
                long c = cix(d, i, j, z);
                double pb[NPR];
                for (int k = 0; k < NPR; k++) pb[k] = pv[k * ks + c];
                geo gm;
                load_geo(d, m, i, j, CENT, &gm);
                double ucon[4], ucov[4], bcon[4];
                ucon_calc(pb, &gm, ucon);
                lower4(ucon, gm.gcov, ucov);
                bcon_calc(pb, ucon, ucov, bcon);
                if (d->ng3 > 0) {
                    E_cent[1 * ks + c] = -gm.g * (ucon[2] * bcon[3] - ucon[3] * bcon[2]);
                    E_cent[2 * ks + c] = -gm.g * (ucon[3] * bcon[1] - ucon[1] * bcon[3]);
                }
                E_cent[3 * ks + c] = -gm.g * (ucon[1] * bcon[2] - ucon[2] * bcon[1]);
            }
}

static inline double up(double f) { return (double)(f <= 0.0); }
static inline double dn(double f) { return (double)(f > 0.0); }

/* consttransport2 with every upwind correction zero (the reference's
 * RESISTIVE || CARTESIAN branch, GPU_const_trans.h:187-211): each edge EMF is
 * the average of its four face EMFs. */
static void emf_average_only(const dims *d, long c, const double *F1, const double *F2, const double *F3,
                             double *emf, const ho_grid *g, int j) {
    long ks = d->ks, jsize = d->G3, isize = (long)d->G2 * d->G3;
    long D1 = d->d1, D2 = d->d2, D3 = d->d3;
    const double factor = 1.0;
    const double *F1r = F1 + RHO * ks, *F2r = F2 + RHO * ks, *F3r = F3 + RHO * ks;
    const double z0 = 0.0;
    emf[1 * ks + c] = 0.25 * ((-factor * F2[B3 * ks + c] - (z0 * up(F2r[c]) + z0 * dn(F2r[c])))
        + (-factor * F2[B3 * ks + c - D3] + (z0 * up(F2r[c - D3]) + z0 * dn(F2r[c - D3]))) +
        +(factor * F3[B2 * ks + c] - (z0 * up(F3r[c]) + z0 * dn(F3r[c])))
        + (factor * F3[B2 * ks + c - D2 * jsize] + (z0 * up(F3r[c - D2 * jsize]) + z0 * dn(F3r[c - D2 * jsize]))));
    emf[2 * ks + c] = 0.25 * ((-factor * F3[B1 * ks + c] - (z0 * up(F3r[c]) + z0 * dn(F3r[c])))
        + (-factor * F3[B1 * ks + c - D1 * isize] + (z0 * up(F3r[c - D1 * isize]) + z0 * dn(F3r[c - D1 * isize])))
        + (factor * F1[B3 * ks + c] - (z0 * up(F1r[c]) + z0 * dn(F1r[c])))
        + (factor * F1[B3 * ks + c - D3] + (z0 * up(F1r[c - D3]) + z0 * dn(F1r[c - D3]))));
    emf[3 * ks + c] = 0.25 * ((factor * F2[B1 * ks + c] - (z0 * up(F2r[c]) + z0 * dn(F2r[c])))
        + (factor * F2[B1 * ks + c - D1 * isize] + (z0 * up(F2r[c - D1 * isize]) + z0 * dn(F2r[c - D1 * isize])))
        + (-factor * F1[B2 * ks + c] - (z0 * up(F1r[c]) + z0 * dn(F1r[c])))
        + (-factor * F1[B2 * ks + c - D2 * jsize] + (z0 * up(F1r[c - D2 * jsize]) + z0 * dn(F1r[c - D2 * jsize]))));
    if ((g->pole1 && j == d->ng2) || (g->pole2 && j == d->n2 + d->ng2)) {
        emf[3 * ks + c] = 0.;
        emf[1 * ks + c] = -0.5 * factor * (F2[B3 * ks + c] + F2[B3 * ks + c - D3]);
    }
}

/* consttransport2 (GPU_const_trans.h:121-338): edge EMFs from the four face
 * fluxes plus the upwinded centre-minus-face corrections, the upwind side
 * chosen by the sign of the mass flux through each face; polar edge rule. */
static void emf_edges(const ho_grid *g, const dims *d, const double *E_cent, const double *F1,
                      const double *F2, const double *F3, double *emf) {
    long ks = d->ks;
    long jsize = d->G3, isize = (long)d->G2 * d->G3;
    long D1 = d->d1, D2 = d->d2, D3 = d->d3;
    const double factor = 1.0;
    const double *Ec1 = E_cent + 1 * ks, *Ec2 = E_cent + 2 * ks, *Ec3 = E_cent + 3 * ks;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = d->ng1 * d->d1; i < d->ng1 * d->d1 + d->n1 + d->d1; i++)
        for (int j = d->ng2 * d->d2; j < d->ng2 * d->d2 + d->n2 + d->d2; j++)
            for (int z = d->ng3 * d->d3; z < d->ng3 * d->d3 + d->n3 + d->d3; z++) {
                long c = cix(d, i, j, z);
                if (!g->ct_upwind) {
                    emf_average_only(d, c, F1, F2, F3, emf, g, j);
                    continue;
                }
                double dE_LEFT_13_1 = Ec1[c] - factor * F3[B2 * ks + c];
                double dE_LEFT_13_2 = Ec1[c - jsize * D2] - factor * F3[B2 * ks + c - jsize * D2];
                double dE_RIGHT_13_1 = factor * F3[B2 * ks + c + D3 - D3] - Ec1[c - D3];
                double dE_RIGHT_13_2 = factor * F3[B2 * ks + c + D3 - jsize * D2 - D3] - Ec1[c - jsize * D2 - D3];
                double dE_LEFT_12_1 = Ec1[c] + factor * F2[B3 * ks + c];
                double dE_LEFT_12_2 = Ec1[c - D3] + factor * F2[B3 * ks + c - D3];
                double dE_RIGHT_12_1 = -factor * F2[B3 * ks + c + D2 * jsize - D2 * jsize] - Ec1[c - D2 * jsize];
                double dE_RIGHT_12_2 = -factor * F2[B3 * ks + c + D2 * jsize - D2 * jsize - D3] - Ec1[c - D2 * jsize - D3];
                double dE_LEFT_21_1 = Ec2[c] - factor * F1[B3 * ks + c];
                double dE_LEFT_21_2 = Ec2[c - D3] - factor * F1[B3 * ks + c - D3];
                double dE_RIGHT_21_1 = factor * F1[B3 * ks + c + D1 * isize - D1 * isize] - Ec2[c - D1 * isize];
                double dE_RIGHT_21_2 = factor * F1[B3 * ks + c + D1 * isize - D1 * isize - D3] - Ec2[c - D1 * isize - D3];
                double dE_LEFT_23_1 = Ec2[c] + factor * F3[B1 * ks + c];
                double dE_LEFT_23_2 = Ec2[c - D1 * isize] + factor * F3[B1 * ks + c - D1 * isize];
                double dE_RIGHT_23_1 = -factor * F3[B1 * ks + c + D3 - D3] - Ec2[c - D3];
                double dE_RIGHT_23_2 = -factor * F3[B1 * ks + c + D3 - isize * D1 - D3] - Ec2[c - isize * D1 - D3];
                double dE_LEFT_31_1 = Ec3[c] + factor * F1[B2 * ks + c];
                double dE_LEFT_31_2 = Ec3[c - D2 * jsize] + factor * F1[B2 * ks + c - D2 * jsize];
                double dE_RIGHT_31_1 = -factor * F1[B2 * ks + c + D1 * isize - D1 * isize] - Ec3[c - D1 * isize];
                double dE_RIGHT_31_2 = -factor * F1[B2 * ks + c + D1 * isize - D1 * isize - D2 * jsize] - Ec3[c - D1 * isize - D2 * jsize];
                double dE_LEFT_32_1 = Ec3[c] - factor * F2[B1 * ks + c];
                double dE_LEFT_32_2 = Ec3[c - D1 * isize] - factor * F2[B1 * ks + c - D1 * isize];
                double dE_RIGHT_32_1 = factor * F2[B1 * ks + c + D2 * jsize - D2 * jsize] - Ec3[c - D2 * jsize];
                double dE_RIGHT_32_2 = factor * F2[B1 * ks + c + D2 * jsize - D1 * isize - D2 * jsize] - Ec3[c - D1 * isize - D2 * jsize];
                const double *F1r = F1 + RHO * ks, *F2r = F2 + RHO * ks, *F3r = F3 + RHO * ks;

                emf[1 * ks + c] = 0.25 * ((-factor * F2[B3 * ks + c] - (dE_LEFT_13_1 * up(F2r[c]) + dE_LEFT_13_2 * dn(F2r[c])))
                    + (-factor * F2[B3 * ks + c - D3] + (dE_RIGHT_13_1 * up(F2r[c - D3]) + dE_RIGHT_13_2 * dn(F2r[c - D3]))) +
                    +(factor * F3[B2 * ks + c] - (dE_LEFT_12_1 * up(F3r[c]) + dE_LEFT_12_2 * dn(F3r[c])))
                    + (factor * F3[B2 * ks + c - D2 * jsize] + (dE_RIGHT_12_1 * up(F3r[c - D2 * jsize]) + dE_RIGHT_12_2 * dn(F3r[c - D2 * jsize]))));
                emf[2 * ks + c] = 0.25 * ((-factor * F3[B1 * ks + c] - (dE_LEFT_21_1 * up(F3r[c]) + dE_LEFT_21_2 * dn(F3r[c])))
                    + (-factor * F3[B1 * ks + c - D1 * isize] + (dE_RIGHT_21_1 * up(F3r[c - D1 * isize]) + dE_RIGHT_21_2 * dn(F3r[c - D1 * isize])))
                    + (factor * F1[B3 * ks + c] - (dE_LEFT_23_1 * up(F1r[c]) + dE_LEFT_23_2 * dn(F1r[c])))
                    + (factor * F1[B3 * ks + c - D3] + (dE_RIGHT_23_1 * up(F1r[c - D3]) + dE_RIGHT_23_2 * dn(F1r[c - D3]))));
                emf[3 * ks + c] = 0.25 * ((factor * F2[B1 * ks + c] - (dE_LEFT_31_1 * up(F2r[c]) + dE_LEFT_31_2 * dn(F2r[c])))
                    + (factor * F2[B1 * ks + c - D1 * isize] + (dE_RIGHT_31_1 * up(F2r[c - D1 * isize]) + dE_RIGHT_31_2 * dn(F2r[c - D1 * isize])))
                    + (-factor * F1[B2 * ks + c] - (dE_LEFT_32_1 * up(F1r[c]) + dE_LEFT_32_2 * dn(F1r[c])))
                    + (-factor * F1[B2 * ks + c - D2 * jsize] + (dE_RIGHT_32_1 * up(F1r[c - D2 * jsize]) + dE_RIGHT_32_2 * dn(F1r[c - D2 * jsize]))));
                if ((g->pole1 && j == d->ng2) || (g->pole2 && j == d->n2 + d->ng2)) {
                    emf[3 * ks + c] = 0.;
                    emf[1 * ks + c] = -0.5 * factor * (F2[B3 * ks + c] + F2[B3 * ks + c - D3]);
                }
            }
}

/* E_average (const_trans.c:268-503) for one block holding every phi cell:
 * the polar x1-EMF is replaced by its phi average (computed on dt-scaled
 * values, as packsend2E / unpackreceive2E do), the x3-EMF there is zeroed. */
static void emf_pole_average(const ho_grid *g, const dims *d, double *emf, double dt) {
    long ks = d->ks;
    for (int side = 0; side < 2; side++) {
        if ((side == 0 && !g->pole1) || (side == 1 && !g->pole2)) continue;
        int jp = side == 0 ? d->ng2 : d->n2 + d->ng2;
        for (int i = d->ng1; i < d->n1 + 2 * d->ng1; i++) {
            double avg = 0.;
            for (int z = d->ng3; z < d->n3 + d->ng3; z++) avg += dt * emf[1 * ks + cix(d, i, jp, z)];
            avg /= (double)(d->n3);
            double avg_new = avg / ((double)1);
            for (int z = d->ng3; z < d->n3 + 2 * d->ng3; z++) {
                emf[1 * ks + cix(d, i, jp, z)] = avg_new / dt;
                emf[3 * ks + cix(d, i, jp, z)] = 0.;
            }
        }
    }
}

/* consttransport3 (GPU_const_trans.h:426-529): face-B update from the edge EMFs */
static void face_update(const ho_grid *g, const dims *d, const ho_geom *m, const double *psi,
                        double *psf, const double *E, double Dt) {
    long ks = d->ks;
    long isize = (long)d->G2 * d->G3, jsz = d->G3;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = d->ng1 * d->d1; i < d->ng1 * d->d1 + d->n1 + d->d1; i++)
        for (int j = d->ng2 * d->d2; j < d->ng2 * d->d2 + d->n2 + d->d2; j++)
            for (int z = d->ng3 * d->d3; z < d->ng3 * d->d3 + d->n3 + d->d3; z++) {
                long c = cix(d, i, j, z);
                long gi = gix(d, i, j);
                int in1 = i < d->n1 + d->ng1 + d->d1, in2 = j < d->n2 + d->ng2, in3 = z < d->n3 + d->ng3;
                if (in1 && in2 && in3) {
                    double gdf = m->gdet[FACE1 * d->gs + gi];
                    double temp = 0.;
                    temp += 1.0 / ((double)1) * psi[c] * gdf;
                    temp += -Dt / ((double)1 * g->dx2) * (E[3 * ks + c + jsz] - E[3 * ks + c]);
                    if (d->ng3 > 0) temp += Dt / ((double)1 * g->dx3) * (E[2 * ks + c + d->d3] - E[2 * ks + c]);
                    psf[c] = temp / gdf;
                }
                int j3 = i < d->n1 + d->ng1 && j < d->n2 + d->ng2 && z < d->n3 + d->ng3 + d->d3;
                if (j3 && d->ng3 > 0) {
                    double gdf = m->gdet[FACE3 * d->gs + gi];
                    double temp = psi[2 * ks + c] * gdf;
                    temp += -Dt / g->dx1 * (E[2 * ks + c + isize] - E[2 * ks + c]);
                    temp += Dt / g->dx2 * (E[1 * ks + c + jsz] - E[1 * ks + c]);
                    psf[2 * ks + c] = temp / gdf;
                }
                int j2 = i < d->n1 + d->ng1 && j < d->n2 + d->ng2 + d->d2 && z < d->n3 + d->ng3;
                if (j2) {
                    double gdf = m->gdet[FACE2 * d->gs + gi];
                    double temp = 0.;
                    temp += 1.0 / ((double)1) * psi[1 * ks + c] * gdf;
                    temp += Dt / ((double)1 * g->dx1) * (E[3 * ks + c + isize] - E[3 * ks + c]);
                    if (d->ng3 > 0) temp += -Dt / ((double)1 * g->dx3) * (E[1 * ks + c + d->d3] - E[1 * ks + c]);
                    psf[1 * ks + c] = temp / gdf;
                }
            }
}

/* ------------------------------------------------------------- sources -- */
/* source (GPU_phys_mhd.h:34-175): gdet T^kappa_nu Gamma^nu_{lambda kappa} */
static void source(double gam, const double *ph, const geo *gm, const dims *d, const ho_geom *m,
                   int i, int j, double *dU, const cstate *q) {
    double mhd[4][4];
    long gi = gix(d, i, j), gs = d->gs;
    double P = (gam - 1.) * ph[UU];
    double u = ph[UU];
    double w = P + ph[RHO] + u;
    double bsq = dot4(q->bcon, q->bcov);
    double eta = w + bsq;
    double ptot = P + 0.5 * bsq;
    for (int dir = 0; dir < 4; dir++)
        for (int jj = 0; jj < 4; jj++)
            mhd[dir][jj] = eta * q->ucon[dir] * q->ucov[jj] + ptot * (dir == jj ? 1. : 0.) - q->bcon[dir] * q->bcov[jj];
    for (int k = 0; k < NPR; k++) dU[k] = 0.;
#define CONN(s, k) (m->conn[(long)((s) * 4 + (k)) * gs + gi])
    for (int k = 0; k < 4; k++) {
        double c;
        dU[UU] += mhd[0][k] * CONN(0, k);
        dU[U1] += mhd[1][k] * CONN(4, k);
        dU[U2] += mhd[2][k] * CONN(7, k);
        dU[U3] += mhd[3][k] * CONN(9, k);
        c = CONN(1, k); dU[UU] += mhd[1][k] * c; dU[U1] += mhd[0][k] * c;
        c = CONN(2, k); dU[UU] += mhd[2][k] * c; dU[U2] += mhd[0][k] * c;
        c = CONN(3, k); dU[UU] += mhd[3][k] * c; dU[U3] += mhd[0][k] * c;
        c = CONN(5, k); dU[U1] += mhd[2][k] * c; dU[U2] += mhd[1][k] * c;
        c = CONN(6, k); dU[U1] += mhd[3][k] * c; dU[U3] += mhd[1][k] * c;
        c = CONN(8, k); dU[U2] += mhd[3][k] * c; dU[U3] += mhd[2][k] * c;
    }
#undef CONN
    dU[UU] *= gm->g;
    dU[U1] *= gm->g;
    dU[U2] *= gm->g;
    dU[U3] *= gm->g;
    dU[KTOT] *= gm->g;
}

/* ------------------------------------------------------------ inversion -- */
/* Noble et al. 2006 2D (W, v^2) scheme, GPU_utoprim_2d.h */
static double vsq_calc(double W, double Bsq, double Qtsq, double QdotBsq) {
    double Wsq = W * W;
    double Xsq = (Bsq + W) * (Bsq + W);
    return (Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * Xsq);
}
static double x1_of_x0(double x0, double Bsq, double Qtsq, double QdotBsq) {
    double vsq = fabs(vsq_calc(x0, Bsq, Qtsq, QdotBsq));
    return (vsq > 1.) ? (1.0 - 1.e-15) : vsq;
}
static void validate_x(double x[2], const double x0[2]) {
    x[0] = fabs(x[0]);
    x[0] = (x[0] > W_TOO_BIG) ? x0[0] : x[0];
    x[1] = (x[1] < 0.) ? 0. : x[1];
    x[1] = (x[1] > 1.) ? (1. - 1.e-15) : x[1];
}
/* func_vsq (GPU_utoprim_2d.h): residuals and Newton step, ideal gas */
static void func_vsq(double gam, const double x[2], double dx[2], double *f, double *df,
                     double Bsq, double Qtsq, double QdotBsq, double Qdotn, double D) {
    double Wsq = x[0] * x[0];
    double gtmp = 1. - x[1];
    double p_tmp = (gam - 1.) * (fma(x[0], gtmp, -D * sqrt(gtmp))) / gam;
    double dPdW = (gam - 1.) * (1. - x[1]) / gam;
    double dPdvsq = (gam - 1.) * (fma(0.5, D / sqrt(1. - x[1]), -x[0])) / gam;
    double t2 = -0.5 * Bsq + dPdvsq;
    double t3 = Bsq + x[0];
    double t4 = t3 * t3;
    double t9 = 1. / Wsq;
    double t11 = Qtsq - x[1] * t4 + QdotBsq * (Bsq + 2.0 * x[0]) * t9;
    double t16 = QdotBsq * t9;
    double t18 = -Qdotn - 0.5 * Bsq * (1.0 + x[1]) + 0.5 * t16 - x[0] + p_tmp;
    double t21 = 1. / t3;
    double t23 = 1. / x[0];
    double t24 = t16 * t23;
    double t25 = -1.0 + dPdW - t24;
    double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + x[1] * Wsq * x[0]) * t9 * t23;
    double t36 = 1. / t35;
    dx[0] = -(t2 * t11 + t4 * t18) * t21 * t36;
    double t40 = (x[1] + t24) * t3;
    dx[1] = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
    double resid0 = t11, resid1 = t18;
    *df = -resid0 * resid0 - resid1 * resid1;
    *f = -0.5 * (*df);
}
static int newton_2d(double gam, double x[2], double Bsq, double Qtsq, double QdotBsq, double Qdotn,
                     double D, double tolerance) {
    double f = 1., df = 1., dx[2], x_old[2], errx = 1.;
    int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
    x_old[0] = x[0]; x_old[1] = x[1];
    while (keep) {
        func_vsq(gam, x, dx, &f, &df, Bsq, Qtsq, QdotBsq, Qdotn, D);
        errx = 0.;
        x_old[0] = x[0]; x_old[1] = x[1];
        x[0] += dx[0]; x[1] += dx[1];
        validate_x(x, x_old);
        errx = (x[0] == 0.) ? fabs(x[0] - x_old[0]) : fabs((x[0] - x_old[0]) / x[0]);
        if ((fabs(errx) <= tolerance) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
        if (doing_extra == 1) i_extra++;
        if (((fabs(errx) <= tolerance) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
            keep = 0;
        n_iter++;
    }
    if ((isfinite(f) == 0) || (isfinite(df) == 0)) return 2;
    if (fabs(errx) > MY_MIN(tolerance, MIN_NEWT_TOL)) return 1;
    return 0;
}

/* scalars shared by the three inversions (Utoprim_new_body*, GPU_utoprim_*.h) */
typedef struct { double Bcon[4], Qcon[4], ncon[4], Bsq, QdotB, QdotBsq, Qtsq, Qdotn, D; } invq;
static void inv_scalars(const double *U, const double *gcov, const double *gcon, invq *s) {
    double Bcov[4], Qcov[4], Qsq, ncov;
    s->Bcon[0] = 0.;
    for (int i = 1; i < 4; i++) s->Bcon[i] = U[B1 + i - 1];
    lower4(s->Bcon, gcov, Bcov);
    for (int i = 0; i < 4; i++) Qcov[i] = U[UU + i];
    raise4(Qcov, gcon, s->Qcon);
    s->Bsq = 0.;
    for (int i = 1; i < 4; i++) s->Bsq += s->Bcon[i] * Bcov[i];
    s->QdotB = 0.;
    for (int i = 0; i < 4; i++) s->QdotB += Qcov[i] * s->Bcon[i];
    s->QdotBsq = s->QdotB * s->QdotB;
    ncov = -sqrt(-1. / gcon[0]);
    s->ncon[0] = gcon[0] * ncov;
    s->ncon[1] = gcon[1] * ncov;
    s->ncon[2] = gcon[2] * ncov;
    s->ncon[3] = gcon[3] * ncov;
    s->Qdotn = s->Qcon[0] * ncov;
    Qsq = 0.;
    for (int i = 0; i < 4; i++) Qsq += Qcov[i] * s->Qcon[i];
    s->Qtsq = Qsq + s->Qdotn * s->Qdotn;
    s->D = U[RHO];
}
static int guess_utsq(const double *gcov, const double *prim, double *utsq_out) {
    double utsq = gcov[4] * prim[U1] * prim[U1];
    utsq += 2. * gcov[5] * prim[U2] * prim[U1];
    utsq += 2. * gcov[6] * prim[U3] * prim[U1];
    utsq += gcov[7] * prim[U2] * prim[U2];
    utsq += 2 * gcov[8] * prim[U3] * prim[U2];
    utsq += gcov[9] * prim[U3] * prim[U3];
    if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
    if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 2;
    *utsq_out = utsq;
    return 0;
}
static void set_velocity(const invq *s, double gamma, double W, double *prim) {
    for (int i = 1; i < 4; i++) {
        double Qtcon = s->Qcon[i] + s->ncon[i] * s->Qdotn;
        prim[U1 + i - 1] = gamma / (W + s->Bsq) * (Qtcon + s->QdotB * s->Bcon[i] / W);
    }
}
/* Transform U into the normal-observer frame (Utoprim_2d prologue) */
static int inv_prologue(const double *U, double gdet, const double *gcon, double *prim, double *U_tmp) {
    if (U[0] <= 0.) return -100;
    for (int i = B1; i <= B3; i++) prim[i] = U[i] / gdet;
    double alpha = 1.0 / sqrt(-gcon[0]);
    U_tmp[RHO] = alpha * U[RHO] / gdet;
    U_tmp[UU] = alpha * (U[UU] - U[RHO]) / gdet;
    for (int i = U1; i <= U3; i++) U_tmp[i] = alpha * U[i] / gdet;
    for (int i = B1; i <= B3; i++) U_tmp[i] = alpha * U[i] / gdet;
    return 0;
}

static int body_2d(double gam, const double *U, const double *gcov, const double *gcon, double *prim) {
    invq s;
    double utsq, x[2];
    inv_scalars(U, gcov, gcon, &s);
    if (guess_utsq(gcov, prim, &utsq)) return 2;
    double gammasq = 1. + utsq;
    double gamma = sqrt(gammasq);
    double rho0 = s.D / gamma;
    double u = prim[UU];
    double p = (gam - 1.) * u;
    double w = rho0 + u + p;
    double W_last = w * gammasq;
    int i_increase = 0;
    while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <= W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) && (i_increase < 10)) {
        W_last *= 10.;
        i_increase++;
    }
    x[0] = fabs(W_last);
    x[1] = x1_of_x0(W_last, s.Bsq, s.Qtsq, s.QdotBsq);
    int retval = newton_2d(gam, x, s.Bsq, s.Qtsq, s.QdotBsq, s.Qdotn, s.D, NEWT_TOL);
    double W = x[0], vsq = x[1];
    if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
    if (W <= 0. || W > W_TOO_BIG) return 3;
    if (vsq >= 1.) return 4;
    double gtmp = sqrt(1. - vsq);
    gamma = 1. / gtmp;
    rho0 = s.D * gtmp;
    w = W * (1. - vsq);
    p = (gam - 1.) * (w - rho0) / gam;
    u = w - (rho0 + p);
    if (rho0 <= 0.) return 5;
    if (u <= 0.) return 6;
    prim[RHO] = rho0;
    prim[UU] = u;
    set_velocity(&s, gamma, W, prim);
    return 0;
}

/* Utoprim_2d (GPU_utoprim_2d.h:1-98) */
int ho_utoprim_2d(double gam, double *U, const double *gcov, const double *gcon, double gdet, double *prim) {
    double U_tmp[NPR], prim_tmp[5];
    int ret = inv_prologue(U, gdet, gcon, prim, U_tmp);
    if (ret) return ret;
    for (int i = 0; i < B1; i++) prim_tmp[i] = prim[i];
    ret = body_2d(gam, U_tmp, gcov, gcon, prim_tmp);
    if (ret == 0)
        for (int i = 0; i < B1; i++) prim[i] = prim_tmp[i];
    return ret;
}

/* Entropy-based 1D fallback in v^2 (GPU_utoprim_1dvsq2fix1.h) */
static double W_of_vsq2(double gam, double vsq, double *p, double *rho, double *u, double D, double K_atm) {
    double gtmp = (1. - vsq);
    *rho = D * sqrt(gtmp);
    *p = K_atm * pow(*rho, gam);
    *u = *p / (gam - 1.);
    return (*rho + *u + *p) / gtmp;
}
static double dWdvsq_calc2(double gam, double vsq, double rho, double p) {
    return (gam * (2. - gam) * p + (gam - 1.) * rho) / (2. * (gam - 1.) * (1. - vsq) * (1. - vsq));
}
static void func_1d_gnr2(double gam, const double x[1], double dx[1], double *f, double *df,
                         double Bsq, double Qtsq, double QdotBsq, double D, double K_atm) {
    double p, rho, u;
    double W = W_of_vsq2(gam, x[0], &p, &rho, &u, D, K_atm);
    double Wsq = W * W;
    double dWdvsq = dWdvsq_calc2(gam, x[0], rho, p);
    double fact_tmp = (Bsq + W);
    double resid = Qtsq - x[0] * fact_tmp * fact_tmp + QdotBsq * (Bsq + 2. * W) / Wsq;
    double jac = -fact_tmp * (fact_tmp + 2. * dWdvsq * (x[0] + QdotBsq / (W * Wsq)));
    dx[0] = -resid / jac;
    *f = 0.5 * resid * resid;
    *df = -2. * (*f);
}
static void validate_x2(double x[1], const double x0[1]) {
    double small = 1.e-10;
    x[0] = (x[0] >= 1.0) ? (0.5 * (x0[0] + 1.)) : x[0];
    x[0] = (x[0] < -small) ? (0.5 * x0[0]) : x[0];
    x[0] = fabs(x[0]);
}
static int newton_1d_vsq(double gam, double x[1], double Bsq, double Qtsq, double QdotBsq, double D,
                         double K_atm, double tolerance) {
    double f = 1., df = 1., dx[1], x_old[1], errx = 1., W = 0., W_old = 0., rho, p, u;
    int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
    x_old[0] = x[0];
    while (keep) {
        func_1d_gnr2(gam, x, dx, &f, &df, Bsq, Qtsq, QdotBsq, D, K_atm);
        errx = 0.;
        x_old[0] = x[0];
        x[0] += dx[0];
        validate_x2(x, x_old);
        W_old = W;
        W = W_of_vsq2(gam, x[0], &p, &rho, &u, D, K_atm);
        errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
        errx += (x[0] == 0.) ? fabs(x[0] - x_old[0]) : fabs((x[0] - x_old[0]) / x[0]);
        if ((fabs(errx) <= tolerance) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
        if (doing_extra == 1) i_extra++;
        if (((fabs(errx) <= tolerance) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
            keep = 0;
        n_iter++;
    }
    if ((isfinite(f) == 0) || (isfinite(df) == 0)) return 2;
    if (fabs(errx) > MY_MIN(tolerance, MIN_NEWT_TOL)) return 1;
    return 0;
}
static int body_1dvsq(double gam, const double *U, const double *gcov, const double *gcon, double *prim, double K_atm) {
    invq s;
    double utsq, x[1], p, rho0, u;
    inv_scalars(U, gcov, gcon, &s);
    if (guess_utsq(gcov, prim, &utsq)) return 2;
    double gammasq = 1. + utsq;
    x[0] = 1. - 1. / gammasq;
    int retval = newton_1d_vsq(gam, x, s.Bsq, s.Qtsq, s.QdotBsq, s.D, K_atm, NEWT_TOL);
    if (retval != 0) return retval * 100 + 1;
    double vsq = x[0];
    if ((vsq >= 1.) || (vsq < 0.)) return 4;
    double W = W_of_vsq2(gam, vsq, &p, &rho0, &u, s.D, K_atm);
    double gtmp = sqrt(1. - vsq);
    double gamma = 1. / gtmp;
    if (rho0 <= 0.) return 5;
    if (u <= 0.) return 6;
    prim[RHO] = rho0;
    prim[UU] = u;
    set_velocity(&s, gamma, W, prim);
    return 0;
}
int ho_utoprim_1dvsq2fix1(double gam, double *U, const double *gcov, const double *gcon, double gdet, double *prim) {
    double U_tmp[NPR], prim_tmp[5];
    int ret = inv_prologue(U, gdet, gcon, prim, U_tmp);
    if (ret) return ret;
    for (int i = 0; i < B1; i++) prim_tmp[i] = prim[i];
    double K_atm = U[KTOT] / U[RHO];
    ret = body_1dvsq(gam, U_tmp, gcov, gcon, prim_tmp, K_atm);
    if (ret == 0)
        for (int i = 0; i < B1; i++) prim[i] = prim_tmp[i];
    return ret;
}

/* Entropy-based 1D fallback in W with an inner rho solve (GPU_utoprim_1dfix1.h) */
static void func_gnr2_rho(double gam, const double x[1], double dx[1], double *f, double *df,
                          double D, double K_atm, double W_for_gnr2) {
    double A = D * D;
    double B0 = A * gam * K_atm;
    double B = B0 / (gam - 1.);
    double rho = x[0];
    double W = W_for_gnr2;
    double C = pow(rho, gam - 1.);
    double resid = rho * W - A - B * C;
    double jac = W - B0 * C / rho;
    dx[0] = -resid / jac;
    *f = 0.5 * resid * resid;
    *df = -2. * (*f);
}
static int gnr2(double gam, double x[1], double D, double K_atm, double W_for_gnr2) {
    double f = 1., df = 1., dx[1], x_old[1], errx = 1.;
    int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
    while (keep) {
        func_gnr2_rho(gam, x, dx, &f, &df, D, K_atm, W_for_gnr2);
        x_old[0] = x[0];
        x[0] += dx[0];
        x[0] = fabs(x[0]);
        errx = (x[0] == 0.) ? fabs(x[0] - x_old[0]) : fabs((x[0] - x_old[0]) / x[0]);
        /* the reference never enters its extra-iteration phase here */
        if (doing_extra == 1) i_extra++;
        if (((fabs(errx) <= 1.0e-15) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
            keep = 0;
        n_iter++;
    }
    if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x[0]) == 0)) return 2;
    if (fabs(errx) > 1.0e-10) return 1;
    return 0;
}
static void func_1d_orig1(double gam, const double x[1], double dx[1], double *f, double *df, double Bsq,
                          double Qtsq, double QdotBsq, double D, double K_atm, double rho_for_gnr2) {
    double x_rho[1], rho_g, W_for_gnr2 = x[0];
    int ntries = 0;
    rho_g = x_rho[0] = rho_for_gnr2;
    while ((gnr2(gam, x_rho, D, K_atm, W_for_gnr2)) && (ntries++ < 10)) {
        rho_g *= 10.;
        x_rho[0] = rho_g;
    }
    double rho = x_rho[0];
    double Dc = D;
    double t1 = Dc * Dc;
    double t2 = QdotBsq * t1;
    double t3 = t2 * Bsq;
    double t5 = Bsq * Bsq;
    double t8 = t1 * Bsq;
    double t10 = t1 * x[0];
    double t21 = x[0] * x[0];
    double t23 = rho * rho;
    double t26 = 1. / t1;
    double resid = (t3 + (2.0 * t2 + ((Qtsq - t5) * t1 + (-2.0 * t8 - t10) * x[0]) * x[0]) * x[0] + (t5 + (2.0 * Bsq + x[0]) * x[0]) * t21 * t23) * t26 / t21;
    double t29 = t1 * t1;
    double t30 = QdotBsq * t29;
    double t32 = gam * K_atm;
    double t33 = pow(rho, 1.0 * gam);
    double t34 = t32 * t33;
    double t38 = t23 * t33;
    double t51 = gam * t1 * K_atm * t33;
    double t67 = t21 * x[0];
    double jac = -2.0 * (t30 * Bsq * t34 + (t30 * t34 + ((-t38 * Bsq * t32 + Bsq * gam * t1 * K_atm * t33) * t1 + (-t38 * gam * K_atm + t51) * t1 * x[0]) * t21) * x[0] + ((-t3 + (-t2 + (-t8 - t10) * t21) * x[0]) * x[0] + (-t5 - Bsq * x[0]) * t67 * t23) * t23) * t26 / (t51 - x[0] * t23) / t67;
    dx[0] = -resid / jac;
    *f = 0.5 * resid * resid;
    *df = -2. * (*f);
}
static int newton_1d_w(double gam, double x[1], double Bsq, double Qtsq, double QdotBsq, double D,
                       double K_atm, double rho_for_gnr2, double tolerance) {
    double f = 1., df = 1., dx[1], x_old[1], errx = 1.;
    int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
    while (keep) {
        func_1d_orig1(gam, x, dx, &f, &df, Bsq, Qtsq, QdotBsq, D, K_atm, rho_for_gnr2);
        x_old[0] = x[0];
        x[0] += dx[0];
        int i_increase = 0;
        while (((x[0] * x[0] * x[0] * (x[0] + 2. * Bsq) - QdotBsq * (2. * x[0] + Bsq)) <= x[0] * x[0] * (Qtsq - Bsq * Bsq)) && (i_increase < 10)) {
            x[0] -= (1. * i_increase) * dx[0] / 10.;
            i_increase++;
        }
        x[0] = fabs(x[0]);
        errx = (x[0] == 0.) ? fabs(x[0] - x_old[0]) : fabs((x[0] - x_old[0]) / x[0]);
        if ((fabs(errx) <= tolerance) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
        if (doing_extra == 1) i_extra++;
        if (((fabs(errx) <= tolerance) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
            keep = 0;
        n_iter++;
    }
    if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x[0]) == 0)) return 2;
    if (fabs(errx) > MY_MIN(tolerance, MIN_NEWT_TOL)) return 1;
    return 0;
}
static int body_1dw(double gam, const double *U, const double *gcov, const double *gcon, double *prim, double K_atm) {
    invq s;
    double utsq, x[1];
    inv_scalars(U, gcov, gcon, &s);
    if (guess_utsq(gcov, prim, &utsq)) return 2;
    double gammasq = 1. + utsq;
    double gamma = sqrt(gammasq);
    double rho0 = s.D / gamma;
    double p = K_atm * pow(rho0, gam);
    double u = p / (gam - 1.);
    double w = rho0 + u + p;
    double W_last = w * gammasq;
    int i_increase = 0;
    while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <= W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) && (i_increase < 10)) {
        W_last *= 10.;
        i_increase++;
    }
    x[0] = W_last;
    int retval = newton_1d_w(gam, x, s.Bsq, s.Qtsq, s.QdotBsq, s.D, K_atm, rho0, NEWT_TOL);
    double W = x[0];
    if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
    if (W <= 0. || W > W_TOO_BIG) return 3;
    double vsq = vsq_calc(W, s.Bsq, s.Qtsq, s.QdotBsq);
    if (vsq >= 1.) return 4;
    double gtmp = sqrt(1. - vsq);
    gamma = 1. / gtmp;
    rho0 = s.D * gtmp;
    p = K_atm * pow(rho0, gam);
    u = p / (gam - 1.);
    if (rho0 <= 0.) return 5;
    if (u <= 0.) return 6;
    prim[RHO] = rho0;
    prim[UU] = u;
    set_velocity(&s, gamma, W, prim);
    return 0;
}
int ho_utoprim_1dfix1(double gam, double *U, const double *gcov, const double *gcon, double gdet, double *prim) {
    double U_tmp[NPR], prim_tmp[5];
    int ret = inv_prologue(U, gdet, gcon, prim, U_tmp);
    if (ret) return ret;
    for (int i = 0; i < B1; i++) prim_tmp[i] = prim[i];
    double K_atm = U[KTOT] / U[RHO];
    ret = body_1dw(gam, U_tmp, gcov, gcon, prim_tmp, K_atm);
    if (ret == 0)
        for (int i = 0; i < B1; i++) prim[i] = prim_tmp[i];
    return ret;
}

/* Newman & Hamlin (2014) inversion: fixed point on the pressure with a
 * closed-form cubic root for W and Aitken acceleration (GPU_utoprim_nm.h).
 * The reference keeps the pressure history in p_array[3] but indexes it up to
 * the iteration count (at most 30) when the Aitken step does not trigger;
 * here the history has room for every iteration, so those writes land in
 * their own slots instead of the neighbouring stack. */
static int nm_last_max_index;
/* largest pressure-history index the last ho_utoprim_nm call used; the
 * reference's 3-slot history is only well defined when it is <= 2 */
int ho_utoprim_nm_max_index(void) { return nm_last_max_index; }

int ho_utoprim_nm(double gam, double *U, const double *gcov, const double *gcon, double gdet, double *prim) {
    double U_tmp[NPR], pt[5];
    nm_last_max_index = 0;
    int ret = inv_prologue(U, gdet, gcon, prim, U_tmp);
    if (ret) return ret;
    for (int i = 0; i < B1; i++) pt[i] = prim[i];
    invq s;
    inv_scalars(U_tmp, gcov, gcon, &s);
    const double Bsq = s.Bsq, QdotBsq = s.QdotBsq, Qtsq = s.Qtsq, Qdotn = s.Qdotn;
    double a, d, z = 0., phi, R, Wsq, p_array[32], epsilon, p_old, p_new, vsq, w, gamma = 1., rho0 = 0., u = 0., errx;
    int iter = 0, iter_tot = 0, set_variables = 0;
    const double gamma_eos = gam;
    p_array[0] = (gamma_eos - 1.) * pt[UU];
    p_new = p_array[0];
    d = 0.5 * (Qtsq * Bsq - QdotBsq);
    if (d < 0.0) return 1;
    do {
        set_variables = 0;
        a = -Qdotn + p_new + 0.5 * Bsq;
        phi = acos(1. / a * sqrt((27. * d) / (4. * a)));
        epsilon = a / 3. - 2. / 3. * a * cos(2. / 3. * phi + 2. / 3. * 3.14159265358979323846);
        z = epsilon - Bsq;
        vsq = (Qtsq * z * z + QdotBsq * (Bsq + 2. * z)) / (z * z * pow(Bsq + z, 2.));
        if (fabs(vsq) < 1e-15) vsq = 0.0;
        if (fabs(vsq) >= 1.0) return 1;
        Wsq = 1. / (1. - vsq);
        w = z * (1. - vsq);
        gamma = 1. / sqrt(1. - vsq);
        rho0 = U_tmp[RHO] / gamma;
        u = (w - rho0) / gamma_eos;
        iter++;
        iter_tot++;
        if (iter > nm_last_max_index) nm_last_max_index = iter;
        p_array[iter] = (gamma_eos - 1.) * u;
        p_old = p_array[iter - 1];
        p_new = p_array[iter];
        if (iter >= 2) {
            R = (p_array[iter] - p_array[iter - 1]) / (p_array[iter - 1] - p_array[iter - 2]);
            if (R < 1. && R > 0.) {
                set_variables = 1;
                p_new = p_array[iter - 1] + (p_array[iter] - p_array[iter - 1]) / (1. - R);
                p_old = p_array[iter];
                iter = 0;
                p_array[iter] = p_new;
            }
        }
        errx = fabs(p_new - p_old) / fabs(p_new + p_old);
    } while (errx > NEWT_TOL && iter_tot < 30);
    if (fabs(errx) > MY_MIN(NEWT_TOL, MIN_NEWT_TOL)) return 1;
    if (set_variables == 1) {
        a = -Qdotn + p_new + 0.5 * Bsq;
        phi = acos(1. / a * sqrt((27. * d) / (4. * a)));
        epsilon = a / 3. - 2. / 3. * a * cos(2. / 3. * phi + 2. / 3. * 3.14159265358979323846);
        z = epsilon - Bsq;
        vsq = (Qtsq * z * z + QdotBsq * (Bsq + 2. * z)) / (z * z * pow(Bsq + z, 2.));
        Wsq = 1. / (1. - vsq);
        w = z / Wsq;
        if (vsq >= 1.0 || vsq < 0. || z <= 0. || z > 1.e20 || !isfinite(vsq) || !isfinite(z)) return 4;
        gamma = sqrt(Wsq);
        rho0 = U_tmp[RHO] / gamma;
        u = (w - rho0) / gamma_eos;
        p_new = (gamma_eos - 1.) * u;
    }
    if (rho0 < 0.0) return 5;
    if (p_new < 0.0) return 6;
    pt[RHO] = rho0;
    pt[UU] = u;
    for (int i = 1; i < 4; i++) {
        double Qtcon = s.Qcon[i] + s.ncon[i] * s.Qdotn;
        pt[U1 + i - 1] = gamma / (z + Bsq) * (Qtcon + s.QdotB * s.Bcon[i] / z);
    }
    for (int i = 0; i < B1; i++) prim[i] = pt[i];
    return 0;
}

/* --------------------------------------------------------------- floors -- */
/* fixup_cell (GPU_fixup.h:989-1800) with its body as written for an ideal
 * gas, DRIFT_FLOOR 1, no neutron star, radiation or EOS table. The reference
 * compiles that body out (#if 0, GPU_fixup.h:1007) and leaves only the
 * `r < radfix_dens` reset, dead with radfix_dens = 0 (config.h:40); the
 * product offers the body as an opt-in. Floor constants of the torus build
 * (config.h:274-287). */
#define RHOMINLIMIT 1.e-20
#define UUMINLIMIT 1.e-20
#define BSQORHOMAX 25.
#define BSQOUMAX 750.
#define UORHOMAX 150.

/* ut_calc_3vel (GPU_phys_mhd.h:18-31) */
static void ut_calc_3vel(const double *vcon, const geo *gm, double *ut) {
    const double *g = gm->gcov;
    double AA = g[0];
    double BB = 2. * (g[1] * vcon[1] + g[2] * vcon[2] + g[3] * vcon[3]);
    double CC = g[4] * vcon[1] * vcon[1] + g[7] * vcon[2] * vcon[2] + g[9] * vcon[3] * vcon[3]
              + 2. * (g[5] * vcon[1] * vcon[2] + g[6] * vcon[1] * vcon[3] + g[8] * vcon[2] * vcon[3]);
    double DD = -1. / (AA + BB + CC);
    double one_over_alpha_sq = -gm->gcon[0];
    if (DD < one_over_alpha_sq) DD = one_over_alpha_sq;
    *ut = sqrt(DD);
}

/* ucon_to_utcon (GPU_phys_mhd.h:3-15) */
static void ucon_to_utcon(const double *ucon, const geo *gm, double *utcon) {
    double alpha = 1. / sqrt(-gm->gcon[0]);
    double beta[4];
    for (int j = 1; j < 4; j++) beta[j] = gm->gcon[j] * alpha * alpha;
    double gamma = alpha * ucon[0];
    utcon[0] = 0;
    for (int j = 1; j < 4; j++) utcon[j] = ucon[j] + gamma * beta[j] / alpha;
}

static int fixup_cell(double gam, double *pf, const geo *gm) {
    cstate q;
    double pf_prefloor[NPR], ucondr[4], Bcon[4], Bcov[4], vcon[4], ucon[4], utcon[4];
    double rhoflr = RHOMINLIMIT, uuflr = UUMINLIMIT;
    get_state(pf, gm, &q);
    double bsq = dot4(q.bcon, q.bcov);
    double u = pf[UU];
    for (int k = 0; k < NPR; k++) pf_prefloor[k] = pf[k];
    if (rhoflr < bsq / BSQORHOMAX) rhoflr = bsq / (BSQORHOMAX);
    if (uuflr < bsq / BSQOUMAX) uuflr = bsq / (BSQOUMAX);
    if (rhoflr < u / UORHOMAX) rhoflr = u / (UORHOMAX);
    if (rhoflr < RHOMINLIMIT) rhoflr = RHOMINLIMIT;
    if (uuflr < UUMINLIMIT) uuflr = UUMINLIMIT;
    int dofloor = 0;
    if (pf[RHO] < rhoflr) { pf[RHO] = rhoflr; dofloor = 1; }
    if (u < uuflr) { pf[UU] = uuflr; u = uuflr; dofloor = 1; }
    double trans = 10. * bsq / MY_MIN(pf[RHO], u) - 1.;
    if (dofloor && trans > 0.) {
        if (trans > 1.) trans = 1.;
        double betapar = -q.bcon[0] / ((bsq + SMALL) * q.ucon[0]);
        double betasq = betapar * betapar * bsq;
        double betasqmax = 1. - 1. / (GAMMAMAX * GAMMAMAX);
        if (betasq > betasqmax) betasq = betasqmax;
        double gamma = 1. / sqrt(1 - betasq);
        for (int m = 0; m < 4; m++) ucondr[m] = gamma * (q.ucon[m] + betapar * q.bcon[m]);
        Bcon[0] = 0.;
        for (int m = 1; m < 4; m++) Bcon[m] = pf[B1 - 1 + m];
        lower4(Bcon, gm->gcov, Bcov);
        double udotB = dot4(q.ucon, Bcov);
        double Bsq = dot4(Bcon, Bcov);
        double B = sqrt(Bsq);
        double wold = pf_prefloor[RHO] + pf_prefloor[UU] * gam;
        double QdotB = udotB * wold * q.ucon[0];
        double wnew = pf[RHO] + pf[UU] * gam;
        double x = 2. * QdotB / (B * wnew * ucondr[0] + SMALL);
        double vpar = x / (ucondr[0] * (1. + sqrt(1. + x * x)));
        double one_over_ucondr_t = 1. / ucondr[0];
        vcon[0] = 1.;
        for (int m = 1; m < 4; m++) vcon[m] = vpar * Bcon[m] / (B + SMALL) + ucondr[m] * one_over_ucondr_t;
        double ut;
        ut_calc_3vel(vcon, gm, &ut);
        for (int m = 0; m < 4; m++) ucon[m] = ut * vcon[m];
        ucon_to_utcon(ucon, gm, utcon);
        for (int m = 1; m < 4; m++) pf[m + UU] = utcon[m] * trans + pf_prefloor[m + UU] * (1. - trans);
    }
    double gamma;
    if (gamma_calc(pf, gm, &gamma)) return 4;
    if (gamma > GAMMAMAX) {
        double f = sqrt((GAMMAMAX * GAMMAMAX - 1.) / (gamma * gamma - 1.));
        pf[U1] *= f;
        pf[U2] *= f;
        pf[U3] *= f;
    }
    return 0;
}

int ho_fixup_cell(double gam, double *pf, const double *gcov10, const double *gcon10, double gdet) {
    geo gm;
    for (int k = 0; k < 10; k++) { gm.gcov[k] = gcov10[k]; gm.gcon[k] = gcon10[k]; }
    gm.g = gdet;
    return fixup_cell(gam, pf, &gm);
}

/* fixuputoprim (GPU_fixup.h:735-800) for one failed zone: the floor state
 * with zero velocity, passed through the floors when they are on */
static void reset_failed(double gam, double *pf, const geo *gm, int floors) {
    pf[RHO] = RHOMINLIMIT;
    pf[UU] = UUMINLIMIT;
    pf[U1] = 0.0;
    pf[U2] = 0.0;
    pf[U3] = 0.0;
    if (floors) (void)fixup_cell(gam, pf, gm);
}

/* fixup_utoprim (fixup.c:764-827): each failed active zone, in (i, j, z)
 * order, takes the average of the first usable stencil of good neighbours
 * (the 8 neighbours in the x1-x2 plane numbered 1 2 3 / 8 x 4 / 7 6 5 with
 * 1 at (i-1, j+1), plus 9 = z+1 and 10 = z-1); a repaired zone counts as good
 * for the zones after it. Only RHO..U3 are set. The two-point x1 and x2
 * stencils are selected by the flags of the other direction, as written
 * there (AVG2_X1 when 2 and 6 are good, AVG2_X2 when 4 and 8 are). */
void ho_fixup_utoprim(const ho_grid *g, double *pv, int *pflag, int *failimage) {
    dims d = mkdims(g);
    long ks = d.ks;
    long sj = d.G3, si = (long)d.G2 * d.G3, sz = d.d3;
    for (int i = d.ng1; i < d.ng1 + d.n1; i++)
        for (int j = d.ng2; j < d.ng2 + d.n2; j++)
            for (int z = d.ng3; z < d.ng3 + d.n3; z++) {
                long c = cix(&d, i, j, z);
                if (pflag[c] == 0) continue;
                int pf[11];
                pf[1] = !pflag[c - si + sj]; pf[2] = !pflag[c + sj]; pf[3] = !pflag[c + si + sj];
                pf[8] = !pflag[c - si];                           pf[4] = !pflag[c + si];
                pf[7] = !pflag[c - si - sj]; pf[6] = !pflag[c - sj]; pf[5] = !pflag[c + si - sj];
                pf[9] = !pflag[c + sz]; pf[10] = !pflag[c - sz];
#define P(o) pv[k * ks + c + (o)]
                if (pf[2] && pf[4] && pf[6] && pf[8] && pf[9] && pf[10]) {
                    for (int k = 0; k < B1; k++)
                        P(0) = 1. / 6. * (P(sj) + P(-sj) + P(-si) + P(si) + P(1) + P(-1));
                } else if (pf[1] && pf[3] && pf[5] && pf[7] && pf[9] && pf[10]) {
                    for (int k = 0; k < B1; k++)
                        P(0) = 1. / 6. * (P(si + sj) + P(si - sj) + P(-si + sj) + P(-si - sj) + P(1) + P(-1));
                } else if (pf[2] && pf[4] && pf[6] && pf[8]) {
                    for (int k = 0; k < B1; k++) P(0) = 0.25 * (P(sj) + P(-sj) + P(-si) + P(si));
                } else if (pf[1] && pf[3] && pf[5] && pf[7]) {
                    for (int k = 0; k < B1; k++) P(0) = 0.25 * (P(si + sj) + P(si - sj) + P(-si + sj) + P(-si - sj));
                } else if (pf[2] && pf[6]) {
                    for (int k = 0; k < B1; k++) P(0) = 0.5 * (P(-si) + P(si));
                } else if (pf[4] && pf[8]) {
                    for (int k = 0; k < B1; k++) P(0) = 0.5 * (P(-sj) + P(sj));
                } else if (pf[9] && pf[10]) {
                    for (int k = 0; k < B1; k++) P(0) = 0.5 * (P(-1) + P(1));
                } else {
                    failimage[4 * ks + c]++;
                    for (int k = RHO; k <= UU; k++)
                        P(0) = 0.5 * (0.25 * (P(sj) + P(-sj) + P(-si) + P(si))
                                      + 0.25 * (P(si + sj) + P(si - sj) + P(-si + sj) + P(-si - sj)));
                    pv[U1 * ks + c] = pv[U2 * ks + c] = pv[U3 * ks + c] = 0.;
                }
#undef P
                pflag[c] = 0;
            }
}

/* --------------------------------------------------------------- update -- */
/* fixup kernel (GPU_fixup.h:5-424): cache U(p^n) on the half step, apply the
 * flux divergence and geometric source, rebuild U[B] from the new face field,
 * invert with the Noble 2D scheme and the entropy fallbacks. The floor routine
 * fixup_cell (GPU_fixup.h:989) is compiled out in the reference; with
 * g->floors it runs here as written, and g->repair adds the failed-zone
 * repair of fixuputoprim (1) or fixup_utoprim (2) after the inversion. */
static void update(const ho_grid *g, const dims *d, const ho_geom *m, ho_state *s, int full, double Dt) {
    long ks = d->ks;
    long isize = (long)d->G2 * d->G3;
    const double *pin = s->p;           /* p^n, guess for the half step */
    const double *pb = full ? s->ph : s->p;
    double *pout = full ? s->p : s->ph;
    const double *psf = full ? s->ps : s->psh;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int i = d->ng1; i < d->ng1 + d->n1; i++)
        for (int j = d->ng2; j < d->ng2 + d->n2; j++)
            for (int z = d->ng3; z < d->ng3 + d->n3; z++) {
                long c = cix(d, i, j, z);
                long gi = gix(d, i, j);
                geo gm;
                cstate q;
                double pf[NPR], U[NPR], dU[NPR];
                load_geo(d, m, i, j, CENT, &gm);
                if (!full) {
                    for (int k = 0; k < NPR; k++) { pf[k] = 0.0; pf[k] += (1.0 / ((double)1)) * pin[k * ks + c]; }
                    get_state(pf, &gm, &q);
                    double vdummy;
                    primtoflux(g->gam, pf, &q, 0, &gm, U, &vdummy, &vdummy);
                    for (int k = 0; k < NPR; k++) s->U[k * ks + c] = U[k];
                } else {
                    for (int k = 0; k < NPR; k++) U[k] = s->U[k * ks + c];
                    for (int k = 0; k < NPR; k++) { pf[k] = 0.0; pf[k] += (1.0 / ((double)1)) * pb[k * ks + c]; }
                    get_state(pf, &gm, &q);
                }
                for (int k = 0; k < NPR; k++) {
                    if (d->ng1 > 0) U[k] -= Dt * (s->F1[k * ks + c + isize] - s->F1[k * ks + c]) / (g->dx1 * (double)1);
                    if (d->ng2 > 0) U[k] -= Dt * (s->F2[k * ks + c + d->G3] - s->F2[k * ks + c]) / (g->dx2 * (double)1);
                    if (d->ng3 > 0) U[k] -= Dt * (s->F3[k * ks + c + 1] - s->F3[k * ks + c]) / (g->dx3 * (double)1);
                }
                source(g->gam, pf, &gm, d, m, i, j, dU, &q);
                for (int k = 0; k < NPR; k++) U[k] += Dt * (dU[k]);
                U[B1] = 0.0;
                U[B2] = 0.0;
                U[B1] += (psf[0 * ks + c] * m->gdet[FACE1 * d->gs + gi] + psf[0 * ks + c + isize] * m->gdet[FACE1 * d->gs + gix(d, i + d->d1, j)]) / (2.0 * (double)1);
                U[B2] += (psf[1 * ks + c] * m->gdet[FACE2 * d->gs + gi] + psf[1 * ks + c + d->G3] * m->gdet[FACE2 * d->gs + gix(d, i, j + d->d2)]) / (2.0 * (double)1);
                if (d->ng3 > 0)
                    U[B3] = (psf[2 * ks + c] * m->gdet[FACE3 * d->gs + gi] + psf[2 * ks + c + 1 * d->d3] * m->gdet[FACE3 * d->gs + gi]) / 2.0;
                int flag = g->inversion == 1 ? ho_utoprim_nm(g->gam, U, gm.gcov, gm.gcon, gm.g, pf)
                                             : ho_utoprim_2d(g->gam, U, gm.gcov, gm.gcon, gm.g, pf);
                if (flag) {
                    s->failimage[c]++;
                    flag = ho_utoprim_1dvsq2fix1(g->gam, U, gm.gcov, gm.gcon, gm.g, pf);
                    if (flag) {
                        s->failimage[1 * ks + c]++;
                        flag = ho_utoprim_1dfix1(g->gam, U, gm.gcov, gm.gcon, gm.g, pf);
                        if (flag) s->failimage[2 * ks + c]++;
                    }
                }
                if (g->floors && fixup_cell(g->gam, pf, &gm)) {
                    flag = -333;
                    s->failimage[3 * ks + c]++;
                }
                if (g->repair == 1 && flag != 0) reset_failed(g->gam, pf, &gm, g->floors);
                s->pflag[c] = flag;
                for (int k = 0; k < NPR; k++) pout[k * ks + c] = pf[k];
            }
    if (g->repair == 2) ho_fixup_utoprim(g, pout, s->pflag, s->failimage);
}

/* ---------------------------------------------------------------- stage -- */
void ho_stage(const ho_grid *g, const ho_geom *m, ho_state *s, int full, double Dt, double dt,
              int calc_dt, double *dtdir) {
    dims d = mkdims(g);
    const double *pin = full ? s->ph : s->p;
    const double *psin = full ? s->psh : s->ps;
    double dtd;
    /* advance_GPU order: x3, x2, x1 fluxes */
    if (d.ng3 > 0) { fluxes(g, &d, m, pin, psin, 3, s->F3, &dtd); if (calc_dt) dtdir[3] = dtd; }
    else if (calc_dt) dtdir[3] = 1e9;
    fluxes(g, &d, m, pin, psin, 2, s->F2, &dtd);
    if (calc_dt) dtdir[2] = dtd;
    fluxes(g, &d, m, pin, psin, 1, s->F1, &dtd);
    if (calc_dt) dtdir[1] = dtd;
    if (g->bc2 == HO_BC_POLE_REFL) fix_flux(g, &d, s->F1, s->F2, s->F3);
    emf_centre(&d, m, pin, s->E_cent);
    emf_edges(g, &d, s->E_cent, s->F1, s->F2, s->F3, s->emf);
    if (g->bc2 == HO_BC_POLE_TRANS) emf_pole_average(g, &d, s->emf, dt);
    face_update(g, &d, m, s->ps, full ? s->ps : s->psh, s->emf, Dt);
    update(g, &d, m, s, full, Dt);
}

/* ----------------------------------------------------------- boundaries -- */
/* inflow_check (GPU_bounds.h:1368-1410): zero the x1 four-velocity of a ghost
 * cell whose flow points into the domain (type 0: u^1 > 0, type 1: u^1 < 0) */
static void inflow_check(double *pr, const geo *gm, int type) {
    double ucon[4], gamma;
    ucon_calc(pr, gm, ucon);
    if (((ucon[1] > 0.) && (type == 0)) || ((ucon[1] < 0.) && (type == 1))) {
        gamma_calc(pr, gm, &gamma);
        pr[U1] /= gamma;
        pr[U2] /= gamma;
        pr[U3] /= gamma;
        double alpha = 1. / sqrt(-gm->gcon[0]);
        double beta1 = gm->gcon[1] * alpha * alpha;
        pr[U1] = beta1 / alpha;
        double vsq = gm->gcov[4] * pr[U1] * pr[U1];
        vsq += 2. * gm->gcov[5] * pr[U2] * pr[U1];
        vsq += 2. * gm->gcov[6] * pr[U3] * pr[U1];
        vsq += gm->gcov[7] * pr[U2] * pr[U2];
        vsq += 2 * gm->gcov[8] * pr[U3] * pr[U2];
        vsq += gm->gcov[9] * pr[U3] * pr[U3];
        vsq = MY_MAX(1.e-13, vsq);
        if (vsq >= 1.) vsq = 1. - 1. / (GAMMAMAX * GAMMAMAX);
        gamma = 1. / sqrt(1. - vsq);
        pr[U1] *= gamma;
        pr[U2] *= gamma;
        pr[U3] *= gamma;
    }
}

static void copy_cell(const dims *d, double *pv, long dst, long src) {
    for (int k = 0; k < NPR; k++) pv[k * d->ks + dst] = pv[k * d->ks + src];
}

/*
 * Ghost fill. Order follows bound_prim (bounds.c:11-131): x1 first over every
 * (j, z), then the x3 periodic exchange, then the x2 edges.
 *  x1 OUTFLOW: copy the edge cell, then inflow_check with the ghost cell's own
 *     metric (type 0 at the inner edge, type 1 at the outer edge); copy face
 *     B^2, B^3 (GPU_bounds.h:3-178 without its neutron-star constants).
 *  x2 POLE_TRANS: mirror across the axis with a half-turn in phi, flip u^2,
 *     u^3, B^2, B^3 (boundprim2_trans, GPU_bounds.h:510-606).
 *  x2 POLE_REFL: POLEFIX velocity taper of the first two rows, mirror copy,
 *     flip u^2 and B^2 (boundprim2_reflective, GPU_bounds.h:305-508).
 *  PERIODIC: copy from the opposite edge, all planes and the face field.
 */
void ho_bound_dim(const ho_grid *g, const ho_geom *m, double *pv, double *ps, int dim) {
    dims d = mkdims(g);
    long ks = d.ks;
    /* x1 */
    if (dim == 1 && d.d1) {
        for (int j = 0; j < d.G2; j++)
            for (int z = 0; z < d.G3; z++)
                for (int t = 0; t < d.ng1; t++) {
                    int ilo = t, ihi = d.n1 + d.ng1 + t;
                    if (g->bc1 == HO_BC_PERIODIC) {
                        copy_cell(&d, pv, cix(&d, ilo, j, z), cix(&d, ilo + d.n1, j, z));
                        copy_cell(&d, pv, cix(&d, ihi, j, z), cix(&d, ihi - d.n1, j, z));
                        for (int c = 0; c < 3; c++) {
                            ps[c * ks + cix(&d, ilo, j, z)] = ps[c * ks + cix(&d, ilo + d.n1, j, z)];
                            ps[c * ks + cix(&d, ihi, j, z)] = ps[c * ks + cix(&d, ihi - d.n1, j, z)];
                        }
                    } else {
                        geo gm;
                        double pr[NPR];
                        long src, dst;
                        if (!(g->halo & 1)) {
                            src = cix(&d, d.ng1, j, z);
                            dst = cix(&d, ilo, j, z);
                            for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + src];
                            load_geo(&d, m, ilo, j, CENT, &gm);
                            inflow_check(pr, &gm, 0);
                            for (int k = 0; k < NPR; k++) pv[k * ks + dst] = pr[k];
                            ps[1 * ks + dst] = ps[1 * ks + src];
                            ps[2 * ks + dst] = ps[2 * ks + src];
                        }
                        if (!(g->halo & 2)) {
                            src = cix(&d, d.n1 + d.ng1 - 1, j, z);
                            dst = cix(&d, ihi, j, z);
                            for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + src];
                            load_geo(&d, m, ihi, j, CENT, &gm);
                            inflow_check(pr, &gm, 1);
                            for (int k = 0; k < NPR; k++) pv[k * ks + dst] = pr[k];
                            ps[1 * ks + dst] = ps[1 * ks + src];
                            ps[2 * ks + dst] = ps[2 * ks + src];
                        }
                    }
                }
    }
    /* x3: periodic */
    if (dim == 3 && d.d3) {
        for (int i = 0; i < d.G1; i++)
            for (int j = 0; j < d.G2; j++)
                for (int t = 0; t < d.ng3; t++) {
                    long lo = cix(&d, i, j, t), lo_src = cix(&d, i, j, t + d.n3);
                    long hi = cix(&d, i, j, d.n3 + d.ng3 + t), hi_src = cix(&d, i, j, d.ng3 + t);
                    copy_cell(&d, pv, lo, lo_src);
                    copy_cell(&d, pv, hi, hi_src);
                    for (int c = 0; c < 3; c++) {
                        ps[c * ks + lo] = ps[c * ks + lo_src];
                        ps[c * ks + hi] = ps[c * ks + hi_src];
                    }
                }
    }
    /* x2 */
    if (dim == 2 && d.d2) {
        int n2 = d.n2, ng = d.ng2;
        for (int i = 0; i < d.G1; i++)
            for (int z = 0; z < d.G3; z++) {
                if (g->bc2 == HO_BC_PERIODIC) {
                    for (int t = 0; t < ng; t++) {
                        long lo = cix(&d, i, t, z), lo_src = cix(&d, i, t + n2, z);
                        long hi = cix(&d, i, n2 + ng + t, z), hi_src = cix(&d, i, ng + t, z);
                        copy_cell(&d, pv, lo, lo_src);
                        copy_cell(&d, pv, hi, hi_src);
                        for (int c = 0; c < 3; c++) {
                            ps[c * ks + lo] = ps[c * ks + lo_src];
                            ps[c * ks + hi] = ps[c * ks + hi_src];
                        }
                    }
                } else if (g->bc2 == HO_BC_POLE_TRANS) {
                    int zs = d.d3 ? (z - d.ng3 + d.n3 / 2) % d.n3 + d.ng3 : z;
                    if (g->pole1)
                        for (int jj = -ng; jj < 0; jj++) {
                            long dst = cix(&d, i, jj + ng, z), src = cix(&d, i, -jj - 1 + ng, zs);
                            copy_cell(&d, pv, dst, src);
                            pv[U2 * ks + dst] *= -1.0;
                            pv[U3 * ks + dst] *= -1.0;
                            pv[B2 * ks + dst] *= -1.0;
                            pv[B3 * ks + dst] *= -1.0;
                            ps[0 * ks + dst] = ps[0 * ks + src];
                            ps[2 * ks + dst] = -ps[2 * ks + src];
                        }
                    if (g->pole2)
                        for (int jj = n2; jj < n2 + ng; jj++) {
                            long dst = cix(&d, i, jj + ng, z), src = cix(&d, i, 2 * n2 - jj - 1 + ng, zs);
                            copy_cell(&d, pv, dst, src);
                            pv[U2 * ks + dst] *= -1.0;
                            pv[U3 * ks + dst] *= -1.0;
                            pv[B2 * ks + dst] *= -1.0;
                            pv[B3 * ks + dst] *= -1.0;
                            ps[0 * ks + dst] = ps[0 * ks + src];
                            ps[2 * ks + dst] = -ps[2 * ks + src];
                        }
                } else if (g->bc2 == HO_BC_POLE_REFL) {
                    const int jref = 2; /* POLEFIX, config.h:490 */
                    if (g->pole1) {
                        for (int jj = 0; jj < jref; jj++) {
                            long c = cix(&d, i, jj + ng, z), r = cix(&d, i, jref + ng, z);
                            pv[U2 * ks + c] = (jj + 0.5) / (jref + 0.5) * pv[U2 * ks + r];
                            pv[RHO * ks + c] = pv[RHO * ks + r];
                            pv[UU * ks + c] = pv[UU * ks + r];
                            pv[U1 * ks + c] = pv[U1 * ks + r];
                            pv[U3 * ks + c] = pv[U3 * ks + r];
                            pv[KTOT * ks + c] = pv[KTOT * ks + r];
                        }
                        for (int t = 1; t <= ng; t++) copy_cell(&d, pv, cix(&d, i, ng - t, z), cix(&d, i, ng + t - 1, z));
                        for (int jj = 0; jj < ng; jj++) {
                            pv[U2 * ks + cix(&d, i, jj, z)] *= -1.;
                            pv[B2 * ks + cix(&d, i, jj, z)] *= -1.;
                        }
                        for (int t = 1; t <= ng; t++) {
                            ps[0 * ks + cix(&d, i, ng - t, z)] = ps[0 * ks + cix(&d, i, ng + t - 1, z)];
                            ps[2 * ks + cix(&d, i, ng - t, z)] = ps[2 * ks + cix(&d, i, ng + t - 1, z)];
                        }
                    }
                    if (g->pole2) {
                        for (int jj = 0; jj < jref; jj++) {
                            long c = cix(&d, i, n2 + ng - 1 - jj, z), r = cix(&d, i, n2 + ng - 1 - jref, z);
                            pv[U2 * ks + c] = (jj + 0.5) / (jref + 0.5) * pv[U2 * ks + r];
                            pv[RHO * ks + c] = pv[RHO * ks + r];
                            pv[UU * ks + c] = pv[UU * ks + r];
                            pv[U1 * ks + c] = pv[U1 * ks + r];
                            pv[U3 * ks + c] = pv[U3 * ks + r];
                            pv[KTOT * ks + c] = pv[KTOT * ks + r];
                        }
                        for (int t = 0; t < ng; t++) copy_cell(&d, pv, cix(&d, i, n2 + ng + t, z), cix(&d, i, n2 + ng - 1 - t, z));
                        for (int jj = n2 + ng; jj < n2 + 2 * ng; jj++) {
                            pv[U2 * ks + cix(&d, i, jj, z)] *= -1.;
                            pv[B2 * ks + cix(&d, i, jj, z)] *= -1.;
                        }
                        for (int t = 0; t < ng; t++) {
                            ps[0 * ks + cix(&d, i, n2 + ng + t, z)] = ps[0 * ks + cix(&d, i, n2 + ng - 1 - t, z)];
                            ps[2 * ks + cix(&d, i, n2 + ng + t, z)] = ps[2 * ks + cix(&d, i, n2 + ng - 1 - t, z)];
                        }
                    }
                }
                /* HO_BC_OUTFLOW in x2: plain copy of the edge row (not on an x2
                 * side shared with a neighbour block: halo bits 2, 3) */
                else {
                    for (int t = 0; t < ng; t++) {
                        if (!(g->halo & 4)) {
                            copy_cell(&d, pv, cix(&d, i, t, z), cix(&d, i, ng, z));
                            ps[0 * ks + cix(&d, i, t, z)] = ps[0 * ks + cix(&d, i, ng, z)];
                            ps[2 * ks + cix(&d, i, t, z)] = ps[2 * ks + cix(&d, i, ng, z)];
                        }
                        if (!(g->halo & 8)) {
                            copy_cell(&d, pv, cix(&d, i, n2 + ng + t, z), cix(&d, i, n2 + ng - 1, z));
                            ps[0 * ks + cix(&d, i, n2 + ng + t, z)] = ps[0 * ks + cix(&d, i, n2 + ng - 1, z)];
                            ps[2 * ks + cix(&d, i, n2 + ng + t, z)] = ps[2 * ks + cix(&d, i, n2 + ng - 1, z)];
                        }
                    }
                }
            }
    }
}

void ho_bound(const ho_grid *g, const ho_geom *m, double *pv, double *ps) {
    ho_bound_dim(g, m, pv, ps, 1);
    ho_bound_dim(g, m, pv, ps, 3);
    ho_bound_dim(g, m, pv, ps, 2);
}

/* divb_calc (diag.c:153-199), staggered-field definition, max over active cells */
double ho_divb_max(const ho_grid *g, const ho_geom *m, const double *ps) {
    dims d = mkdims(g);
    long ks = d.ks;
    double mx = 0.;
    for (int i = d.ng1; i < d.ng1 + d.n1; i++)
        for (int j = d.ng2; j < d.ng2 + d.n2; j++)
            for (int z = d.ng3; z < d.ng3 + d.n3; z++) {
                double divb = 0.0;
                long c = cix(&d, i, j, z);
                if (d.d1) divb += 0.25 * (ps[0 * ks + c + (long)d.G2 * d.G3] * m->gdet[FACE1 * d.gs + gix(&d, i + 1, j)] - ps[0 * ks + c] * m->gdet[FACE1 * d.gs + gix(&d, i, j)]) / g->dx1;
                if (d.d2) divb += 0.25 * (ps[1 * ks + c + d.G3] * m->gdet[FACE2 * d.gs + gix(&d, i, j + 1)] - ps[1 * ks + c] * m->gdet[FACE2 * d.gs + gix(&d, i, j)]) / g->dx2;
                if (d.d3) divb += 0.25 * (ps[2 * ks + c + 1] * m->gdet[FACE3 * d.gs + gix(&d, i, j)] - ps[2 * ks + c] * m->gdet[FACE3 * d.gs + gix(&d, i, j)]) / g->dx3;
                divb = fabs(divb);
                if (divb > mx) mx = divb;
            }
    return mx;
}
