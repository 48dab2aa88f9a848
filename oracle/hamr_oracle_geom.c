/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Host metric tables of one uniform block, restated in plain C from the
 * reference so that the oracle (and the CPU arm of the benchmark) can set up
 * a problem without the product library. Same table layout as the device
 * tables (GPU_main.cu:139-300): gcov/gcon plane (s*5 + loc), gdet plane loc,
 * conn plane (s*4 + l), each indexed (i*G2 + j) with plane stride gsize.
 *
 * Followed, in their operation order (bit-identical tables are the point):
 *   coord()                       coord.c:26-109 (SPHERICAL_GR ghost mirror)
 *   vofx_matthewcoords, bl_coord  coord.c:111-211 (uniform theta map)
 *   gcov_func_spherical           metric.c:13-271 (Kerr-Schild, no tilt)
 *   gcov_func_cartesian           metric.c:273 (Minkowski)
 *   dxdxp_func                    metric.c:501-519 (central differences)
 *   gdet_func, gcon_func          metric.c:392-414
 *   conn_func                     metric.c:427-464 (central differences)
 *   LU_decompose, LU_substitution, invert_matrix  lu.c
 *   set_grid loop                 main.c:380-455
 */
#include <float.h>
#include <math.h>
#include <string.h>

#include "hamr_oracle.h"

#define GD 4
enum { GL_FACE1 = 0, GL_FACE2 = 1, GL_CORN = 2, GL_CENT = 3, GL_FACE3 = 4 };

/* default grid map (config.h:555-568) */
static const double G_RADEXP = 1.0, G_RTRANS = 5000000., G_RB = 0.;
static const double G_BRAVO = 0.0, G_TANGO = 1.0, G_CHARLIE = 0.0, G_DELTA = 3.0;
static const double G_SINGSMALL = 1.E-20;

typedef struct {
    int cart;    /* 1: Minkowski in Cartesian code coordinates */
    double a;    /* spin */
} gmap;

/* vofx_matthewcoords + the COORDSINGFIX clamp of bl_coord */
static void g_bl(const gmap *m, const double *X, double *r, double *th, double *ph) {
    double V[GD];
    if (m->cart) {
        *r = sqrt(X[1] * X[1] + X[2] * X[2] + X[3] * X[3]);
        *th = 0.;
        *ph = 0.;
        return;
    }
    V[0] = X[0];
    const double Xt = pow(log(G_RTRANS - G_RB), 1. / G_RADEXP);
    if (X[1] < Xt)
        V[1] = exp(pow(X[1], G_RADEXP)) + G_RB;
    else if (X[1] >= Xt && X[1] < 1.01 * Xt)
        V[1] = 10. * (X[1] / Xt - 1.) * ((X[1] - Xt) * G_RADEXP * exp(pow(Xt, G_RADEXP)) * pow(Xt, -1. + G_RADEXP) + G_RTRANS) +
               (1. - 10. * (X[1] / Xt - 1.)) * (exp(pow(X[1], G_RADEXP)) + G_RB);
    else
        V[1] = (X[1] - Xt) * G_RADEXP * exp(pow(Xt, G_RADEXP)) * pow(Xt, -1. + G_RADEXP) + G_RTRANS;
    const double A1 = 1. / (1. + pow(G_CHARLIE * (log(V[1]) / log(10.)), G_DELTA));
    const double A2 = G_BRAVO * (log(V[1]) / log(10.)) + G_TANGO;
    const double A3 = pow(0.5, 1. - A2);
    double sgn = 1.;
    const double X2 = (X[2] + 1.0) / 2.0;
    double Xc = sqrt(pow(X2, 2.));
    if (X2 < 0.0) sgn = -1.;
    if (X2 > 1.0) {
        sgn = -1.;
        Xc = 2. - Xc;
    }
    if (X2 >= 0.5) {
        Xc = 1. - Xc;
        V[2] = M_PI - sgn * (A1 * M_PI * Xc + M_PI * (1. - A1) * (A3 * pow(Xc, A2) + 0.50 / M_PI * sin(M_PI + 2. * M_PI * (A3 * pow(Xc, A2)))));
    } else {
        V[2] = sgn * (A1 * M_PI * Xc + M_PI * (1. - A1) * (A3 * pow(Xc, A2) + 0.50 / M_PI * sin(M_PI + 2. * M_PI * (A3 * pow(Xc, A2)))));
    }
    V[3] = X[3];
    if (fabs(V[2]) < G_SINGSMALL) {
        if (V[2] >= 0.0) V[2] = G_SINGSMALL;
        if (V[2] < 0.0) V[2] = -G_SINGSMALL;
    }
    if (fabs(M_PI - V[2]) < G_SINGSMALL) {
        if (V[2] >= M_PI) V[2] = M_PI + G_SINGSMALL;
        if (V[2] < M_PI) V[2] = M_PI - G_SINGSMALL;
    }
    *r = V[1];
    *th = V[2];
    *ph = V[3];
}

/* LU_decompose: Crout with implicit partial pivoting, in place */
static int g_lu(double A[GD][GD], int perm[GD]) {
    double rn[GD], big, t;
    int imax = 0;
    for (int i = 0; i < GD; i++) {
        big = 0.;
        for (int j = 0; j < GD; j++) {
            t = fabs(A[i][j]);
            if (t > big) big = t;
        }
        if (big == 0.) return 1;
        rn[i] = 1. / big;
    }
    for (int j = 0; j < GD; j++) {
        for (int i = 0; i < j; i++)
            for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
        big = 0.0;
        for (int i = j; i < GD; i++) {
            for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
            t = fabs(A[i][j]) * rn[i];
            if (t >= big) {
                big = t;
                imax = i;
            }
        }
        if (imax != j) {
            if ((j == (GD - 2)) && (A[j][j + 1] == 0.)) {
                imax = j;
            } else {
                for (int k = 0; k < GD; k++) {
                    t = A[j][k];
                    A[j][k] = A[imax][k];
                    A[imax][k] = t;
                }
                rn[imax] = rn[j];
            }
        }
        perm[j] = imax;
        if (A[j][j] == 0.) A[j][j] = 1.e-30;
        if (j != (GD - 1)) {
            t = 1. / A[j][j];
            for (int i = j + 1; i < GD; i++) A[i][j] *= t;
        }
    }
    return 0;
}

/* LU_substitution */
static void g_lusub(double A[GD][GD], double B[GD], const int perm[GD]) {
    for (int i = 0; i < GD; i++) {
        double s = B[perm[i]];
        B[perm[i]] = B[i];
        for (int j = i - 1; j >= 0; j--) s -= A[i][j] * B[j];
        B[i] = s;
    }
    for (int i = GD - 1; i >= 0; i--) {
        for (int j = i + 1; j < GD; j++) B[i] -= A[i][j] * B[j];
        B[i] /= A[i][i];
    }
}

/* invert_matrix: column by column */
static int g_inv(double M[GD][GD], double Mi[GD][GD]) {
    double T[GD][GD], col[GD];
    int perm[GD];
    memcpy(T, M, sizeof(T));
    if (g_lu(T, perm)) return 1;
    for (int i = 0; i < GD; i++) {
        for (int j = 0; j < GD; j++) col[j] = 0.;
        col[i] = 1.;
        g_lusub(T, col, perm);
        for (int j = 0; j < GD; j++) Mi[j][i] = col[j];
    }
    return 0;
}

/* gdet_func */
static double g_det(double g[GD][GD], int *fails) {
    double T[GD][GD];
    int perm[GD];
    memcpy(T, g, sizeof(T));
    if (g_lu(T, perm)) (*fails)++;
    double d = 1.;
    for (int j = 0; j < GD; j++) d *= T[j][j];
    return sqrt(fabs(d));
}

/* dxdxp_func */
static void g_dxdxp(const gmap *m, const double *X, double J[GD][GD]) {
    double Xh[GD], Xl[GD], Vh[GD], Vl[GD];
    for (int k = 0; k < GD; k++) {
        for (int l = 0; l < GD; l++) Xh[l] = X[l];
        for (int l = 0; l < GD; l++) Xl[l] = X[l];
        Xh[k] += 0.00001;
        Xl[k] -= 0.00001;
        Vh[0] = Xh[0];
        Vl[0] = Xl[0];
        g_bl(m, Xh, &Vh[1], &Vh[2], &Vh[3]);
        g_bl(m, Xl, &Vl[1], &Vl[2], &Vl[3]);
        for (int j = 0; j < GD; j++) J[j][k] = (Vh[j] - Vl[j]) / (Xh[k] - Xl[k]);
    }
}

/* gcov_func: Kerr-Schild pulled back to code coordinates, or Minkowski */
static void g_cov(const gmap *m, const double *X, double gp[GD][GD]) {
    double g[GD][GD], J[GD][GD], r, th, ph;
    for (int j = 0; j < GD; j++)
        for (int k = 0; k < GD; k++) g[j][k] = 0.;
    if (m->cart) {
        g[0][0] = -1.0;
        g[1][1] = 1.0;
        g[2][2] = 1.0;
        g[3][3] = 1.0;
        memcpy(gp, g, sizeof(g));
        return;
    }
    const double a = m->a;
    g_bl(m, X, &r, &th, &ph);
    const double cth = cos(th), sth = sin(th);
    const double s2 = sth * sth;
    const double rho2 = r * r + a * a * cth * cth;
    g_dxdxp(m, X, J);
    g[0][0] = (-1. + 2. * r / rho2);
    g[0][1] = (2. * r / rho2);
    g[0][3] = (-2. * a * r * s2 / rho2);
    g[1][0] = g[0][1];
    g[1][1] = (1. + 2. * r / rho2);
    g[1][3] = (-a * s2 * (1. + 2. * r / rho2));
    g[2][2] = rho2;
    g[3][0] = g[0][3];
    g[3][1] = g[1][3];
    g[3][3] = s2 * (rho2 + a * a * s2 * (1. + 2. * r / rho2));
    for (int i = 0; i < GD; i++)
        for (int j = 0; j < GD; j++) {
            gp[i][j] = 0.;
            for (int k = 0; k < GD; k++)
                for (int l = 0; l < GD; l++) gp[i][j] += g[k][l] * J[k][i] * J[l][j];
        }
}

/* conn_func: Gamma^i_{jk} by central differences of gcov, index raised */
static void g_conn(const gmap *m, const double *X, double gn[GD][GD], double C[GD][GD][GD]) {
    double T[GD][GD][GD], Xh[GD], Xl[GD], gh[GD][GD], gl[GD][GD];
    for (int k = 0; k < GD; k++) {
        for (int l = 0; l < GD; l++) Xh[l] = X[l];
        for (int l = 0; l < GD; l++) Xl[l] = X[l];
        Xh[k] += 1.e-5;
        Xl[k] -= 1.e-5;
        g_cov(m, Xh, gh);
        g_cov(m, Xl, gl);
        for (int i = 0; i < GD; i++)
            for (int j = 0; j < GD; j++) C[i][j][k] = (gh[i][j] - gl[i][j]) / (Xh[k] - Xl[k]);
    }
    for (int i = 0; i < GD; i++)
        for (int j = 0; j < GD; j++)
            for (int k = 0; k < GD; k++) T[i][j][k] = 0.5 * (C[j][i][k] + C[k][i][j] - C[k][j][i]);
    for (int i = 0; i < GD; i++)
        for (int j = 0; j < GD; j++)
            for (int k = 0; k < GD; k++) {
                C[i][j][k] = 0.;
                for (int l = 0; l < GD; l++) C[i][j][k] += gn[i][l] * T[l][j][k];
            }
}

/* coord(): code coordinates of location loc of zone (i, j, z), i and j
 * counted from the first active zone; theta ghosts mirror across the axis */
static void g_coord(const gmap *m, int n2, const double *sx, const double *dx, int i, int j, int z, int loc,
                    double *X) {
    int jl = j;
    X[0] = 0.0;
    if (!m->cart) {
        if (j < 0) jl = -j - 1;
        if (j >= n2) jl = 2 * n2 - 1 - j;
        if (j == n2 && loc == GL_FACE2) jl = j;
    }
    switch (loc) {
    case GL_FACE1:
        X[1] = sx[1] + i * dx[1];
        X[2] = sx[2] + (jl + 0.5) * dx[2];
        X[3] = sx[3] + (z + 0.5) * dx[3];
        break;
    case GL_FACE2:
        X[1] = sx[1] + (i + 0.5) * dx[1];
        X[2] = sx[2] + jl * dx[2];
        X[3] = sx[3] + (z + 0.5) * dx[3];
        break;
    case GL_FACE3:
        X[1] = sx[1] + (i + 0.5) * dx[1];
        X[2] = sx[2] + (jl + 0.5) * dx[2];
        X[3] = sx[3] + z * dx[3];
        break;
    default:
        X[1] = sx[1] + (i + 0.5) * dx[1];
        X[2] = sx[2] + (jl + 0.5) * dx[2];
        X[3] = sx[3] + (z + 0.5) * dx[3];
    }
    if (!m->cart) {
        if (j < 0) {
            X[2] = X[2] + 1;
            X[2] = -X[2];
            X[2] = X[2] - 1;
        }
        if (!(j == n2 && loc == GL_FACE2) && j >= n2) {
            X[2] = X[2] + 1;
            X[2] = 4. - X[2];
            X[2] = X[2] - 1;
        }
    }
}

static const int G_SI[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
static const int G_SJ[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};

static void g_put(double *gcov, double *gcon, double *gdet, long gs, long idx, int loc, double gc[GD][GD],
                  double gn[GD][GD], double g) {
    for (int s = 0; s < 10; s++) {
        gcov[(long)(s * 5 + loc) * gs + idx] = gc[G_SI[s]][G_SJ[s]];
        gcon[(long)(s * 5 + loc) * gs + idx] = gn[G_SI[s]][G_SJ[s]];
    }
    gdet[(long)loc * gs + idx] = g;
}

int ho_build_geometry(int coords, double spin, int n1, int n2, int n3, int ng, long gsize, const double *startx,
                      const double *dx, double *gcov, double *gcon, double *gdet, double *conn) {
    if (n1 < 1 || n2 < 1 || n3 < 1 || ng < 0 || (coords != 0 && coords != 1)) return -1;
    const gmap m = {coords, spin};
    const int ng1 = n1 > 1 ? ng : 0, ng2 = n2 > 1 ? ng : 0;
    const long G1 = n1 + 2 * ng1, G2 = n2 + 2 * ng2;
    if (gsize < G1 * G2) return -1;
    memset(gcov, 0, sizeof(double) * 50 * gsize);
    memset(gcon, 0, sizeof(double) * 50 * gsize);
    memset(gdet, 0, sizeof(double) * 5 * gsize);
    memset(conn, 0, sizeof(double) * 40 * gsize);
    int fails = 0;
#pragma omp parallel for collapse(2) reduction(+ : fails) schedule(static)
    for (int i = -ng1; i < n1 + ng1; i++)
        for (int j = -ng2; j < n2 + ng2; j++) {
            const long idx = (long)(i + ng1) * G2 + (j + ng2);
            double X[GD], gc[GD][GD], gn[GD][GD], C[GD][GD][GD], g;
            g_coord(&m, n2, startx, dx, i, j, 0, GL_CENT, X);
            g_cov(&m, X, gc);
            g = g_det(gc, &fails);
            fails += g_inv(gc, gn);
            g_put(gcov, gcon, gdet, gsize, idx, GL_CENT, gc, gn, g);
            g_conn(&m, X, gn, C);
            for (int s = 0; s < 10; s++)
                for (int l = 0; l < GD; l++) conn[(long)(s * 4 + l) * gsize + idx] = C[l][G_SI[s]][G_SJ[s]];
            const int locs[3] = {GL_FACE1, GL_FACE3, GL_FACE2};
            for (int t = 0; t < 3; t++) {
                g_coord(&m, n2, startx, dx, i, j, 0, locs[t], X);
                g_cov(&m, X, gc);
                g = g_det(gc, &fails);
                fails += g_inv(gc, gn);
                g_put(gcov, gcon, gdet, gsize, idx, locs[t], gc, gn, g);
            }
        }
    return fails ? -5 : 0;
}

int ho_bl_coord(int coords, double spin, const double *X, double *rthph) {
    const gmap m = {coords, spin};
    g_bl(&m, X, &rthph[0], &rthph[1], &rthph[2]);
    return 0;
}

#ifdef _OPENMP
#include <omp.h>
int ho_num_threads(void) { return omp_get_max_threads(); }
#else
int ho_num_threads(void) { return 1; }
#endif

/* Check of the exact-division method the CUDA library uses for divisions by
 * the constant zone widths (div_rcp): q0 = a*rb, r = fma(-q0, b, a),
 * q = r == 0 ? q0 : fma(r, rb, q0) with rb = 1/b correctly rounded. Returns how
 * many of the n*m quotients a[i]/b[j] it does not reproduce bit for bit
 * (compared as bit patterns; both sides are IEEE binary64 round-to-nearest). */
long ho_div_rcp_mismatches(const double *a, long n, const double *b, long m) {
    return ho_div_rcp_mismatches_g(a, n, b, m, 0);
}

/* The same with the guard of the form that also covers infinite operands and
 * a zero divisor (guard = 1): q = (r == 0 || r not finite) ? q0 : fma(r, rb, q0). */
long ho_div_rcp_mismatches_g(const double *a, long n, const double *b, long m, int guard) {
    long bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
    for (long j = 0; j < m; j++) {
        const double rb = 1.0 / b[j];
        for (long i = 0; i < n; i++) {
            const double q0 = a[i] * rb;
            const double r = fma(-q0, b[j], a[i]);
            const double q = (r == 0.0 || (guard && !(fabs(r) <= DBL_MAX))) ? q0 : fma(r, rb, q0);
            const double e = a[i] / b[j];
            if (memcmp(&q, &e, sizeof(double)) != 0) bad++;
        }
    }
    return bad;
}
