// Host-side metric tables for one uniform block (the product's geometry
// builder; no device code). Follows set_grid (main.c:380-455): at every
// (i, j) of the ghosted block the metric is evaluated at the zone centre, the
// x1-, x2- and x3-faces, and the connection at the zone centre.
//
// The coordinate map, Kerr-Schild metric, finite-difference Jacobian and
// connection, and the pivoted LU used for det/inverse keep the reference's
// operation order, so the tables agree with the reference's own bit for bit
// (tests/test_geometry.py):
//   coord            coord.c:26-109
//   vofx_matthewcoords / bl_coord  coord.c:111-211
//   gcov_func_spherical            metric.c:13-271 (no tilt)
//   dxdxp_func       metric.c:501-519 (central differences, step 1e-5)
//   gdet_func / gcon_func          metric.c:392-414
//   conn_func        metric.c:427-464 (central differences, step 1e-5)
//   LU_decompose / LU_substitution / invert_matrix   lu.c:17-45,157-313,806-843
//     (Crout decomposition with implicit partial pivoting, Numerical Recipes
//      ludcmp/lubksb)
#include <cmath>
#include <cstring>

#include "../../include/hamr_b200.h"

namespace {

constexpr int NDIM = 4;
constexpr int NPG = 5;
enum { FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3, FACE3 = 4 };

// grid-map constants of the reference's default uniform-theta grid
// (config.h:555-568)
constexpr double RADEXP = 1.0, RTRANS = 5000000., RB = 0.;
constexpr double BRAVO = 0.0, TANGO = 1.0, CHARLIE = 0.0, DELTA = 3.0;
constexpr double SINGSMALL = 1.E-20;
constexpr double FD_EPS = 1.e-5;

struct Map {
    int coords;  // 0: spherical Kerr-Schild, 1: Cartesian Minkowski
    double a;
};

// code coordinates -> (r, theta, phi)
void bl_coord(const Map &m, const double *X, double *r, double *th, double *phi) {
    double V[NDIM];
    if (m.coords == 1) {
        *r = std::sqrt(X[1] * X[1] + X[2] * X[2] + X[3] * X[3]);
        *th = 0.;
        *phi = 0.;
        return;
    }
    V[0] = X[0];
    double Xtrans = std::pow(std::log(RTRANS - RB), 1. / RADEXP);
    if (X[1] < Xtrans) {
        V[1] = std::exp(std::pow(X[1], RADEXP)) + RB;
    } else if (X[1] >= Xtrans && X[1] < 1.01 * Xtrans) {
        V[1] = 10. * (X[1] / Xtrans - 1.) * ((X[1] - Xtrans) * RADEXP * std::exp(std::pow(Xtrans, RADEXP)) * std::pow(Xtrans, -1. + RADEXP) + RTRANS) +
               (1. - 10. * (X[1] / Xtrans - 1.)) * (std::exp(std::pow(X[1], RADEXP)) + RB);
    } else {
        V[1] = (X[1] - Xtrans) * RADEXP * std::exp(std::pow(Xtrans, RADEXP)) * std::pow(Xtrans, -1. + RADEXP) + RTRANS;
    }
    double A1 = 1. / (1. + std::pow(CHARLIE * (std::log(V[1]) / std::log(10.)), DELTA));
    double A2 = BRAVO * (std::log(V[1]) / std::log(10.)) + TANGO;
    double A3 = std::pow(0.5, 1. - A2);
    double sign = 1.;
    double X_2 = (X[2] + 1.0) / 2.0;
    double Xc = std::sqrt(std::pow(X_2, 2.));
    if (X_2 < 0.0) sign = -1.;
    if (X_2 > 1.0) {
        sign = -1.;
        Xc = 2. - Xc;
    }
    if (X_2 >= 0.5) {
        Xc = 1. - Xc;
        V[2] = M_PI - sign * (A1 * M_PI * Xc + M_PI * (1. - A1) * (A3 * std::pow(Xc, A2) + 0.50 / M_PI * std::sin(M_PI + 2. * M_PI * (A3 * std::pow(Xc, A2)))));
    } else {
        V[2] = sign * (A1 * M_PI * Xc + M_PI * (1. - A1) * (A3 * std::pow(Xc, A2) + 0.50 / M_PI * std::sin(M_PI + 2. * M_PI * (A3 * std::pow(Xc, A2)))));
    }
    V[3] = X[3];
    // keep off the polar axis (COORDSINGFIX)
    if (std::fabs(V[2]) < SINGSMALL) {
        if (V[2] >= 0.0) V[2] = SINGSMALL;
        if (V[2] < 0.0) V[2] = -SINGSMALL;
    }
    if (std::fabs(M_PI - V[2]) < SINGSMALL) {
        if (V[2] >= M_PI) V[2] = M_PI + SINGSMALL;
        if (V[2] < M_PI) V[2] = M_PI - SINGSMALL;
    }
    *r = V[1];
    *th = V[2];
    *phi = V[3];
}

// Crout LU with implicit partial pivoting, in place; returns nonzero for a
// row-wise singular matrix
int lu_decompose(double A[NDIM][NDIM], int permute[NDIM]) {
    double row_norm[NDIM];
    const double absmin = 1.e-30;
    double absmax, maxtemp;
    int max_row = 0;
    const int n = NDIM;
    for (int i = 0; i < n; i++) {
        absmax = 0.;
        for (int j = 0; j < n; j++) {
            maxtemp = std::fabs(A[i][j]);
            if (maxtemp > absmax) absmax = maxtemp;
        }
        if (absmax == 0.) return 1;
        row_norm[i] = 1. / absmax;
    }
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < j; i++)
            for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
        absmax = 0.0;
        for (int i = j; i < n; i++) {
            for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
            maxtemp = std::fabs(A[i][j]) * row_norm[i];
            if (maxtemp >= absmax) {
                absmax = maxtemp;
                max_row = i;
            }
        }
        if (max_row != j) {
            if ((j == (n - 2)) && (A[j][j + 1] == 0.)) {
                max_row = j;
            } else {
                for (int k = 0; k < n; k++) {
                    maxtemp = A[j][k];
                    A[j][k] = A[max_row][k];
                    A[max_row][k] = maxtemp;
                }
                row_norm[max_row] = row_norm[j];
            }
        }
        permute[j] = max_row;
        if (A[j][j] == 0.) A[j][j] = absmin;
        if (j != (n - 1)) {
            maxtemp = 1. / A[j][j];
            for (int i = (j + 1); i < n; i++) A[i][j] *= maxtemp;
        }
    }
    return 0;
}

void lu_substitution(const double A[NDIM][NDIM], double B[NDIM], const int permute[NDIM]) {
    const int n = NDIM;
    for (int i = 0; i < n; i++) {
        double tmpvar = B[permute[i]];
        B[permute[i]] = B[i];
        for (int j = (i - 1); j >= 0; j--) tmpvar -= A[i][j] * B[j];
        B[i] = tmpvar;
    }
    for (int i = (n - 1); i >= 0; i--) {
        for (int j = (i + 1); j < n; j++) B[i] -= A[i][j] * B[j];
        B[i] /= A[i][i];
    }
}

int invert(const double Am[NDIM][NDIM], double Aminv[NDIM][NDIM]) {
    int permute[NDIM];
    double dxm[NDIM], Amtmp[NDIM][NDIM];
    std::memcpy(Amtmp, Am, sizeof(Amtmp));
    if (lu_decompose(Amtmp, permute) != 0) return 1;
    for (int i = 0; i < NDIM; i++) {
        for (int j = 0; j < NDIM; j++) dxm[j] = 0.;
        dxm[i] = 1.;
        lu_substitution(Amtmp, dxm, permute);
        for (int j = 0; j < NDIM; j++) Aminv[j][i] = dxm[j];
    }
    return 0;
}

double gdet_of(const double gcov[NDIM][NDIM], int *fail) {
    int permute[NDIM];
    double tmp[NDIM][NDIM];
    std::memcpy(tmp, gcov, sizeof(tmp));
    if (lu_decompose(tmp, permute) != 0) {
        (*fail)++;
    }
    double detg = 1.;
    for (int j = 0; j < NDIM; j++) detg *= tmp[j][j];
    return std::sqrt(std::fabs(detg));
}

// d(r, theta, phi)/dX by central differences
void dxdxp_of(const Map &m, const double *X, double dxdxp[NDIM][NDIM]) {
    double Xh[NDIM], Xl[NDIM], Vh[NDIM], Vl[NDIM];
    for (int k = 0; k < NDIM; k++) {
        for (int l = 0; l < NDIM; l++) Xh[l] = X[l];
        for (int l = 0; l < NDIM; l++) Xl[l] = X[l];
        Xh[k] += 0.00001;
        Xl[k] -= 0.00001;
        Vh[0] = Xh[0];
        Vl[0] = Xl[0];
        bl_coord(m, Xh, &Vh[1], &Vh[2], &Vh[3]);
        bl_coord(m, Xl, &Vl[1], &Vl[2], &Vl[3]);
        for (int j = 0; j < NDIM; j++) dxdxp[j][k] = (Vh[j] - Vl[j]) / (Xh[k] - Xl[k]);
    }
}

void gcov_of(const Map &m, const double *X, double gcovp[NDIM][NDIM]) {
    double gcov[NDIM][NDIM];
    for (int j = 0; j < NDIM; j++)
        for (int k = 0; k < NDIM; k++) gcov[j][k] = 0.;
    if (m.coords == 1) {
        gcov[0][0] = -1.0;
        gcov[1][1] = 1.0;
        gcov[2][2] = 1.0;
        gcov[3][3] = 1.0;
        std::memcpy(gcovp, gcov, sizeof(gcov));
        return;
    }
    const double a = m.a;
    double r, th, phi, dxdxp[NDIM][NDIM];
    bl_coord(m, X, &r, &th, &phi);
    double cth = std::cos(th);
    double sth = std::sin(th);
    double s2 = sth * sth;
    double rho2 = r * r + a * a * cth * cth;
    dxdxp_of(m, X, dxdxp);
    gcov[0][0] = (-1. + 2. * r / rho2);
    gcov[0][1] = (2. * r / rho2);
    gcov[0][3] = (-2. * a * r * s2 / rho2);
    gcov[1][0] = gcov[0][1];
    gcov[1][1] = (1. + 2. * r / rho2);
    gcov[1][3] = (-a * s2 * (1. + 2. * r / rho2));
    gcov[2][2] = rho2;
    gcov[3][0] = gcov[0][3];
    gcov[3][1] = gcov[1][3];
    gcov[3][3] = s2 * (rho2 + a * a * s2 * (1. + 2. * r / rho2));
    for (int i = 0; i < NDIM; i++)
        for (int j = 0; j < NDIM; j++) {
            gcovp[i][j] = 0.;
            for (int k = 0; k < NDIM; k++)
                for (int l = 0; l < NDIM; l++) gcovp[i][j] += gcov[k][l] * dxdxp[k][i] * dxdxp[l][j];
        }
}

// Gamma^i_{jk} by central differences of the metric
void conn_of(const Map &m, const double *X, const double gcon[NDIM][NDIM], double conn[NDIM][NDIM][NDIM]) {
    double tmp[NDIM][NDIM][NDIM], Xh[NDIM], Xl[NDIM], gh[NDIM][NDIM], gl[NDIM][NDIM];
    for (int k = 0; k < NDIM; k++) {
        for (int l = 0; l < NDIM; l++) Xh[l] = X[l];
        for (int l = 0; l < NDIM; l++) Xl[l] = X[l];
        Xh[k] += FD_EPS;
        Xl[k] -= FD_EPS;
        gcov_of(m, Xh, gh);
        gcov_of(m, Xl, gl);
        for (int i = 0; i < NDIM; i++)
            for (int j = 0; j < NDIM; j++) conn[i][j][k] = (gh[i][j] - gl[i][j]) / (Xh[k] - Xl[k]);
    }
    for (int i = 0; i < NDIM; i++)
        for (int j = 0; j < NDIM; j++)
            for (int k = 0; k < NDIM; k++) tmp[i][j][k] = 0.5 * (conn[j][i][k] + conn[k][i][j] - conn[k][j][i]);
    for (int i = 0; i < NDIM; i++)
        for (int j = 0; j < NDIM; j++)
            for (int k = 0; k < NDIM; k++) {
                conn[i][j][k] = 0.;
                for (int l = 0; l < NDIM; l++) conn[i][j][k] += gcon[i][l] * tmp[l][j][k];
            }
}

// code coordinates of location loc of zone (i, j, z); i, j counted from the
// first active zone; ghost zones beyond the polar axis mirror back across it
void coord_of(const Map &m, int n2, const double *startx, const double *dx, int i, int j, int z, int loc, double *X) {
    X[0] = 0.0;
    int j_local = j;
    const bool sph = m.coords == 0;
    if (sph) {
        if (j < 0) j_local = -j - 1;
        if (j >= n2) j_local = 2 * n2 - 1 - j;
        if (j == n2 && loc == FACE2) j_local = j;
    }
    if (loc == FACE1) {
        X[1] = startx[1] + i * dx[1];
        X[2] = startx[2] + (j_local + 0.5) * dx[2];
        X[3] = startx[3] + (z + 0.5) * dx[3];
    } else if (loc == FACE2) {
        X[1] = startx[1] + (i + 0.5) * dx[1];
        X[2] = startx[2] + j_local * dx[2];
        X[3] = startx[3] + (z + 0.5) * dx[3];
    } else if (loc == FACE3) {
        X[1] = startx[1] + (i + 0.5) * dx[1];
        X[2] = startx[2] + (j_local + 0.5) * dx[2];
        X[3] = startx[3] + z * dx[3];
    } else {
        X[1] = startx[1] + (i + 0.5) * dx[1];
        X[2] = startx[2] + (j_local + 0.5) * dx[2];
        X[3] = startx[3] + (z + 0.5) * dx[3];
    }
    if (sph) {
        if (j < 0) {
            X[2] = X[2] + 1;
            X[2] = -X[2];
            X[2] = X[2] - 1;
        }
        if (j == n2 && loc == FACE2) {
        } else if (j >= n2) {
            X[2] = X[2] + 1;
            X[2] = 4. - X[2];
            X[2] = X[2] - 1;
        }
    }
}

const int SYM_I[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
const int SYM_J[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};

}  // namespace

extern "C" int hamr_build_geometry(int coords, double spin, int n1, int n2, int n3, int ng, long gsize,
                                   const double *startx, const double *dx, double *gcov_out,
                                   double *gcon_out, double *gdet_out, double *conn_out) {
    if (n1 < 1 || n2 < 1 || n3 < 1 || ng < 0 || !startx || !dx || !gcov_out || !gcon_out || !gdet_out || !conn_out)
        return HAMR_E_ARG;
    if (coords != 0 && coords != 1) return HAMR_E_ARG;
    const Map m{coords, spin};
    const int ng1 = n1 > 1 ? ng : 0, ng2 = n2 > 1 ? ng : 0;
    const long G1 = n1 + 2 * ng1, G2 = n2 + 2 * ng2;
    if (gsize == 0) gsize = G1 * G2 + (64 - (G1 * G2) % 64);
    if (gsize < G1 * G2) return HAMR_E_ARG;
    std::memset(gcov_out, 0, sizeof(double) * 10 * NPG * gsize);
    std::memset(gcon_out, 0, sizeof(double) * 10 * NPG * gsize);
    std::memset(gdet_out, 0, sizeof(double) * NPG * gsize);
    std::memset(conn_out, 0, sizeof(double) * 10 * NDIM * gsize);
    int fail = 0;
    auto put = [&](long idx, int loc, const double gc[NDIM][NDIM], const double gn[NDIM][NDIM], double g) {
        for (int s = 0; s < 10; s++) {
            gcov_out[(long)(s * NPG + loc) * gsize + idx] = gc[SYM_I[s]][SYM_J[s]];
            gcon_out[(long)(s * NPG + loc) * gsize + idx] = gn[SYM_I[s]][SYM_J[s]];
        }
        gdet_out[(long)loc * gsize + idx] = g;
    };
    for (int i = -ng1; i < n1 + ng1; i++)
        for (int j = -ng2; j < n2 + ng2; j++) {
            const long idx = (long)(i + ng1) * G2 + (j + ng2);
            double X[NDIM], gc[NDIM][NDIM], gn[NDIM][NDIM], cn[NDIM][NDIM][NDIM], g;
            coord_of(m, n2, startx, dx, i, j, 0, CENT, X);
            gcov_of(m, X, gc);
            g = gdet_of(gc, &fail);
            fail += invert(gc, gn);
            put(idx, CENT, gc, gn, g);
            conn_of(m, X, gn, cn);
            for (int s = 0; s < 10; s++)
                for (int l = 0; l < NDIM; l++) conn_out[(long)(s * NDIM + l) * gsize + idx] = cn[l][SYM_I[s]][SYM_J[s]];
            const int locs[3] = {FACE1, FACE3, FACE2};
            for (int t = 0; t < 3; t++) {
                coord_of(m, n2, startx, dx, i, j, 0, locs[t], X);
                gcov_of(m, X, gc);
                g = gdet_of(gc, &fail);
                fail += invert(gc, gn);
                put(idx, locs[t], gc, gn, g);
            }
        }
    return fail ? HAMR_E_PHYSICS : HAMR_OK;
}

extern "C" int hamr_bl_coord(int coords, double spin, const double *X, double *rthph) {
    if (!X || !rthph) return HAMR_E_ARG;
    const Map m{coords, spin};
    bl_coord(m, X, &rthph[0], &rthph[1], &rthph[2]);
    return HAMR_OK;
}
