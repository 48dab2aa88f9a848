// Adjoint (reverse mode) of the FP64 RK2 step for axisymmetric blocks: 2-D
// (n3 == 1), PPM, HLL, upwinded CT, Noble 2D inversion, outflow x1 with the
// no-inflow check, reflective polar axis in x2. Included at the end of
// hamr_kernels.cu.
//
// The step is reversed phase by phase. Linear phases (ghost fill copies,
// flux divergence, face update, edge EMF, polar flux fix) have their
// transposes written out; nonlinear per-item maps (face flux, centre EMF,
// geometric source, conserved variables of a state, no-inflow check) get
// their local derivatives from the forward routines themselves, instantiated
// with forward-mode dual numbers (hamr_dual.cuh), and their transposes are
// applied to the incoming cotangents. The inversion is reversed by the
// implicit-function theorem: U(p) = W at the solution, so
// W_bar = (dU/dp)^-T p_bar over the five hydrodynamic primitives. Limiter and
// upwind branches are the ones the forward step took; the CFL step sizes are
// held fixed.
#include "hamr_dual.cuh"

namespace {

constexpr int ADJ_NP = 8;   // differentiated primitives: RHO, UU, U1-3, B1-3 (KTOT enters no flux)

// --- templated copies of the double-only forward helpers ------------------
// (the same operations as inflow_check and source in this file)
template <typename T>
__device__ __forceinline__ void inflow_check_t(T *pr, const Geo<double> &gm, int type) {
    T ucon[4], gamma;
    ucon_calc(pr, gm, ucon);
    if (((ucon[1] > T(0.)) && (type == 0)) || ((ucon[1] < T(0.)) && (type == 1))) {
        gamma_calc(pr, gm, &gamma);
        pr[U1] /= gamma;
        pr[U2] /= gamma;
        pr[U3] /= gamma;
        const double alpha = 1. / sqrt(-gm.gcon[0]);
        const double beta1 = gm.gcon[1] * alpha * alpha;
        pr[U1] = T(beta1 / alpha);
        T vsq = gm.gcov[4] * pr[U1] * pr[U1];
        vsq += T(2.) * gm.gcov[5] * pr[U2] * pr[U1];
        vsq += T(2.) * gm.gcov[6] * pr[U3] * pr[U1];
        vsq += gm.gcov[7] * pr[U2] * pr[U2];
        vsq += T(2.) * gm.gcov[8] * pr[U3] * pr[U2];
        vsq += gm.gcov[9] * pr[U3] * pr[U3];
        vsq = d_max(T(1.e-13), vsq);
        if (vsq >= T(1.)) vsq = T(1. - 1. / (80. * 80.));
        gamma = T(1.) / d_sqrt(T(1.) - vsq);
        pr[U1] *= gamma;
        pr[U2] *= gamma;
        pr[U3] *= gamma;
    }
}

template <typename T, typename G>
__device__ __forceinline__ void source_t(T gam, const T *ph, const Geo<G> &gm, const Dims &d, const Geom &m,
                                         long gi, T *dU, const State<T> &q) {
    T mhd[4][4];
    const long gs = d.gs;
    const T P = (gam - T(1.)) * ph[UU];
    const T u = ph[UU];
    const T w = P + ph[RHO] + u;
    const T bsq = dot4(q.bcon, q.bcov);
    const T eta = w + bsq;
    const T ptot = P + T(0.5) * bsq;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            mhd[a][b] = eta * q.ucon[a] * q.ucov[b] + ptot * T(a == b ? 1. : 0.) - q.bcon[a] * q.bcov[b];
    for (int k = 0; k < NPR; k++) dU[k] = T(0.);
#define CONN(s, k) __ldg(&m.conn[(long)((s) * 4 + (k)) * gs + gi])
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
    dU[UU] *= gm.g;
    dU[U1] *= gm.g;
    dU[U2] *= gm.g;
    dU[U3] *= gm.g;
    dU[KTOT] *= gm.g;
}

// inputs of a state map: the ADJ_NP primitives, then gamma (index ADJ_NP)
// (every index compile-time after unrolling, so the duals stay in registers)
template <int N>
__device__ __forceinline__ void seed_state(const double *pr, double gam, int pass, Dual<N> *pd, Dual<N> &gd) {
#pragma unroll
    for (int k = 0; k < NPR; k++) {
        pd[k].v = pr[k];
#pragma unroll
        for (int q = 0; q < N; q++) pd[k].d[q] = (k < ADJ_NP && k == pass * N + q) ? 1. : 0.;
    }
    gd.v = gam;
#pragma unroll
    for (int q = 0; q < N; q++) gd.d[q] = (ADJ_NP == pass * N + q) ? 1. : 0.;
}

__device__ __forceinline__ void block_add(double v, double *target) {
    // CTA sum by warp shuffles, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.) atomicAdd(target, v);
}

}  // namespace

namespace {

// ---- PPM stencil weights -------------------------------------------------
// para (GPU_interp.h:60-111) is linear in its five inputs on each branch of
// its limiter and clamps; these are the weights of the lower (upper == false)
// or upper edge value in the branch the values take, built from the
// branch-local coefficients of the three MC slopes (the dual-number
// derivative of para, without carrying five derivatives through every
// operation)
__device__ __forceinline__ void para_weights(const double *y, bool upper, double *w) {
    double dq[4], c0[4], c1[4], c2[4];   // slope i = c0 y[i-1] + c1 y[i] + c2 y[i+1]
#pragma unroll
    for (int i = 1; i < 4; i++) {
        const double Dqm = 2. * (y[i] - y[i - 1]);
        const double Dqp = 2. * (y[i + 1] - y[i]);
        const double Dqc = 0.5 * (y[i + 1] - y[i - 1]);
        const double aDqm = d_fabs(Dqm), aDqp = d_fabs(Dqp), aDqc = d_fabs(Dqc);
        const double mn = d_min(aDqm, aDqp);
        const double on = (double)(Dqm * Dqp > 0.);
        const double sc = Dqc > 0. ? 1. : -1.;
        const bool selc = aDqc < mn, selm = aDqm < aDqp;
        dq[i] = (sc * (selc ? aDqc : mn)) * on;
        const double gc = sc * (Dqc < 0. ? -1. : 1.) * on * 0.5;
        const double gm = sc * (Dqm < 0. ? -1. : 1.) * on * 2.;
        const double gp = sc * (Dqp < 0. ? -1. : 1.) * on * 2.;
        c0[i] = selc ? -gc : (selm ? -gm : 0.);
        c1[i] = selc ? 0. : (selm ? gm : -gp);
        c2[i] = selc ? gc : (selm ? 0. : gp);
    }
    double l = 0.5 * (y[2] + y[1]) - div6(dq[2] - dq[1]);   // the forward's edges, bit for bit
    double r = 0.5 * (y[3] + y[2]) - div6(dq[3] - dq[2]);
    const double s6 = 1. / 6.0;
    double wl[5] = {c0[1] * s6, 0.5 + (c1[1] - c0[2]) * s6, 0.5 + (c2[1] - c1[2]) * s6, -c2[2] * s6, 0.};
    double wr[5] = {0., c0[2] * s6, 0.5 + (c1[2] - c0[3]) * s6, 0.5 + (c2[2] - c1[3]) * s6, -c2[3] * s6};
    const double qa = (r - y[2]) * (y[2] - l);
    const double qd = (r - l);
    const double qe = 6.0 * (y[2] - 0.5 * (l + r));
    const bool flat = qa <= 0.;
    const bool fixl = qd * (qd - qe) < 0.0, fixr = !fixl && qd * (qd + qe) < 0.0;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const double e2 = k == 2 ? 1. : 0.;
        const double a = flat ? e2 : wl[k], b = flat ? e2 : wr[k];
        wl[k] = fixl ? 3. * e2 - 2. * b : a;
        wr[k] = fixr ? 3. * e2 - 2. * a : b;
    }
#pragma unroll
    for (int k = 0; k < 5; k++) w[k] = upper ? wr[k] : wl[k];
}

// ---- reverse mode of one state's fluxes, conserved variables and speeds ----
// Hand-written transpose of get_state + primtoflux (GPU_phys_mhd.h:432-628,
// 672-761) over a constant metric: the forward values are recomputed, then
// the cotangents run back through the flux formulas, the magnetosonic
// quadratic, the scalars (w, P, b^2, eta, ptot, entropy K), b_mu, b^mu, u_mu,
// u^mu and gamma, in the branch the forward took (clamped speeds and a
// clamped Lorentz factor pass no derivative).
struct StateBar {
    double ucon[4], ucov[4], bcon[4], bcov[4];
    double rho, u, gam, eta, ptot, w, P, bsq, K;
};

// flux along D (D == 0: conserved variables) reversed, given the cotangent cb
template <int D>
__device__ __forceinline__ void flux_rev(const double *pr, const State<double> &q, double g, double eta, double K,
                                         const double *cb, StateBar &a) {
    double c[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) c[k] = cb[k] * g;
    const double frb = c[RHO] + c[UU] + c[KTOT] * K;   // F[UU] and F[KTOT] carry F[RHO]
    a.K += c[KTOT] * (pr[RHO] * q.ucon[D]);
    a.rho += frb * q.ucon[D];
    a.ucon[D] += frb * pr[RHO];
    const double mb[4] = {c[UU], c[U1], c[U2], c[U3]};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        a.eta += mb[j] * q.ucon[D] * q.ucov[j];
        a.ucon[D] += mb[j] * eta * q.ucov[j];
        a.ucov[j] += mb[j] * eta * q.ucon[D];
        a.bcon[D] -= mb[j] * q.bcov[j];
        a.bcov[j] -= mb[j] * q.bcon[D];
    }
    a.ptot += mb[D];
#pragma unroll
    for (int i = 1; i < 4; i++) {
        if (i == D) continue;   // b^D u^D - b^D u^D: identically zero
        const double cB = c[B1 + i - 1];
        a.bcon[i] += cB * q.ucon[D];
        a.ucon[D] += cB * q.bcon[i];
        a.bcon[D] -= cB * q.ucon[i];
        a.ucon[i] -= cB * q.bcon[D];
    }
}

// forward values the reverse needs
struct StateFwd {
    State<double> q;
    double gam_l, P, w, bsq, eta, K;
    bool gfree;   // the Lorentz factor is sqrt(1 + q^2), not clamped
};

// need_k: the entropy K = P rho^-gam is wanted (its pow is skipped, K = 0,
// where no entropy-flux cotangent can reach it)
__device__ __forceinline__ void state_fwd(const double *pr, const Geo<double> &gm, double gam, StateFwd &f,
                                          bool need_k = true) {
    const double *gc = gm.gcov;
    get_state(pr, gm, f.q);
    gamma_calc(pr, gm, &f.gam_l);
    const double u1 = pr[U1], u2 = pr[U2], u3 = pr[U3];
    const double qsq = gc[4] * u1 * u1 + gc[7] * u2 * u2 + gc[9] * u3 * u3
                     + 2. * (gc[5] * u1 * u2 + gc[6] * u1 * u3 + gc[8] * u2 * u3);
    f.gfree = !(qsq < 0.);
    f.P = (gam - 1.) * pr[UU];
    f.w = pr[RHO] + f.P + pr[UU];
    f.bsq = dot4(f.q.bcon, f.q.bcov);
    f.eta = f.w + f.bsq;
    f.K = need_k ? entropy(gam, pr) : 0.;
}

__device__ __forceinline__ void bar_zero(StateBar &a) {
#pragma unroll
    for (int k = 0; k < 4; k++) a.ucon[k] = a.ucov[k] = a.bcon[k] = a.bcov[k] = 0.;
    a.rho = a.u = a.gam = a.eta = a.ptot = a.w = a.P = a.bsq = a.K = 0.;
}

// from the cotangents of the scalars and of u^mu, u_mu, b^mu, b_mu back to
// the primitives (pbar, ADJ_NP) and gamma (added to gbar)
__device__ __forceinline__ void state_back(const double *pr, const Geo<double> &gm, double gam, const StateFwd &f,
                                           StateBar &a, double *pbar, double &gbar) {
    const double *gc = gm.gcov, *gn = gm.gcon;
    const State<double> &q = f.q;
    const double u = pr[UU], rho = pr[RHO];
    // eta = w + b^2, ptot = P + b^2/2, w = rho + P + u, P = (gam - 1) u,
    // K = (gam - 1) u rho^-gam
    a.w += a.eta;
    a.bsq += a.eta + 0.5 * a.ptot;
    a.P += a.ptot + a.w;
    a.rho += a.w;
    a.u += a.w + a.P * (gam - 1.);
    a.gam += a.P * u;
    if (a.K != 0.) {
        const double rg = pow(rho, -gam);
        a.u += a.K * (gam - 1.) * rg;
        a.gam += a.K * (u * rg - f.K * log(rho));
        a.rho -= a.K * gam * f.K / rho;
    }
    // b^2 = b^mu b_mu; b_mu = g_{mu nu} b^nu
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        a.bcon[mu] += a.bsq * q.bcov[mu];
        a.bcov[mu] += a.bsq * q.bcon[mu];
    }
    {
        double t[4];
        lower4(a.bcov, gc, t);
#pragma unroll
        for (int mu = 0; mu < 4; mu++) a.bcon[mu] += t[mu];
    }
    // b^j = (B^j + b^0 u^j) / u^0, then b^0 = B^i u_i
    double Bb[3];
    const double ru0 = 1. / q.ucon[0];
#pragma unroll
    for (int j = 1; j < 4; j++) {
        const double bj = a.bcon[j] * ru0;
        Bb[j - 1] = bj;
        a.bcon[0] += bj * q.ucon[j];
        a.ucon[j] += bj * q.bcon[0];
        a.ucon[0] -= bj * q.bcon[j];
    }
#pragma unroll
    for (int i = 1; i < 4; i++) {
        Bb[i - 1] += a.bcon[0] * q.ucov[i];
        a.ucov[i] += a.bcon[0] * pr[B1 + i - 1];
    }
    // u_mu = g_{mu nu} u^nu
    {
        double t[4];
        lower4(a.ucov, gc, t);
#pragma unroll
        for (int mu = 0; mu < 4; mu++) a.ucon[mu] += t[mu];
    }
    // u^0 = gamma / alpha, u^j = u~^j - gamma beta^j / alpha, beta^j = g^{0j} alpha^2
    // (1/alpha = sqrt(-g^tt); beta^j / alpha = g^{0j} alpha)
    const double sg = d_sqrt(-gn[0]), alpha = 1. / sg;
    double gb = a.ucon[0] * sg;
#pragma unroll
    for (int j = 1; j < 4; j++) gb -= a.ucon[j] * (gn[j] * alpha);
    double ub3[3] = {a.ucon[1], a.ucon[2], a.ucon[3]};
    if (f.gfree) {
        const double u1 = pr[U1], u2 = pr[U2], u3 = pr[U3];
        const double qb = 0.5 * gb / f.gam_l;   // gamma = sqrt(1 + q^2)
        ub3[0] += 2. * qb * (gc[4] * u1 + gc[5] * u2 + gc[6] * u3);
        ub3[1] += 2. * qb * (gc[5] * u1 + gc[7] * u2 + gc[8] * u3);
        ub3[2] += 2. * qb * (gc[6] * u1 + gc[8] * u2 + gc[9] * u3);
    }
    pbar[RHO] = a.rho;
    pbar[UU] = a.u;
    pbar[U1] = ub3[0];
    pbar[U2] = ub3[1];
    pbar[U3] = ub3[2];
    pbar[B1] = Bb[0];
    pbar[B2] = Bb[1];
    pbar[B3] = Bb[2];
    gbar += a.gam;
}

// pbar (ADJ_NP) and gbar (added) from the cotangents of the fluxes along DIR
// (fb), of the conserved variables (ub) and of the fast speeds along DIR
// (DIR == 0: conserved variables only)
template <int DIR>
__device__ void state_vjp_from(const double *pr, const Geo<double> &gm, double gam, const StateFwd &f,
                               const double *fb, const double *ub, double cmxb, double cmnb, double *pbar,
                               double &gbar) {
    const double *gn = gm.gcon;
    const State<double> &q = f.q;
    const double u = pr[UU], w = f.w, bsq = f.bsq, eta = f.eta;
    StateBar a;
    bar_zero(a);
    flux_rev<0>(pr, q, gm.g, eta, f.K, ub, a);
    if (DIR != 0) {
        flux_rev<DIR>(pr, q, gm.g, eta, f.K, fb, a);
        // fast speeds: the roots of A v^2 - B v + C = 0 (forward in primtoflux)
        const double Acon_0 = gn[DIR], Asq = gn[DIR == 1 ? 4 : (DIR == 2 ? 7 : 9)], Bsq = gn[0], AB = Acon_0;
        const double rw = 1. / w, reta = 1. / eta;
        const double cs2 = gam * (gam - 1.) * u * rw;
        const double va2 = bsq * reta;
        double cms2 = cs2 + va2 - cs2 * va2;
        const bool cfree = !(cms2 < 0.) && !(cms2 > 1.);
        if (cms2 < 0.) cms2 = SMALL_D;
        if (cms2 > 1.) cms2 = 1.;
        const double Au = q.ucon[DIR], Bu = q.ucon[0];
        const double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
        const double A = Bu2 - (Bsq + Bu2) * cms2;
        const double B = 2. * (AuBu - (AB + AuBu) * cms2);
        const double C = Au2 - (Asq + Au2) * cms2;
        double discr = B * B - 4. * A * C;
        const bool dfree = !(discr < 0.);
        if (!dfree) discr = 0.;
        const double sq = d_sqrt(discr);
        const double rA = 1. / A, r2A = 0.5 * rA;
        const double vp = -(-B + sq) * r2A, vm = -(-B - sq) * r2A;
        const double vpb = (vp > vm ? cmxb : 0.) + (vp < vm ? cmnb : 0.);
        const double vmb = (vp > vm ? 0. : cmxb) + (vp < vm ? 0. : cmnb);
        double Bb = (vpb + vmb) * r2A;
        const double sb = (vmb - vpb) * r2A;
        double Ab = -(vpb * vp + vmb * vm) * rA, Cb = 0.;
        if (dfree && sq > 0.) {
            const double Db = 0.5 * sb / sq;
            Bb += 2. * B * Db;
            Ab -= 4. * C * Db;
            Cb = -4. * A * Db;
        }
        const double om = 1. - cms2;
        a.ucon[DIR] += 2. * Bu * om * Bb + 2. * Au * om * Cb;
        a.ucon[0] += 2. * Bu * om * Ab + 2. * Au * om * Bb;
        if (cfree) {
            const double cmsb = -(Bsq + Bu2) * Ab - 2. * (AB + AuBu) * Bb - (Asq + Au2) * Cb;
            // 1 - va2 = w / eta, without the cancellation where b^2 >> w
            const double cs2b = cmsb * (w * reta), va2b = cmsb * (1. - cs2);
            a.bsq += va2b * reta;
            a.eta -= va2b * va2 * reta;
            const double numb = cs2b * rw;
            a.w -= cs2b * cs2 * rw;
            a.u += numb * gam * (gam - 1.);
            a.gam += numb * u * (2. * gam - 1.);
        }
    }
    state_back(pr, gm, gam, f, a, pbar, gbar);
}

template <int DIR>
__device__ __forceinline__ void state_vjp(const double *pr, const Geo<double> &gm, double gam, const double *fb,
                                          const double *ub, double cmxb, double cmnb, double *pbar, double &gbar) {
    StateFwd f;
    state_fwd(pr, gm, gam, f, ub[KTOT] != 0. || (DIR != 0 && fb[KTOT] != 0.));
    state_vjp_from<DIR>(pr, gm, gam, f, fb, ub, cmxb, cmnb, pbar, gbar);
}

// geometric source of a state reversed (source in hamr_kernels.cu,
// GPU_phys_mhd.h:34-175): the cotangents wb of dU[UU..U3] give, through the
// connection, the cotangent of the stress tensor T^a_k = eta u^a u_k +
// ptot delta^a_k - b^a b_k, and from there the state's
__device__ void source_vjp(const double *pr, const Geo<double> &gm, double gam, const Dims &d, const Geom &m, long gi,
                           const double *wb, double *pbar, double &gbar) {
    StateFwd f;
    state_fwd(pr, gm, gam, f, false);   // the source has no entropy row
    const State<double> &q = f.q;
    StateBar a;
    bar_zero(a);
    const long gs = d.gs;
#pragma unroll
    for (int al = 0; al < 4; al++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double tb = 0.;
#pragma unroll
            for (int mm = 0; mm < 4; mm++) tb += wb[mm] * __ldg(&m.conn[(long)(sym4(mm, al) * 4 + k) * gs + gi]);
            tb *= gm.g;
            a.eta += tb * q.ucon[al] * q.ucov[k];
            a.ucon[al] += tb * f.eta * q.ucov[k];
            a.ucov[k] += tb * f.eta * q.ucon[al];
            if (al == k) a.ptot += tb;
            a.bcon[al] -= tb * q.bcov[k];
            a.bcov[k] -= tb * q.bcon[al];
        }
    state_back(pr, gm, gam, f, a, pbar, gbar);
}

// face fluxes of direction DIR, reversed: aF (cotangent of the fluxes) ->
// ap (primitives of the stencil, atomics), aps (normal face field), agam.
// A lane pair takes one face, one lane per side (s = 0 left, 1 right): each
// lane reconstructs its side, evaluates it, swaps the result with its
// partner for the HLL combination, reverses its side's state map by hand
// (state_vjp) and scatters over its PPM stencil, whose branch-local linear
// weights it takes from 5-direction dual numbers.
constexpr int FTEAM = 2;
template <int DIR>
__device__ __forceinline__ void adj_flux_face(const Dims &d, const Geom &m, const double *__restrict__ pv,
                                              const double *__restrict__ ps, const double *__restrict__ aF,
                                              double *ap, double *aps, long tt, double &gsum) {
    constexpr int idel = DIR == 1, jdel = DIR == 2, zdel = DIR == 3;
    const int lane = threadIdx.x & 31, side = lane & 1;
    const unsigned tm = 3u << (lane & ~1);   // this face's lane pair
    const long t = tt / FTEAM;
    if (t < n_faces<DIR>(d)) {
        const int i0 = (d.ng1 - 1) * d.d1 + idel, j0 = (d.ng2 - 1) * d.d2 + jdel, z0 = (d.ng3 - 1) * d.d3 + zdel;
        const int nj = d.n2 + 2 * d.d2 - jdel, nz = d.n3 + 2 * d.d3 - zdel;
        const int z = z0 + (int)(t % nz);
        const int j = j0 + (int)((t / nz) % nj);
        const int i = i0 + (int)(t / ((long)nz * nj));
        const long c = cix(d, i, j, z), ks = d.ks;
        const long stride = idel ? (long)d.G2 * d.G3 : (jdel ? (long)d.G3 : 1L);
        double Fb[NPR];
        bool any = false;
        for (int k = 0; k < NPR; k++) { Fb[k] = aF[k * ks + c]; any |= Fb[k] != 0.; }
        if (any) {   // uniform over the pair: same face
            const int face = DIR == 1 ? FACE1 : (DIR == 2 ? FACE2 : FACE3);
            const int bn = B1 + DIR - 1;
            const bool polefix = DIR == 2 && ((j == d.n2 + d.ng2 && d.pole2) || (j == d.ng2 && d.pole1));
            Geo<double> g0;
            load_geo(d, m, i, j, face, g0);
            // this side's reconstructed state: left = upper edge of the zone
            // below the face (stencil -3..1), right = lower edge of the zone
            // above it (stencil -2..2)
            double pme[NPR];
#pragma unroll
            for (int k = 0; k < ADJ_NP; k++) {
                const double *pk = pv + (long)k * ks + c + (side - 3) * stride;
                double x[5], lo, hi;
#pragma unroll
                for (int s = 0; s < 5; s++) x[s] = pk[s * stride];
                para(x, lo, hi);
                pme[k] = side ? lo : hi;
            }
            pme[bn] = ps[(long)(DIR - 1) * ks + c];
            if (polefix) pme[B1] = 0.;
            pme[KTOT] = 0.;   // read by no flux
            const double gam = d.gam;
            // this side's state, kept for the reverse; the entropy flux only
            // where its cotangent is nonzero
            StateFwd f;
            state_fwd(pme, g0, gam, f, Fb[KTOT] != 0.);
            double ta[NPR], tb[NPR], cmx_me, cmn_me, vd;
            primtoflux(gam, pme, f.q, DIR, g0, f.K, ta, &cmx_me, &cmn_me);
            primtoflux(gam, pme, f.q, 0, g0, f.K, tb, &vd, &vd);
            const double cmx_o = __shfl_xor_sync(tm, cmx_me, 1), cmn_o = __shfl_xor_sync(tm, cmn_me, 1);
            const double cmax_l = side ? cmx_o : cmx_me, cmin_l = side ? cmn_o : cmn_me;
            const double cmax_r = side ? cmx_me : cmx_o, cmin_r = side ? cmn_me : cmn_o;
            // HLL combination reversed (same max/abs selections as the forward)
            const double in_x = 0. > cmax_l ? 0. : cmax_l;
            const bool take_r = !(in_x > cmax_r);
            const double ox = take_r ? cmax_r : in_x;
            const double cmax = ox < 0. ? -ox : ox;
            const double in_n = 0. > -cmin_l ? 0. : -cmin_l;
            const bool take_rn = !(in_n > -cmin_r);
            const double on = take_rn ? -cmin_r : in_n;
            const double cmin = on < 0. ? -on : on;
            // (the cotangents need no bit-level agreement with a reference:
            // one reciprocal of the HLL denominator for all 45 quotients)
            const double rD = 1. / (cmax + cmin + SMALL_D);
            // this side's flux and conserved-variable cotangents, and the
            // speeds' (which need both sides' fluxes)
            double tfb[NPR], tub[NPR], cmaxb = 0., cminb = 0.;
#pragma unroll
            for (int k = 0; k < NPR; k++) {
                const double fo = __shfl_xor_sync(tm, ta[k], 1), uo = __shfl_xor_sync(tm, tb[k], 1);
                const double t1 = side ? fo : ta[k], t2 = side ? uo : tb[k];
                const double t3 = side ? ta[k] : fo, t4 = side ? tb[k] : uo;
                const double Fk = (cmax * t1 + cmin * t3 - cmax * cmin * (t4 - t2)) * rD;
                const double Fbr = Fb[k] * rD;
                tfb[k] = side ? Fbr * cmin : Fbr * cmax;
                tub[k] = side ? -Fbr * cmax * cmin : Fbr * cmax * cmin;
                cmaxb += Fbr * ((t1 - cmin * (t4 - t2)) - Fk);
                cminb += Fbr * ((t3 - cmax * (t4 - t2)) - Fk);
            }
            const double sx = ox < 0. ? -1. : 1., sn = on < 0. ? -1. : 1.;
            double cmxb = 0., cmnb = 0.;
            if (side) {
                if (take_r) cmxb = sx * cmaxb;
                if (take_rn) cmnb = -sn * cminb;
            } else {
                if (!take_r && !(0. > cmax_l)) cmxb = sx * cmaxb;
                if (!take_rn && !(0. > -cmin_l)) cmnb = -sn * cminb;
            }
            double pb[ADJ_NP];
            state_vjp_from<DIR>(pme, g0, gam, f, tfb, tub, cmxb, cmnb, pb, gsum);
            atomicAdd(&aps[(long)(DIR - 1) * ks + c], pb[bn]);
            // PPM stencil weights of this side, primitive by primitive
#pragma unroll 1
            for (int k = 0; k < ADJ_NP; k++) {
                if (k == bn || (polefix && k == B1) || pb[k] == 0.) continue;
                const double *pk = pv + (long)k * ks + c + (side - 3) * stride;
                double x[5], w[5];
#pragma unroll
                for (int s = 0; s < 5; s++) x[s] = pk[s * stride];
                para_weights(x, side == 0, w);   // left state: upper edge of the zone below
#pragma unroll
                for (int s = 0; s < 5; s++)
                    if (w[s] != 0.) atomicAdd(&ap[k * ks + c + (side + s - 3) * stride], pb[k] * w[s]);
            }
        }
    }
}

// both directions' faces in one launch (2-D: x1 then x2 faces), so that the
// two reverses, which only meet in atomics, fill the GPU together
// build options: minimum resident blocks of 128 threads per SM for the
// reverse kernels, which cap their registers: the 2-D torus gradient is
// latency bound at low occupancy, and spilling beats it (face reverse at 5
// blocks: 102 registers with spills against 230 without, 25 % on the whole
// gradient; the state kernels another 1-2 %)
#ifndef HAMR_ADJ_FLUX_MINB
#define HAMR_ADJ_FLUX_MINB 5
#endif
#ifndef HAMR_ADJ_ZONE_MINB
#define HAMR_ADJ_ZONE_MINB 4
#endif
__global__ void __launch_bounds__(BLK, HAMR_ADJ_FLUX_MINB) k_adj_flux12(const Dims d, const Geom m, const double *__restrict__ pv,
                                                     const double *__restrict__ ps, const double *__restrict__ aF1,
                                                     const double *__restrict__ aF2, double *ap, double *aps,
                                                     double *agam) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x, n1 = FTEAM * n_faces<1>(d);
    double gsum = 0.;
    if (t < n1) adj_flux_face<1>(d, m, pv, ps, aF1, ap, aps, t, gsum);
    else adj_flux_face<2>(d, m, pv, ps, aF2, ap, aps, t - n1, gsum);
    block_add(gsum, agam);
}

__device__ __forceinline__ bool active_zone(const Dims &d, int i, int j) {
    return i >= d.ng1 && i < d.ng1 + d.n1 && j >= d.ng2 && j < d.ng2 + d.n2;
}

// flux divergence reversed (2-D): aF(f) = Dt/dx (aW(f) - aW(f - s)) for every
// conserved component the inversion reads from the update (B1, B2 come from
// the faces instead); plus the accretion-rate objective on x1 face column ih
template <int DIR>
__device__ __forceinline__ void adj_divergence_face(const Dims &d, const double *__restrict__ aW, double *aF,
                                                    double Dt, int ih, double mdot_coef, long t) {
    constexpr int idel = DIR == 1, jdel = DIR == 2;
    const int i0 = (d.ng1 - 1) * d.d1 + idel, j0 = (d.ng2 - 1) * d.d2 + jdel;
    const int nj = d.n2 + 2 * d.d2 - jdel;
    const int j = j0 + (int)(t % nj);
    const int i = i0 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks;
    const long stride = idel ? (long)d.G2 * d.G3 : (long)d.G3;
    const double dx = DIR == 1 ? d.dx1 : d.dx2;
    const bool ac = active_zone(d, i, j), am = active_zone(d, i - idel, j - jdel);
    for (int k = 0; k < NPR; k++) {
        if (k == B1 || k == B2) continue;
        double v = 0.;
        if (ac) v += Dt * aW[k * ks + c] / dx;
        if (am) v -= Dt * aW[k * ks + c - stride] / dx;
        aF[k * ks + c] += v;
    }
    if (DIR == 1 && i == ih && j >= d.ng2 && j < d.ng2 + d.n2) aF[RHO * ks + c] += mdot_coef;
}

__global__ void k_adj_divergence12(const Dims d, const double *__restrict__ aW, double *aF1, double *aF2, double Dt,
                                   int ih, double mdot_coef) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x, n1 = n_faces<1>(d);
    if (t < n1) adj_divergence_face<1>(d, aW, aF1, Dt, ih, mdot_coef, t);
    else if (t < n1 + n_faces<2>(d)) adj_divergence_face<2>(d, aW, aF2, Dt, -1, 0., t - n1);
}

// inversion reversed by the implicit-function theorem (active zones).
// The solution p of the inversion satisfies G(p; W, B, gamma) = 0 with, over
// the five hydrodynamic primitives, the rows mass, energy and momenta
// (U(p) - W, when the Noble 2D solve converged) or the energy row replaced by
// the entropy relation u = K rho^gamma / (gamma - 1), K = W_KTOT / W_RHO
// (when an entropy fallback produced p). Then W_bar = -(dG/dW)^T x, with
// (dG/dp)^T x = p_bar, and likewise for the field and gamma. Where no solver
// converged, the hydrodynamic primitives are the guess's. ap: cotangent of
// the output (consumed); apg: of the guess; aW: of the conserved input.
__global__ void __launch_bounds__(BLK, HAMR_ADJ_ZONE_MINB - 1) k_adj_invert(const Dims d, const Geom m, const double *__restrict__ pout,
                                                     const double *__restrict__ pg, const double *__restrict__ W7,
                                                     const double *__restrict__ psf, const int *__restrict__ pflag,
                                                     const int *__restrict__ fail0, double *ap, double *apg,
                                                     double *aW, double *agam) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double gsum = 0.;
    if (t < (long)d.n1 * d.n2 * d.n3) {
        const int z = d.ng3 + (int)(t % d.n3);
        const int j = d.ng2 + (int)((t / d.n3) % d.n2);
        const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
        const long c = cix(d, i, j, z), gi = gix(d, i, j), ks = d.ks;
        double pb[NPR];
        bool any = false;
        for (int k = 0; k < NPR; k++) { pb[k] = ap[k * ks + c]; ap[k * ks + c] = 0.; any |= pb[k] != 0.; }
        if (any) {
            Geo<double> g0;
            load_geo(d, m, i, j, CENT, g0);
            apg[KTOT * ks + c] += pb[KTOT];
            for (int b = 0; b < 3; b++) aW[(B1 + b) * ks + c] += pb[B1 + b] / g0.g;
            if (pflag[c] != 0) {
                for (int k = 0; k < 5; k++) apg[k * ks + c] += pb[k];
            } else {
                // which solver produced p: the forward's count of primary
                // failures in this stage when recorded, else redo the primary
                // solve on the same input
                double U[NPR], pf[NPR];
                U[RHO] = W7[0 * ks + c];
                U[UU] = W7[1 * ks + c];
                U[U1] = W7[2 * ks + c];
                U[U2] = W7[3 * ks + c];
                U[U3] = W7[4 * ks + c];
                U[KTOT] = W7[5 * ks + c];
                U[B3] = W7[6 * ks + c];
                face_average_b(d, m, psf, i, j, c, gi, U);
                bool entropy_row;
                if (fail0) {
                    entropy_row = fail0[c] != 0;
                } else {
                    for (int k = 0; k < NPR; k++) pf[k] = pg[k * ks + c];
                    entropy_row = utoprim_2d(d.gam, U, g0.gcov, g0.gcon, g0.g, pf) != 0;
                }
                constexpr int N = ADJ_NP + 1;
                const Geo<double> &gm = g0;   // the metric is data: no derivative parts
                double pr[NPR];
                for (int k = 0; k < NPR; k++) pr[k] = pout[k * ks + c];
                Dual<N> pd[NPR], gd;
                seed_state(pr, d.gam, 0, pd, gd);
                State<Dual<N>> q;
                get_state(pd, gm, q);
                Dual<N> G[NPR], vd;
                primtoflux(gd, pd, q, 0, gm, entropy(gd, pd), G, &vd, &vd);
                const double K = U[KTOT] / U[RHO];
                double rg = 0.;   // rho^gamma / (gamma - 1) at the solution
                if (entropy_row) {
                    // u - K rho^gamma / (gamma - 1), K held (it is data)
                    const Dual<N> rgd = d_pow(pd[RHO], gd) / (gd - 1.);
                    G[UU] = pd[UU] - K * rgd;
                    rg = rgd.v;
                }
                // (dG/dp5)^T x = pb[0..4], Gaussian elimination with partial pivoting
                double A[5][6];
                for (int r = 0; r < 5; r++) {
                    for (int s2 = 0; s2 < 5; s2++) A[r][s2] = G[s2].d[r];
                    A[r][5] = pb[r];
                }
                bool ok = true;
                for (int col = 0; col < 5 && ok; col++) {
                    int piv = col;
                    for (int r = col + 1; r < 5; r++)
                        if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
                    if (!(fabs(A[piv][col]) > 0.)) { ok = false; break; }
                    if (piv != col)
                        for (int s2 = 0; s2 < 6; s2++) { const double tmp = A[col][s2]; A[col][s2] = A[piv][s2]; A[piv][s2] = tmp; }
                    for (int r = col + 1; r < 5; r++) {
                        const double f = A[r][col] / A[col][col];
                        for (int s2 = col; s2 < 6; s2++) A[r][s2] -= f * A[col][s2];
                    }
                }
                if (ok) {
                    double x[5];
                    for (int r = 4; r >= 0; r--) {
                        double v = A[r][5];
                        for (int s2 = r + 1; s2 < 5; s2++) v -= A[r][s2] * x[s2];
                        x[r] = v / A[r][r];
                    }
                    // -(dG/dW)^T x
                    aW[RHO * ks + c] += x[RHO];
                    for (int r = U1; r <= U3; r++) aW[r * ks + c] += x[r];
                    if (entropy_row) {
                        aW[KTOT * ks + c] += x[UU] * rg / U[RHO];
                        aW[RHO * ks + c] -= x[UU] * rg * U[KTOT] / (U[RHO] * U[RHO]);
                    } else {
                        aW[UU * ks + c] += x[UU];
                    }
                    // the field: p[B] = U[B]/gdet also moves the hydro solution
                    for (int b = 0; b < 3; b++) {
                        double v = 0.;
                        for (int r = 0; r < 5; r++) v += x[r] * G[r].d[B1 + b];
                        aW[(B1 + b) * ks + c] -= v / g0.g;
                    }
                    for (int r = 0; r < 5; r++) gsum -= x[r] * G[r].d[ADJ_NP];
                }
            }
        }
    }
    block_add(gsum, agam);
}

}  // namespace

namespace {

// source term reversed (active zones): ap += Dt (d dU / d pb)^T aW, agam;
// and the U^n cache: aU += aW
__global__ void __launch_bounds__(BLK, HAMR_ADJ_ZONE_MINB) k_adj_source(const Dims d, const Geom m, const double *__restrict__ pb,
                                                     const double *__restrict__ aW, double *ap, double *aU,
                                                     double Dt, double *agam) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double gsum = 0.;
    if (t < (long)d.n1 * d.n2 * d.n3) {
        const int z = d.ng3 + (int)(t % d.n3);
        const int j = d.ng2 + (int)((t / d.n3) % d.n2);
        const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
        const long c = cix(d, i, j, z), gi = gix(d, i, j), ks = d.ks;
        double wb[NPR];
        bool any = false;
        for (int k = 0; k < NPR; k++) { wb[k] = aW[k * ks + c]; any |= (k >= UU && k <= U3 && wb[k] != 0.); }
        // U^n feeds both sub-steps' updates: aU += aW over the components the
        // inversion reads from the update (not B1, B2, which come from the faces)
        for (int k = 0; k < NPR; k++)
            if (k != B1 && k != B2) aU[k * ks + c] += wb[k];
        if (any) {
            Geo<double> g0;
            load_geo(d, m, i, j, CENT, g0);
            double pr[NPR], pbar[ADJ_NP], gb = 0.;
            for (int k = 0; k < NPR; k++) pr[k] = pb[k * ks + c];
            const double w4[4] = {wb[UU], wb[U1], wb[U2], wb[U3]};
            source_vjp(pr, g0, d.gam, d, m, gi, w4, pbar, gb);
            for (int k = 0; k < ADJ_NP; k++) ap[k * ks + c] += Dt * pbar[k];
            gsum += Dt * gb;
        }
    }
    block_add(gsum, agam);
}

// conserved variables of a state reversed (U(p^n) cached by the half
// sub-step, active zones): ap += (dU/dp)^T aU, agam; aU consumed
__global__ void __launch_bounds__(BLK, HAMR_ADJ_ZONE_MINB) k_adj_cons_of_state(const Dims d, const Geom m, const double *__restrict__ pv,
                                                            double *aU, double *ap, double *agam) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double gsum = 0.;
    if (t < (long)d.n1 * d.n2 * d.n3) {
        const int z = d.ng3 + (int)(t % d.n3);
        const int j = d.ng2 + (int)((t / d.n3) % d.n2);
        const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
        const long c = cix(d, i, j, z), ks = d.ks;
        double ub[NPR];
        bool any = false;
        for (int k = 0; k < NPR; k++) { ub[k] = aU[k * ks + c]; aU[k * ks + c] = 0.; any |= ub[k] != 0.; }
        if (any) {
            Geo<double> g0;
            load_geo(d, m, i, j, CENT, g0);
            double pr[NPR], pb[ADJ_NP];
            for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + c];
            state_vjp<0>(pr, g0, d.gam, ub, ub, 0., 0., pb, gsum);
            for (int k = 0; k < ADJ_NP; k++) ap[k * ks + c] += pb[k];
        }
    }
    block_add(gsum, agam);
}

// centre EMF reversed (2-D: x3 component only; active zones plus one ring):
// ap += (d Ec3 / d p)^T aEc3
__global__ void __launch_bounds__(BLK) k_adj_emf_centre(const Dims d, const Geom m, const double *__restrict__ pv,
                                                         const double *__restrict__ aEc, double *ap) {
    const int ni = d.n1 + 2 * d.d1, nj = d.n2 + 2 * d.d2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj) return;
    const int j = (d.ng2 - d.d2) * d.d2 + (int)(t % nj);
    const int i = (d.ng1 - d.d1) * d.d1 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks;
    const double eb = aEc[3 * ks + c];
    if (eb == 0.) return;
    constexpr int N = 6;   // U1, U2, U3, B1, B2, B3
    Geo<double> g0;
    load_geo(d, m, i, j, CENT, g0);
    const Geo<double> &gm = g0;   // the metric is data: no derivative parts
    Dual<N> pd[NPR];
    for (int k = 0; k < NPR; k++) pd[k] = Dual<N>(pv[k * ks + c]);
    for (int q = 0; q < N; q++) pd[U1 + q].d[q] = 1.;
    Dual<N> ucon[4], ucov[4], bcon[4];
    ucon_calc(pd, gm, ucon);
    lower4(ucon, gm.gcov, ucov);
    bcon_calc(pd, ucon, ucov, bcon);
    const Dual<N> e3 = -gm.g * (ucon[1] * bcon[2] - ucon[2] * bcon[1]);
    for (int q = 0; q < N; q++) ap[(U1 + q) * ks + c] += eb * e3.d[q];
}

// edge EMF reversed (2-D: x3 component, upwind weights from the stage's
// mass fluxes): aemf3 -> aEc3, aF1[B2], aF2[B1] (atomics)
__global__ void k_adj_emf_edge(const Dims d, const double *__restrict__ F1, const double *__restrict__ F2,
                               const double *__restrict__ aemf, double *aEc, double *aF1, double *aF2) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj) return;
    const int j = d.ng2 * d.d2 + (int)(t % nj);
    const int i = d.ng1 * d.d1 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks, is = (long)d.G2 * d.G3, js = d.G3;
    if ((d.pole1 && j == d.ng2) || (d.pole2 && j == d.n2 + d.ng2)) return;   // e3 = 0 on the axis
    const double q = 0.25 * aemf[3 * ks + c];
    if (q == 0.) return;
    const double *F1r = F1 + RHO * ks, *F2r = F2 + RHO * ks;
    const double ua = F2r[c] <= 0., da = F2r[c] > 0.;
    const double ub = F2r[c - is] <= 0., db = F2r[c - is] > 0.;
    const double uc = F1r[c] <= 0., dc = F1r[c] > 0.;
    const double ud = F1r[c - js] <= 0., dd = F1r[c - js] > 0.;
    atomicAdd(&aF2[B1 * ks + c], q * (1. + uc + ud));
    atomicAdd(&aF2[B1 * ks + c - is], q * (1. + dc + dd));
    atomicAdd(&aF1[B2 * ks + c], q * (-1. - ua - ub));
    atomicAdd(&aF1[B2 * ks + c - js], q * (-1. - da - db));
    atomicAdd(&aEc[3 * ks + c], q * (-ua - uc));
    atomicAdd(&aEc[3 * ks + c - js], q * (-da - ud));
    atomicAdd(&aEc[3 * ks + c - is], q * (-ub - dc));
    atomicAdd(&aEc[3 * ks + c - is - js], q * (-db - dd));
}

// face update reversed (2-D), per edge: aemf3 from the cotangent of the
// updated faces apsf
__global__ void k_adj_face_update_emf(const Dims d, const Geom m, const double *__restrict__ apsf, double *aemf,
                                      double Dt) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj) return;
    const int j = d.ng2 + (int)(t % nj);
    const int i = d.ng1 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks, is = (long)d.G2 * d.G3, js = d.G3;
    auto f0 = [&](int ii, int jj) { return ii >= d.ng1 && ii <= d.n1 + d.ng1 && jj >= d.ng2 && jj < d.n2 + d.ng2; };
    auto f1 = [&](int ii, int jj) { return ii >= d.ng1 && ii < d.n1 + d.ng1 && jj >= d.ng2 && jj <= d.n2 + d.ng2; };
    auto g1 = [&](int ii, int jj) { return __ldg(&m.gdet[FACE1 * d.gs + gix(d, ii, jj)]); };
    auto g2 = [&](int ii, int jj) { return __ldg(&m.gdet[FACE2 * d.gs + gix(d, ii, jj)]); };
    double e = 0.;
    if (f0(i, j - 1)) e += apsf[c - js] * (-Dt / (d.dx2 * g1(i, j - 1)));
    if (f0(i, j)) e += apsf[c] * (Dt / (d.dx2 * g1(i, j)));
    if (f1(i - 1, j)) e += apsf[ks + c - is] * (Dt / (d.dx1 * g2(i - 1, j)));
    if (f1(i, j)) e += apsf[ks + c] * (-Dt / (d.dx1 * g2(i, j)));
    aemf[3 * ks + c] = e;
}

// half sub-step: ps^n -> psh is the identity on the updated faces
__global__ void k_adj_face_carry(const Dims d, double *apsh, double *aps) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj) return;
    const int j = d.ng2 + (int)(t % nj);
    const int i = d.ng1 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks;
    if (i <= d.n1 + d.ng1 && j < d.n2 + d.ng2) { aps[c] += apsh[c]; apsh[c] = 0.; }
    if (i < d.n1 + d.ng1 && j <= d.n2 + d.ng2) { aps[ks + c] += apsh[ks + c]; apsh[ks + c] = 0.; }
}

// U[B1], U[B2] from the face averages reversed (2-D), per face: aW -> apsf
__global__ void k_adj_face_average(const Dims d, const Geom m, const double *__restrict__ aW, double *apsf) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj) return;
    const int j = d.ng2 + (int)(t % nj);
    const int i = d.ng1 + (int)(t / nj);
    const long c = cix(d, i, j, 0), ks = d.ks, is = (long)d.G2 * d.G3, js = d.G3;
    double a = 0., b = 0.;
    if (active_zone(d, i, j)) { a += aW[B1 * ks + c]; b += aW[B2 * ks + c]; }
    if (active_zone(d, i - 1, j)) a += aW[B1 * ks + c - is];
    if (active_zone(d, i, j - 1)) b += aW[B2 * ks + c - js];
    if (a != 0.) apsf[c] += a * __ldg(&m.gdet[FACE1 * d.gs + gix(d, i, j)]) / 2.0;
    if (b != 0.) apsf[ks + c] += b * __ldg(&m.gdet[FACE2 * d.gs + gix(d, i, j)]) / 2.0;
}

// reflective-pole and radial flux fixes reversed (2-D); F holds the fixed fluxes
__global__ void k_adj_fix_flux(const Dims d, const double *__restrict__ F1, double *aF1, double *aF2) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long ks = d.ks;
    if (t < d.G1) {
        const int i = (int)t;
        if (!(i >= d.ng1 - d.d1 && i < d.n1 + d.ng1 + d.d1)) return;
        if (d.pole1) {
            const long g = cix(d, i, d.ng2 - 1, 0), a = cix(d, i, d.ng2, 0);
            aF1[B2 * ks + a] -= aF1[B2 * ks + g];
            aF1[B2 * ks + g] = 0.;
            for (int k = 0; k < NPR; k++) aF2[k * ks + a] = 0.;
        }
        if (d.pole2) {
            const long g = cix(d, i, d.n2 + d.ng2, 0), a = cix(d, i, d.n2 + d.ng2 - 1, 0);
            aF1[B2 * ks + a] -= aF1[B2 * ks + g];
            aF1[B2 * ks + g] = 0.;
            for (int k = 0; k < NPR; k++) aF2[k * ks + g] = 0.;
        }
        return;
    }
    const long u = t - d.G1;
    if (u >= d.G2) return;
    const int j = (int)u;
    if (!(j >= d.ng2 - d.d2 && j < d.n2 + d.ng2 + d.d2)) return;
    // clipped mass fluxes (stored as exactly 0) pass no cotangent
    const long ci = RHO * ks + cix(d, d.ng1, j, 0), co = RHO * ks + cix(d, d.n1 + d.ng1, j, 0);
    if (F1[ci] == 0.) aF1[ci] = 0.;
    if (F1[co] == 0.) aF1[co] = 0.;
}

}  // namespace

namespace {

// x2 reflective-axis ghost fill reversed (2-D), one item per (component, i)
// over the NPR primitives and face planes 0 and 2: ghost copies (with the
// sign flips) and the POLEFIX interpolation of the first two rows, in the
// reverse of the forward's order
constexpr int ADJ_X2_COMPS = NPR + 2;
__global__ void k_adj_bound_x2_refl(const Dims d, double *ap, double *aps) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ADJ_X2_COMPS * d.G1) return;
    const int i = (int)(t % d.G1), comp = (int)(t / d.G1), n2 = d.n2, ng = d.ng2, jref = 2;
    const bool face = comp >= NPR;
    const int k = face ? 2 * (comp - NPR) : comp;
    double *a = (face ? aps : ap) + (long)k * d.ks;
    auto C = [&](int j) { return cix(d, i, j, 0); };
    auto mv = [&](long dst, long src, double sgn) { a[src] += sgn * a[dst]; a[dst] = 0.; };
    const double sg = (!face && (k == U2 || k == B2)) ? -1. : 1.;
    const bool fixrow = !face && (k == RHO || k == UU || k == U1 || k == U3 || k == KTOT);
    const bool fixu2 = !face && k == U2;
    if (d.pole2) {
        for (int g = ng - 1; g >= 0; g--) mv(C(n2 + ng + g), C(n2 + ng - 1 - g), sg);
        for (int jj = jref - 1; jj >= 0; jj--) {
            const long c = C(n2 + ng - 1 - jj), r = C(n2 + ng - 1 - jref);
            if (fixu2) {
                a[r] += (jj + 0.5) / (jref + 0.5) * a[c];
                a[c] = 0.;
            } else if (fixrow) {
                mv(c, r, 1.);
            }
        }
    }
    if (d.pole1) {
        for (int g = ng; g >= 1; g--) mv(C(ng - g), C(ng + g - 1), sg);
        for (int jj = jref - 1; jj >= 0; jj--) {
            const long c = C(jj + ng), r = C(jref + ng);
            if (fixu2) {
                a[r] += (jj + 0.5) / (jref + 0.5) * a[c];
                a[c] = 0.;
            } else if (fixrow) {
                mv(c, r, 1.);
            }
        }
    }
}

// x1 outflow ghost fill reversed (2-D), one thread per (side, j): each ghost
// is the edge zone through the no-inflow check (a map of the velocities)
__global__ void k_adj_bound_x1_outflow(const Dims d, const Geom m, const double *__restrict__ pv, double *ap,
                                       double *aps) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2L * d.G2) return;
    const int side = (int)(t / d.G2), j = (int)(t % d.G2);
    const long ks = d.ks;
    const int iedge = side == 0 ? d.ng1 : d.n1 + d.ng1 - 1;
    const long src = cix(d, iedge, j, 0);
    double pr[NPR];
    for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + src];
    for (int g = 0; g < d.ng1; g++) {
        const int ig = side == 0 ? g : d.n1 + d.ng1 + g;
        const long dst = cix(d, ig, j, 0);
        double gb[NPR];
        bool any = false;
        for (int k = 0; k < NPR; k++) { gb[k] = ap[k * ks + dst]; ap[k * ks + dst] = 0.; any |= gb[k] != 0.; }
        aps[ks + src] += aps[ks + dst];
        aps[2 * ks + src] += aps[2 * ks + dst];
        aps[ks + dst] = aps[2 * ks + dst] = 0.;
        if (!any) continue;
        for (int k = 0; k < NPR; k++)
            if (k < U1 || k > U3) ap[k * ks + src] += gb[k];
        Geo<double> g0;
        load_geo(d, m, ig, j, CENT, g0);
        Dual<3> pd[NPR];
        for (int k = 0; k < NPR; k++) pd[k] = Dual<3>(pr[k]);
        for (int q = 0; q < 3; q++) pd[U1 + q].d[q] = 1.;
        inflow_check_t(pd, g0, side);
        for (int q = 0; q < 3; q++) {
            double s = 0.;
            for (int k = U1; k <= U3; k++) s += gb[k] * pd[k].d[q];
            ap[(U1 + q) * ks + src] += s;
        }
    }
}

// J contribution of one step: w * Mdot, Mdot = - sum_j F1[RHO](ih, j) dx2 dx3
// one CTA of BLK threads: the column's terms summed in a fixed order (strided
// partial sums, then a tree in shared memory), so that the objective does not
// depend on the order in which atomics land
__global__ void k_mdot_accum(const Dims d, const double *__restrict__ F1, int ih, double w, double *J) {
    __shared__ double part[BLK];
    double v = 0.;
    for (int t = threadIdx.x; t < d.n2; t += BLK)
        v += -w * F1[RHO * d.ks + cix(d, ih, d.ng2 + t, 0)] * d.dx2 * d.dx3;
    part[threadIdx.x] = v;
    __syncthreads();
    for (int s = BLK / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *J += part[0];
}

}  // namespace

// ===========================================================================
struct hamr_adjoint {
    hamr_ctx *ctx = nullptr;
    int ih = 0;                 // x1 face column of the accretion-rate objective
    std::string err;
    // cotangents (device): of p, ps (the state), ph, psh, U^n, the conserved
    // update W (9 planes), fluxes, centre and edge EMFs
    double *ap = nullptr, *aps = nullptr, *aph = nullptr, *apsh = nullptr, *aU = nullptr, *aW = nullptr;
    double *aF1 = nullptr, *aF2 = nullptr, *aF3 = nullptr, *aEc = nullptr, *aemf = nullptr;
    double *agam = nullptr, *J = nullptr;   // 1 double each
    double *p0 = nullptr, *ps0 = nullptr;   // the step's input state while it is reversed
    std::vector<double *> store;            // checkpoints (12 planes each)
    std::vector<double *> slots;            // two banks of per-step records (REC_PLANES each)
    double *ends[2] = {nullptr, nullptr};   // per bank: the state a segment ends in (12 planes)
    int bank_len = 0;                       // records per bank
    // segments are recomputed on s2 while the previous one is reversed on the
    // context's stream; events order the two over the banks
    cudaStream_t s2 = nullptr;
    cudaEvent_t ev_sweep = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr};
    // captured graphs, per step size and record slot: a forward step with the
    // objective term, a recorded forward step, a reversed step
    using Key = std::tuple<double, const void *, const void *>;
    std::map<Key, cudaGraphExec_t> fwd_graph, rec_graph, bwd_graph;
};

namespace {

int afail(hamr_adjoint *a, cudaError_t e, const char *what) {
    a->err = std::string(what) + ": " + cudaGetErrorString(e);
    return HAMR_E_CUDA;
}

#define ACK(call)                                               \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return afail(a, e_, #call);      \
    } while (0)

// one RK2 step of the context with a fixed dt (no step-size bookkeeping)
int fixed_step(hamr_ctx *ctx, double dt) {
    k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
    return launch_step(ctx, StepSize{nullptr, 0.5, 0.5 * dt, dt}, StepSize{nullptr, 1.0, dt, dt}, nullptr, 0);
}

unsigned nb(long n) { return (unsigned)((n + BLK - 1) / BLK); }

// reverse of one ghost fill (x2 first: the forward fills x1, then x2)
void adj_bound(hamr_ctx *ctx, const double *pv, double *ap, double *aps) {
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    k_adj_bound_x2_refl<<<nb((long)ADJ_X2_COMPS * d.G1), BLK, 0, s>>>(d, ap, aps);
    k_adj_bound_x1_outflow<<<nb(2L * d.G2), BLK, 0, s>>>(d, geom_of(ctx), pv, ap, aps);
}

// what the reverse of one sub-step reads of its forward: input and output
// primitives (ghost-filled) and face fields, the conserved update handed to
// the inversion, the fixed face fluxes and the inversion's solver flags
struct StageRec {
    const double *pin, *pout, *psin, *psout, *W, *F1, *F2;
    const int *pflag;
    const int *fail0;   // primary-solver failures of this stage (nullptr: not recorded)
};

// the stage just run by the context, read from its own buffers
StageRec ctx_stage(const hamr_ctx *ctx, int full) {
    return full ? StageRec{ctx->ph, ctx->p, ctx->psh, ctx->ps, ctx->W, ctx->F1, ctx->F2, ctx->pflag, nullptr}
                : StageRec{ctx->p, ctx->ph, ctx->ps, ctx->psh, ctx->W, ctx->F1, ctx->F2, ctx->pflag, nullptr};
}

// reverse of one sub-step. apin/apsin: cotangents of the stage's input
// primitives and faces (accumulated); apout: of the inversion output
// (consumed); apsout: of the face field it writes.
int adj_stage(hamr_adjoint *a, int full, double dt, double mdot_coef, const StageRec &r) {
    hamr_ctx *ctx = a->ctx;
    const Dims &d = ctx->d;
    const Geom m = geom_of(ctx);
    cudaStream_t s = ctx->stream;
    const double Dt = full ? dt : 0.5 * dt;
    double *apin = full ? a->aph : a->ap, *apsin = full ? a->apsh : a->aps;
    double *apout = full ? a->ap : a->aph, *apsout = full ? a->aps : a->apsh;
    const long ks = d.ks, nz = (long)d.n1 * d.n2, nedge = (long)(d.n1 + 1) * (d.n2 + 1);
    ACK(cudaMemsetAsync(a->aW, 0, NPR * sizeof(double) * ks, s));
    ACK(cudaMemsetAsync(a->aF1, 0, NPR * sizeof(double) * ks, s));
    ACK(cudaMemsetAsync(a->aF2, 0, NPR * sizeof(double) * ks, s));
    ACK(cudaMemsetAsync(a->aEc, 0, 4 * sizeof(double) * ks, s));
    // ghost fill of the output, then the inversion (p_out <- W, guess pin)
    adj_bound(ctx, r.pout, apout, apsout);
    k_adj_invert<<<nb(nz), BLK, 0, s>>>(d, m, r.pout, r.pin, r.W, r.psout, r.pflag, r.fail0, apout, apin, a->aW,
                                        a->agam);
    // U[B1], U[B2] from the updated faces
    k_adj_face_average<<<nb(nedge), BLK, 0, s>>>(d, m, a->aW, apsout);
    // update: U^n (cache), source at pin, flux divergence (+ objective)
    k_adj_source<<<nb(nz), BLK, 0, s>>>(d, m, r.pin, a->aW, apin, a->aU, Dt, a->agam);
    k_adj_divergence12<<<nb(n_faces<1>(d) + n_faces<2>(d)), BLK, 0, s>>>(d, a->aW, a->aF1, a->aF2, Dt, a->ih,
                                                                        full ? mdot_coef : 0.);
    // face update: edge EMFs; ps^n -> psh carries the cotangent over
    k_adj_face_update_emf<<<nb(nedge), BLK, 0, s>>>(d, m, apsout, a->aemf, Dt);
    if (!full) k_adj_face_carry<<<nb(nedge), BLK, 0, s>>>(d, a->apsh, a->aps);
    // edge EMFs -> centre EMFs and fluxes; centre EMFs -> pin
    k_adj_emf_edge<<<nb(nedge), BLK, 0, s>>>(d, r.F1, r.F2, a->aemf, a->aEc, a->aF1, a->aF2);
    k_adj_emf_centre<<<nb((long)(d.n1 + 2) * (d.n2 + 2)), BLK, 0, s>>>(d, m, r.pin, a->aEc, apin);
    // flux fixes, then the face fluxes -> pin (and the normal face field)
    k_adj_fix_flux<<<nb((long)d.G1 + d.G2), BLK, 0, s>>>(d, r.F1, a->aF1, a->aF2);
    k_adj_flux12<<<nb(FTEAM * (n_faces<1>(d) + n_faces<2>(d))), BLK, 0, s>>>(d, m, r.pin, r.psin, a->aF1, a->aF2,
                                                                            apin, apsin, a->agam);
    ACK(cudaGetLastError());
    return HAMR_OK;
}

// One step's record, REC_PLANES planes of the block: its input state (p, ps),
// the half sub-step's output (ph, psh), each sub-step's conserved update,
// fixed x1/x2 fluxes, solver flags (the two int planes share one) and
// solver-failure counts (4 int planes per sub-step, plane 0 = primary).
constexpr int REC_PLANES = 79;
struct Slot {
    double *p, *ps, *ph, *psh, *Wh, *Wf, *F1h, *F2h, *F1f, *F2f;
    int *flh, *flf, *fih, *fif;
};
Slot slot_of(double *base, long ks) {
    Slot r;
    r.p = base; r.ps = base + 9 * ks; r.ph = base + 12 * ks; r.psh = base + 21 * ks;
    r.Wh = base + 24 * ks; r.Wf = base + 31 * ks;
    r.F1h = base + 38 * ks; r.F2h = base + 47 * ks; r.F1f = base + 56 * ks; r.F2f = base + 65 * ks;
    r.flh = reinterpret_cast<int *>(base + 74 * ks); r.flf = r.flh + ks;
    r.fih = reinterpret_cast<int *>(base + 75 * ks); r.fif = r.fih + 4 * ks;
    return r;
}

// one fixed-size step from the record's input state (r.p, r.ps) to
// (next_p, next_ps) that leaves its intermediates in the record: the stages
// write their half-step state, updates, fluxes, flags and solver-failure
// counts straight into the slot. The context's buffer pointers are swapped
// for these while the launches are issued and put back after, so the
// context's own state, and its failure counts, do not see these replays of
// steps the forward sweep already took. The full sub-step updates the faces
// in place, so they are copied to next_ps first; it reads no p^n (the half
// sub-step cached U^n), so p^{n+1} goes straight to next_p.
int record_step(hamr_adjoint *a, double dt, const Slot &r, double *next_p, double *next_ps) {
    hamr_ctx *ctx = a->ctx;
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    const size_t cb = sizeof(double) * d.ks;
    ACK(cudaMemsetAsync(r.fih, 0, 8 * sizeof(int) * d.ks, s));
    ACK(cudaMemcpyAsync(next_ps, r.ps, 3 * cb, cudaMemcpyDeviceToDevice, s));
    struct Swap {
        hamr_ctx *c;
        double *p, *ps, *ph, *psh, *W, *F1, *F2;
        int *pflag, *failimage;
        ~Swap() {
            c->p = p; c->ps = ps; c->ph = ph; c->psh = psh; c->W = W; c->F1 = F1; c->F2 = F2;
            c->pflag = pflag; c->failimage = failimage;
        }
    } keep{ctx, ctx->p, ctx->ps, ctx->ph, ctx->psh, ctx->W, ctx->F1, ctx->F2, ctx->pflag, ctx->failimage};
    ctx->p = r.p; ctx->ps = r.ps; ctx->ph = r.ph; ctx->psh = r.psh;
    ctx->W = r.Wh; ctx->F1 = r.F1h; ctx->F2 = r.F2h; ctx->pflag = r.flh; ctx->failimage = r.fih;
    int rc = launch_stage(ctx, 0, StepSize{nullptr, 0.5, 0.5 * dt, dt}, false);
    if (rc) return rc;
    ctx->p = next_p; ctx->ps = next_ps;
    ctx->W = r.Wf; ctx->F1 = r.F1f; ctx->F2 = r.F2f; ctx->pflag = r.flf; ctx->failimage = r.fif;
    return launch_stage(ctx, 1, StepSize{nullptr, 1.0, dt, dt}, false);
}

// reverse of a whole step from the records of its two sub-steps
int adj_step(hamr_adjoint *a, double dt, double w, const StageRec &half, const StageRec &full) {
    hamr_ctx *ctx = a->ctx;
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    const size_t cb = sizeof(double) * d.ks;
    ACK(cudaMemsetAsync(a->aph, 0, NPR * cb, s));
    ACK(cudaMemsetAsync(a->apsh, 0, 3 * cb, s));
    int rc = adj_stage(a, 1, dt, -w * d.dx2 * d.dx3, full);
    if (rc) return rc;
    if ((rc = adj_stage(a, 0, dt, 0., half))) return rc;
    k_adj_cons_of_state<<<nb((long)d.n1 * d.n2), BLK, 0, s>>>(d, geom_of(ctx), half.pin, a->aU, a->ap, a->agam);
    ACK(cudaGetLastError());
    return HAMR_OK;
}

}  // namespace

namespace {

// reverse of the step taken from the context's current state, recomputing
// its forward: the full sub-step is reversed from the context's buffers right
// after the step, the half sub-step after re-running it from the saved input
int step_backward(hamr_adjoint *a, double dt, double w) {
    hamr_ctx *ctx = a->ctx;
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    const size_t cb = sizeof(double) * d.ks;
    ACK(cudaMemcpyAsync(a->p0, ctx->p, NPR * cb, cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(a->ps0, ctx->ps, 3 * cb, cudaMemcpyDeviceToDevice, s));
    int rc = fixed_step(ctx, dt);
    if (rc) return rc;
    ACK(cudaMemsetAsync(a->aph, 0, NPR * cb, s));
    ACK(cudaMemsetAsync(a->apsh, 0, 3 * cb, s));
    if ((rc = adj_stage(a, 1, dt, -w * d.dx2 * d.dx3, ctx_stage(ctx, 1)))) return rc;
    ACK(cudaMemcpyAsync(ctx->p, a->p0, NPR * cb, cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(ctx->ps, a->ps0, 3 * cb, cudaMemcpyDeviceToDevice, s));
    if ((rc = launch_stage(ctx, 0, StepSize{nullptr, 0.5, 0.5 * dt, dt}, false))) return rc;
    if ((rc = adj_stage(a, 0, dt, 0., ctx_stage(ctx, 0)))) return rc;
    k_adj_cons_of_state<<<nb((long)d.n1 * d.n2), BLK, 0, s>>>(d, geom_of(ctx), ctx->p, a->aU, a->ap, a->agam);
    ACK(cudaGetLastError());
    return HAMR_OK;
}

// forward step + objective term, and reversed step, replayed from graphs
// captured once per step size (the step is launch-bound at these sizes)
// (captured on the context's stream, where the body issues its work, and
// launched on `run`)
template <class F>
int graph_run(hamr_adjoint *a, std::map<hamr_adjoint::Key, cudaGraphExec_t> &cache, hamr_adjoint::Key key,
              cudaStream_t run, F body) {
    cudaStream_t s = a->ctx->stream;
    auto it = cache.find(key);
    if (it == cache.end()) {
        cudaGraph_t g;
        ACK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = body();
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return afail(a, e, "cudaStreamEndCapture");
        cudaGraphExec_t x;
        e = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return afail(a, e, "cudaGraphInstantiate");
        it = cache.emplace(key, x).first;
    }
    ACK(cudaGraphLaunch(it->second, run));
    return HAMR_OK;
}

int fwd_step(hamr_adjoint *a, double dt) {
    return graph_run(a, a->fwd_graph, {dt, nullptr, nullptr}, a->ctx->stream, [&]() -> int {
        const int rc = fixed_step(a->ctx, dt);
        if (rc) return rc;
        k_mdot_accum<<<1, BLK, 0, a->ctx->stream>>>(a->ctx->d, a->ctx->F1, a->ih, dt, a->J);
        return cudaGetLastError() == cudaSuccess ? HAMR_OK : HAMR_E_CUDA;
    });
}

// recorded step on the second stream; next_p/next_ps: where its output goes
int rec_step(hamr_adjoint *a, double dt, double *slot, double *next_p, double *next_ps) {
    return graph_run(a, a->rec_graph, {dt, slot, next_p}, a->s2, [&]() -> int {
        return record_step(a, dt, slot_of(slot, a->ctx->d.ks), next_p, next_ps);
    });
}

// reversed step from slot's record; next_p/next_ps: the step's output state
int bwd_step(hamr_adjoint *a, double dt, double *slot, const double *next_p, const double *next_ps) {
    return graph_run(a, a->bwd_graph, {dt, slot, next_p}, a->ctx->stream, [&]() -> int {
        const Slot r = slot_of(slot, a->ctx->d.ks);
        const StageRec half{r.p, r.ph, r.ps, r.psh, r.Wh, r.F1h, r.F2h, r.flh, r.fih};
        const StageRec full{r.ph, next_p, r.psh, next_ps, r.Wf, r.F1f, r.F2f, r.flf, r.fif};
        return adj_step(a, dt, dt, half, full);
    });
}

int bound_ctx(hamr_ctx *ctx) {
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    const Geom m = geom_of(ctx);
    if (d.d1) k_bound_x1<<<nblk((long)d.ng1 * d.G2 * d.G3), BLK, 0, s>>>(d, m, ctx->p, ctx->ps);
    if (d.d3) k_bound_x3<<<nblk(n_bound_x3(d)), BLK, 0, s>>>(d, ctx->p, ctx->ps);
    if (d.d2) k_bound_x2<<<nblk(n_bound_x2(d)), BLK, 0, s>>>(d, ctx->p, ctx->ps);
    return cudaGetLastError() == cudaSuccess ? HAMR_OK : HAMR_E_CUDA;
}

}  // namespace

extern "C" {

int hamr_adjoint_create(hamr_ctx *ctx, int mdot_face, hamr_adjoint **out) {
    if (!ctx || !out) return HAMR_E_ARG;
    *out = nullptr;
    const hamr_params &p = ctx->prm;
    const Dims &d = ctx->d;
    // the configuration the reverse kernels are written for
    if (p.precision != HAMR_FP64 || p.recon != HAMR_RECON_PPM || p.inversion != HAMR_INV_2D || d.n3 != 1 ||
        p.riemann != HAMR_RIEMANN_HLL || p.halo || p.floors || p.repair ||
        p.ng != 3 || p.bc1 != HAMR_BC_OUTFLOW || p.bc2 != HAMR_BC_POLE_REFL || !p.ct_upwind)
        return HAMR_E_ARG;
    if (mdot_face <= d.ng1 || mdot_face >= d.n1 + d.ng1) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    hamr_adjoint *a = new hamr_adjoint();
    a->ctx = ctx;
    a->ih = mdot_face;
    const size_t cb = sizeof(double) * d.ks;
    struct A { double **p; size_t n; } al[] = {
        {&a->ap, NPR * cb}, {&a->aps, 3 * cb}, {&a->aph, NPR * cb}, {&a->apsh, 3 * cb}, {&a->aU, NPR * cb},
        {&a->aW, NPR * cb}, {&a->aF1, NPR * cb}, {&a->aF2, NPR * cb}, {&a->aF3, NPR * cb}, {&a->aEc, 4 * cb},
        {&a->aemf, 4 * cb}, {&a->agam, sizeof(double)}, {&a->J, sizeof(double)}, {&a->p0, NPR * cb},
        {&a->ps0, 3 * cb}};
    for (auto &x : al) {
        if (cudaMalloc((void **)x.p, x.n) != cudaSuccess) {
            hamr_adjoint_destroy(a);
            return HAMR_E_NOMEM;
        }
        cudaMemsetAsync(*x.p, 0, x.n, ctx->stream);
    }
    bool ok = cudaStreamCreateWithFlags(&a->s2, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t *e : {&a->ev_sweep, &a->ev_rec[0], &a->ev_rec[1], &a->ev_rev[0], &a->ev_rev[1]})
        ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
    if (!ok || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        hamr_adjoint_destroy(a);
        return HAMR_E_CUDA;
    }
    *out = a;
    return HAMR_OK;
}

int hamr_adjoint_destroy(hamr_adjoint *a) {
    if (!a) return HAMR_E_ARG;
    if (a->ctx && a->ctx->stream) cudaStreamSynchronize(a->ctx->stream);
    for (double *p : {a->ap, a->aps, a->aph, a->apsh, a->aU, a->aW, a->aF1, a->aF2, a->aF3, a->aEc, a->aemf,
                      a->agam, a->J, a->p0, a->ps0})
        cudaFree(p);
    if (a->s2) cudaStreamSynchronize(a->s2);
    for (double *p : a->store) cudaFree(p);
    for (double *p : a->slots) cudaFree(p);
    for (double *p : a->ends) cudaFree(p);
    for (cudaEvent_t e : {a->ev_sweep, a->ev_rec[0], a->ev_rec[1], a->ev_rev[0], a->ev_rev[1]})
        if (e) cudaEventDestroy(e);
    if (a->s2) cudaStreamDestroy(a->s2);
    for (auto *g : {&a->fwd_graph, &a->rec_graph, &a->bwd_graph})
        for (auto &kv : *g) cudaGraphExecDestroy(kv.second);
    delete a;
    return HAMR_OK;
}

const char *hamr_adjoint_last_error(hamr_adjoint *a) { return a ? a->err.c_str() : "null adjoint"; }

int hamr_adjoint_cotangent(hamr_adjoint *a, double **ap, double **aps, double **agam) {
    if (!a) return HAMR_E_ARG;
    if (ap) *ap = a->ap;
    if (aps) *aps = a->aps;
    if (agam) *agam = a->agam;
    return HAMR_OK;
}

int hamr_adjoint_zero(hamr_adjoint *a) {
    if (!a) return HAMR_E_ARG;
    const size_t cb = sizeof(double) * a->ctx->d.ks;
    cudaStream_t s = a->ctx->stream;
    ACK(cudaMemsetAsync(a->ap, 0, NPR * cb, s));
    ACK(cudaMemsetAsync(a->aps, 0, 3 * cb, s));
    ACK(cudaMemsetAsync(a->aU, 0, NPR * cb, s));
    ACK(cudaMemsetAsync(a->agam, 0, sizeof(double), s));
    return HAMR_OK;
}

int hamr_step_backward(hamr_adjoint *a, double dt, double mdot_weight) {
    if (!a || !(dt > 0)) return HAMR_E_ARG;
    return step_backward(a, dt, mdot_weight);
}

int hamr_mdot_forward(hamr_adjoint *a, int nsteps, const double *dt, double *J) {
    if (!a || !dt || nsteps < 1) return HAMR_E_ARG;
    hamr_ctx *ctx = a->ctx;
    cudaStream_t s = ctx->stream;
    ACK(cudaMemsetAsync(a->J, 0, sizeof(double), s));
    int rc = bound_ctx(ctx);
    for (int n = 0; n < nsteps && rc == HAMR_OK; n++) {
        if (!(dt[n] > 0)) return HAMR_E_ARG;
        rc = fwd_step(a, dt[n]);
    }
    if (rc) return rc;
    if (J) ACK(cudaMemcpyAsync(J, a->J, sizeof(double), cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    return HAMR_OK;
}

// Gradient of J = sum_n dt[n] Mdot_n over nsteps fixed-size steps with
// respect to the initial state (active primitives and face field, before
// the ghost fill) and the adiabatic index. Checkpoints the state every
// `every` steps on the forward sweep, and reverses segment by segment: each
// segment is recomputed from its checkpoint, recording every step's
// intermediates, then its steps are reversed from those records (no forward
// work in the reverse). Two banks of records let segment sg-1 be recomputed
// on a second stream while segment sg is reversed on the context's stream.
// grad_p (9 planes) / grad_ps (3 planes) are host arrays in the context's
// layout (NULL: not copied). The context's state is restored to its initial
// value on return.
int hamr_adjoint_run(hamr_adjoint *a, int nsteps, const double *dt, int every, double *J, double *grad_p,
                     double *grad_ps, double *grad_gam) {
    if (!a || !dt || nsteps < 1 || every < 1) return HAMR_E_ARG;
    for (int n = 0; n < nsteps; n++)
        if (!(dt[n] > 0)) return HAMR_E_ARG;
    hamr_ctx *ctx = a->ctx;
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    const size_t cb = sizeof(double) * d.ks, state = 12 * cb;
    const int nseg = (nsteps + every - 1) / every;
    const int seglen = every < nsteps ? every : nsteps;
    while (a->store.size() < (size_t)nseg + 1) {   // checkpoints + the initial pre-fill copy
        double *p = nullptr;
        if (cudaMalloc((void **)&p, state) != cudaSuccess) return HAMR_E_NOMEM;
        a->store.push_back(p);
    }
    if (a->bank_len < seglen) {   // (re)allocate both banks for the longer segment
        ACK(cudaStreamSynchronize(s));
        ACK(cudaStreamSynchronize(a->s2));
        for (double *p : a->slots) cudaFree(p);
        a->slots.clear();
        for (auto *g : {&a->rec_graph, &a->bwd_graph}) {
            for (auto &kv : *g) cudaGraphExecDestroy(kv.second);
            g->clear();
        }
        a->bank_len = 0;
        for (int k = 0; k < 2 * seglen; k++) {
            double *p = nullptr;
            if (cudaMalloc((void **)&p, REC_PLANES * cb) != cudaSuccess) return HAMR_E_NOMEM;
            a->slots.push_back(p);
        }
        for (double *&e : a->ends)
            if (!e && cudaMalloc((void **)&e, state) != cudaSuccess) return HAMR_E_NOMEM;
        a->bank_len = seglen;
    }
    auto save = [&](double *dst) {
        cudaMemcpyAsync(dst, ctx->p, NPR * cb, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(dst + NPR * d.ks, ctx->ps, 3 * cb, cudaMemcpyDeviceToDevice, s);
    };
    auto load = [&](const double *src) {
        cudaMemcpyAsync(ctx->p, src, NPR * cb, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(ctx->ps, src + NPR * d.ks, 3 * cb, cudaMemcpyDeviceToDevice, s);
    };
    double *initial = a->store[nseg];
    save(initial);
    // forward sweep with checkpoints
    ACK(cudaMemsetAsync(a->J, 0, sizeof(double), s));
    int rc = bound_ctx(ctx);
    for (int n = 0; n < nsteps && rc == HAMR_OK; n++) {
        if (n % every == 0) save(a->store[n / every]);
        rc = fwd_step(a, dt[n]);
    }
    if (rc) return rc;
    double Jval = 0.;
    ACK(cudaMemcpyAsync(&Jval, a->J, sizeof(double), cudaMemcpyDeviceToHost, s));
    ACK(cudaEventRecord(a->ev_sweep, s));
    ACK(cudaStreamWaitEvent(a->s2, a->ev_sweep, 0));
    if ((rc = hamr_adjoint_zero(a))) return rc;
    // segment sg uses bank sg % 2: record k of the segment is slot k of the
    // bank, and its last step ends in the bank's `ends` state
    auto slot = [&](int b, int k) { return a->slots[(size_t)b * a->bank_len + k]; };
    auto recompute = [&](int sg) -> int {
        const int b = sg & 1, n0 = sg * every, n1 = n0 + every < nsteps ? n0 + every : nsteps;
        ACK(cudaStreamWaitEvent(a->s2, a->ev_rev[b], 0));   // the bank's previous segment is reversed
        const double *src = a->store[sg];
        ACK(cudaMemcpyAsync(slot(b, 0), src, state, cudaMemcpyDeviceToDevice, a->s2));
        for (int n = n0; n < n1; n++) {
            const int k = n - n0;
            double *nx = n + 1 < n1 ? slot(b, k + 1) : a->ends[b];
            const int r = rec_step(a, dt[n], slot(b, k), nx, nx + NPR * d.ks);
            if (r) return r;
        }
        ACK(cudaEventRecord(a->ev_rec[b], a->s2));
        return HAMR_OK;
    };
    auto reverse = [&](int sg) -> int {
        const int b = sg & 1, n0 = sg * every, n1 = n0 + every < nsteps ? n0 + every : nsteps;
        ACK(cudaStreamWaitEvent(s, a->ev_rec[b], 0));
        for (int n = n1 - 1; n >= n0; n--) {
            const int k = n - n0;
            const double *nx = n + 1 < n1 ? slot(b, k + 1) : a->ends[b];
            const int r = bwd_step(a, dt[n], slot(b, k), nx, nx + NPR * d.ks);
            if (r) return r;
        }
        ACK(cudaEventRecord(a->ev_rev[b], s));
        return HAMR_OK;
    };
    rc = recompute(nseg - 1);
    for (int sg = nseg - 1; sg >= 0 && rc == HAMR_OK; sg--) {
        if (sg >= 1 && (rc = recompute(sg - 1))) break;
        rc = reverse(sg);
    }
    if (rc) {
        cudaStreamSynchronize(a->s2);
        return rc;
    }
    // the initial ghost fill, reversed, folds ghost cotangents onto the zones
    load(a->store[0]);
    adj_bound(ctx, ctx->p, a->ap, a->aps);
    ACK(cudaGetLastError());
    if (J) *J = Jval;
    if (grad_p) ACK(cudaMemcpyAsync(grad_p, a->ap, NPR * cb, cudaMemcpyDeviceToHost, s));
    if (grad_ps) ACK(cudaMemcpyAsync(grad_ps, a->aps, 3 * cb, cudaMemcpyDeviceToHost, s));
    if (grad_gam) ACK(cudaMemcpyAsync(grad_gam, a->agam, sizeof(double), cudaMemcpyDeviceToHost, s));
    load(initial);
    ACK(cudaStreamSynchronize(s));
    return HAMR_OK;
}

}  // extern "C"
