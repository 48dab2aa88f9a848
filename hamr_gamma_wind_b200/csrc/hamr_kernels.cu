// sm_100a kernels of the single-block RK2 sub-step and the C ABI
// (include/hamr_b200.h) that drives them.
//
// One sub-step (the work of advance_GPU, step_ch.c:997-1335, for one block):
//   k_flux<3>, k_flux<2>, k_flux<1>   PPM + HLL face fluxes and the directional
//                                      CFL minimum (fluxcalcprep + fluxcalc2D2)
//   k_fix_flux                         reflective-pole flux rules (2-D)
//   k_emf_centre, k_emf_edge           cell-centre and edge EMFs (consttransport1/2)
//   k_pole_average                     phi-averaged polar EMF (E_average, 3-D)
//   k_face_update                      staggered B update (consttransport3)
//   k_cons, k_invert                   conserved update + source, inversion (fixup)
//   k_bound_x1/x3/x2                   ghost fill of the written state
// All arrays use the reference's structure-of-arrays layout; cell index
// (i*G2 + j)*G3 + z puts phi (or x3) innermost, so consecutive threads touch
// consecutive addresses.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/hamr_b200.h"
#include "hamr_physics.cuh"

using namespace hamr;

namespace {

constexpr int BLK = 128;
// CTAs of the inversion's fallback pass (a grid-stride loop over the failed
// zones, whose count is only known on the device)
constexpr int FALLBACK_CTAS = 148;

struct Dims {
    int n1, n2, n3, ng1, ng2, ng3, G1, G2, G3, d1, d2, d3;
    long ks, gs;
    double dx1, dx2, dx3, gam, cour;
    double rdx1, rdx2, rdx3;   // 1/dx, correctly rounded on the host (exact divisions by dx, div_rcp)
    double rgam;               // 1/gam, likewise (the inversion's divisions by gamma)
    // CFL per direction k = 1..3: c0[k] = cour dx_k, and ctop_lim[k], the
    // largest double x with c0[k] / x > 1e-6 (set_cfl_limits)
    double cfl_c0[4], ctop_lim[4];
    int pole1, pole2, bc1, bc2, bc3, ct_upwind, inversion, recon, riemann;
    int halo;   // sides filled by a neighbouring block: bits 0, 1 the lower and upper x1
                // sides, bits 2, 3 the lower and upper x2 sides
};

struct Geom {
    const double *gcov, *gcon, *gdet, *conn;
    // per (i, j) column, when tabulated (else null), planes of gs: at the zone
    // centre 1/gdet, the lapse 1/sqrt(-g^tt) and n_t = -sqrt(-1/g^tt), each
    // with the inversion's own operations; then 1/gdet at the FACE1, FACE2
    // and FACE3 locations (the face update's divisions by the face volume);
    // then the lapse at each of the 5 locations (planes 6-10) and its
    // reciprocal (11-15), with geo_lapse's operations (k_inv_tab). Brace
    // initialisation with the four metric tables leaves it null.
    const double *itab;
};

__device__ __forceinline__ long cix(const Dims &d, int i, int j, int z) { return ((long)i * d.G2 + j) * d.G3 + z; }
__device__ __forceinline__ long gix(const Dims &d, int i, int j) { return (long)i * d.G2 + j; }

__device__ __forceinline__ void load_geo(const Dims &d, const Geom &m, int i, int j, int loc, Geo<double> &o) {
    long idx = gix(d, i, j);
#pragma unroll
    for (int s = 0; s < 10; s++) {
        o.gcon[s] = __ldg(&m.gcon[(long)(s * 5 + loc) * d.gs + idx]);
        o.gcov[s] = __ldg(&m.gcov[(long)(s * 5 + loc) * d.gs + idx]);
    }
    o.g = __ldg(&m.gdet[(long)loc * d.gs + idx]);
    if (m.itab) {
        o.lapse = __ldg(&m.itab[(long)(6 + loc) * d.gs + idx]);
        o.rlapse = __ldg(&m.itab[(long)(11 + loc) * d.gs + idx]);
    } else {
        geo_lapse(o);
    }
}

// temp / (face volume at plane `plane` of the column table), exactly
__device__ __forceinline__ double div_face_volume(const Dims &d, const Geom &m, double temp, double gdf, int plane,
                                                  long gi) {
    return m.itab ? div_rcp_inf(temp, gdf, __ldg(&m.itab[(long)plane * d.gs + gi])) : temp / gdf;
}

// metric at one point, stored in double, used in the arithmetic type T
template <typename T>
__device__ __forceinline__ void load_geo_t(const Dims &d, const Geom &m, int i, int j, int loc, Geo<T> &o) {
    long idx = gix(d, i, j);
#pragma unroll
    for (int s = 0; s < 10; s++) {
        o.gcon[s] = (T)__ldg(&m.gcon[(long)(s * 5 + loc) * d.gs + idx]);
        o.gcov[s] = (T)__ldg(&m.gcov[(long)(s * 5 + loc) * d.gs + idx]);
    }
    o.g = (T)__ldg(&m.gdet[(long)loc * d.gs + idx]);
    if (std::is_same<T, double>::value && m.itab) {
        o.lapse = (T)__ldg(&m.itab[(long)(6 + loc) * d.gs + idx]);
        o.rlapse = (T)__ldg(&m.itab[(long)(11 + loc) * d.gs + idx]);
    } else {
        geo_lapse(o);   // float: the lapse of the float metric, as before
    }
}

// Sub-step sizes either come by value (hamr_stage) or from device memory
// (hamr_advance replays a captured graph while the step size evolves).
struct StepSize {
    const double *dev;  // dev[0] = dt when not NULL
    double frac;        // Dt = frac * dt
    double Dt, dt;      // used when dev == NULL
    __device__ __forceinline__ double sub() const { return dev ? frac * dev[0] : Dt; }
    __device__ __forceinline__ double full() const { return dev ? dev[0] : dt; }
};

// ---------------------------------------------------------------------------
// Face fluxes of direction DIR over the normal range [ng, n + ng] and one ghost
// layer either side transversally (fluxcalc2D2's face set).
// build options: minimum resident blocks of 128 threads per SM for the
// double and float flux kernels (caps their registers per thread)
#ifndef HAMR_FLUX_MINB
#define HAMR_FLUX_MINB 5
#endif
#ifndef HAMR_FLUX_MINB_F
#define HAMR_FLUX_MINB_F 6
#endif
// the FP64 x1/x2 row kernels of the face-frame solvers (HLLC, HLLD), which
// hold both frame states, their fluxes and the HLL state in thread-local
// arrays, take a looser cap: on the 384 x 192 x 192 torus with HLLC, 3
// blocks per SM cut those two kernels by 12 % and 9 % against 5; the face
// kernels and the float kernels measured slower with it
#ifndef HAMR_FLUX_FT_ROWS_MINB
#define HAMR_FLUX_FT_ROWS_MINB 3
#endif
#ifndef HAMR_FLUX_FT_ROWS_MINB_F   // the same in the float step
#define HAMR_FLUX_FT_ROWS_MINB_F HAMR_FLUX_ROWS_MINB_F
#endif

// The CFL limit of a face is cour dx / ctop (fluxcalc2D2's dtij, counted
// when above 1e-6), the block's the minimum over its faces and 1e9. A face
// here contributes its signal speed ctop when cour dx / ctop > 1e-6, that is
// when ctop <= ctop_lim (the largest such double, set on the host), else 0;
// the kernels keep the largest contribution and divide once
// (dt_of_ctop): the same minimum, bit for bit.
__device__ __forceinline__ double ctop_term(const Dims &d, int dir, double ctop) {
    return ctop <= d.ctop_lim[dir] ? ctop : 0.0;
}
__device__ __forceinline__ double dt_of_ctop(const Dims &d, int dir, double cmax) {
    const double v = d.cfl_c0[dir] / cmax;   // +inf for cmax = 0
    return v < 1.e9 ? v : 1.e9;
}

template <int DIR, typename T, int REC>
__device__ __forceinline__ double flux_eval(const Dims &d, const Geo<T> &gm, const double *__restrict__ ps, T *pl,
                                            T *pr, T *__restrict__ F, const long c, const int j);

// one face of direction DIR (t < n_faces): reconstruction, two states, four
// flux evaluations, HLL (or HLLC); returns the face's signal-speed
// contribution to the CFL limit (ctop_term). REC: bit 0 MC reconstruction,
// bit 1 HLLC.
template <int DIR, typename T, int REC>
__device__ __forceinline__ double flux_face(const Dims &d, const Geom &m, const double *__restrict__ pv,
                                            const double *__restrict__ ps, T *__restrict__ F, const long t) {
    constexpr int idel = DIR == 1, jdel = DIR == 2, zdel = DIR == 3;
    const int i0 = (d.ng1 - 1) * d.d1 + idel, ni = d.n1 + 2 * d.d1 - idel;
    const int j0 = (d.ng2 - 1) * d.d2 + jdel, nj = d.n2 + 2 * d.d2 - jdel;
    const int z0 = (d.ng3 - 1) * d.d3 + zdel, nz = d.n3 + 2 * d.d3 - zdel;
    (void)ni;
    const int z = z0 + (int)(t % nz);
    const int j = j0 + (int)((t / nz) % nj);
    const int i = i0 + (int)(t / ((long)nz * nj));
    const long c = cix(d, i, j, z);
    const long stride = idel ? (long)d.G2 * d.G3 : (jdel ? (long)d.G3 : 1L);
    const int face = DIR == 1 ? FACE1 : (DIR == 2 ? FACE2 : FACE3);
    Geo<T> gm;
    load_geo_t(d, m, i, j, face, gm);
    T pl[NPR], pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) {
        const double *pk = pv + (long)k * d.ks + c;
        if constexpr ((REC & 1) == HAMR_RECON_MC) {
            // linear MC: the zones' face values y -+ slope/2 (fluxcalcprep, PPM = 0)
            T x[4];
#pragma unroll
            for (int s = 0; s < 4; s++) x[s] = (T)__ldg(pk + (s - 2) * stride);
            T temp = T(0.5) * slope_lim(x[0], x[1], x[2]);
            pl[k] = x[1] + temp;
            temp = T(0.5) * slope_lim(x[1], x[2], x[3]);
            pr[k] = x[2] - temp;
        } else {
            T x[6];
#pragma unroll
            for (int s = 0; s < 6; s++) x[s] = (T)__ldg(pk + (s - 3) * stride);
            T lo, hi;
            para(x, lo, hi);       // zone c-1: upper edge is the left state
            pl[k] = hi;
            para(x + 1, lo, hi);   // zone c: lower edge is the right state
            pr[k] = lo;
        }
    }
    return flux_eval<DIR, T, REC>(d, gm, ps, pl, pr, F, c, j);
}

// The face flux from the reconstructed states pl, pr (the normal field and
// the polar B1 fix applied here): two states, four flux evaluations, HLL (or
// HLLC), the flux written at cell index c; returns the face's signal-speed
// contribution to the CFL limit (ctop_term).
template <int DIR, typename T, int REC>
__device__ __forceinline__ double flux_eval(const Dims &d, const Geo<T> &gm, const double *__restrict__ ps, T *pl,
                                            T *pr, T *__restrict__ F, const long c, const int j) {
    double dtf = 1.e9;
    const T bn = (T)__ldg(&ps[(long)(DIR - 1) * d.ks + c]);
    pl[B1 + DIR - 1] = bn;
    pr[B1 + DIR - 1] = bn;
    if (DIR == 2 && ((j == d.n2 + d.ng2 && d.pole2) || (j == d.ng2 && d.pole1))) {
        pl[B1] = T(0.);
        pr[B1] = T(0.);
    }
    const T gam = (T)d.gam;
    const double dxd = DIR == 1 ? d.dx1 : (DIR == 2 ? d.dx2 : d.dx3);
    if constexpr ((REC & 2) != 0) {
        // HLLC (or, with bit 4, HLLD) in the orthonormal face frame (fluxcalc2D_FT)
        T Fo[NPR];
        const T ctop = hllc_face<DIR, T, (REC & 4) != 0>(gam, pl, pr, gm, Fo);
#pragma unroll
        for (int k = 0; k < NPR; k++) F[(long)k * d.ks + c] = Fo[k];
        (void)dxd;
        (void)dtf;
        return ctop_term(d, DIR, (double)ctop);
    }
    State<T> q;
    T t1[NPR], t2[NPR], t3[NPR], t4[NPR];
    T cmax_l, cmin_l, cmax_r, cmin_r, vd;
    get_state(pl, gm, q);
    T e = entropy(gam, pl);
    primtoflux(gam, pl, q, DIR, gm, e, t1, &cmax_l, &cmin_l);
    primtoflux(gam, pl, q, 0, gm, e, t2, &vd, &vd);
    get_state(pr, gm, q);
    e = entropy(gam, pr);
    primtoflux(gam, pr, q, DIR, gm, e, t3, &cmax_r, &cmin_r);
    primtoflux(gam, pr, q, 0, gm, e, t4, &vd, &vd);
    const T cmax = d_fabs(d_max(d_max(T(0.), cmax_l), cmax_r));
    const T cmin = d_fabs(d_max(d_max(T(0.), -cmin_l), -cmin_r));
    const T ctop = d_max(cmax, cmin);
    const Divisor<T> dh(cmax + cmin + T(SMALL_D));   // the nine HLL quotients share it
#pragma unroll
    for (int k = 0; k < NPR; k++)
        F[(long)k * d.ks + c] = dh.div(cmax * t1[k] + cmin * t3[k] - cmax * cmin * (t4[k] - t2[k]));
    (void)dxd;
    (void)dtf;
    return ctop_term(d, DIR, (double)ctop);
}

// faces of direction DIR of one block
template <int DIR>
__host__ __device__ __forceinline__ long n_faces(const Dims &d) {
    constexpr int idel = DIR == 1, jdel = DIR == 2, zdel = DIR == 3;
    return (long)(d.n1 + 2 * d.d1 - idel) * (d.n2 + 2 * d.d2 - jdel) * (d.n3 + 2 * d.d3 - zdel);
}

// CTA minimum of the threads' CFL limits by warp shuffles, one atomic per CTA
// (positive doubles order like their bit patterns)
__device__ __forceinline__ void cta_min_dt(double dtf, unsigned long long *slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dtf = d_min(dtf, __shfl_xor_sync(0xffffffffu, dtf, o));
    __shared__ double wmin[BLK / 32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = dtf;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmin[0];
        for (int w = 1; w < BLK / 32; w++) b = d_min(b, wmin[w]);
        atomicMin(slot, (unsigned long long)__double_as_longlong(b));
    }
    __syncthreads();   // wmin is reused by the CTA's next tile
}

// The same from the faces' signal speeds (ctop_term): the CTA's largest, then
// one division, min(1e9, c0 / max) -- the minimum over the CTA's faces of
// the per-face limit c0 / ctop, because correctly rounded division by a
// positive divisor does not increase as the divisor grows
__device__ __forceinline__ void cta_max_ctop(const Dims &d, int dir, double cmx, unsigned long long *slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmx = d_max(cmx, __shfl_xor_sync(0xffffffffu, cmx, o));
    __shared__ double wmax[BLK / 32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = cmx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmax[0];
        for (int w = 1; w < BLK / 32; w++) b = d_max(b, wmax[w]);
        atomicMin(slot, (unsigned long long)__double_as_longlong(dt_of_ctop(d, dir, b)));
    }
    __syncthreads();
}

template <int DIR, typename T, int REC>
__global__ void __launch_bounds__(BLK, sizeof(T) == 8 ? HAMR_FLUX_MINB : HAMR_FLUX_MINB_F) k_flux(const Dims d, const Geom m, const double *__restrict__ pv,
                                               const double *__restrict__ ps, T *__restrict__ F,
                                               unsigned long long *__restrict__ dtbits, int calc_dt) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const double cmx = t < n_faces<DIR>(d) ? flux_face<DIR, T, REC>(d, m, pv, ps, F, t) : 0.0;
    if (calc_dt) cta_max_ctop(d, DIR, cmx, &dtbits[DIR]);
}

// Both edge values of one zone, primitive by primitive (the normal field
// component skipped: the face sets it). PPM (para) or MC.
template <int DIR, typename T, int REC>
__device__ __forceinline__ void zone_edges(const Dims &d, const double *__restrict__ pv, long cz, long stride,
                                           T *lo, T *hi) {
#pragma unroll
    for (int k = 0; k < NPR; k++) {
        if (k == B1 + DIR - 1) continue;
        const double *pk = pv + (long)k * d.ks + cz;
        if constexpr ((REC & 1) == HAMR_RECON_MC) {
            const T y1 = (T)__ldg(pk - stride), y2 = (T)__ldg(pk), y3 = (T)__ldg(pk + stride);
            const T temp = T(0.5) * slope_lim(y1, y2, y3);
            lo[k] = y2 - temp;
            hi[k] = y2 + temp;
        } else {
            T x[5];
#pragma unroll
            for (int s = 0; s < 5; s++) x[s] = (T)__ldg(pk + (s - 2) * stride);
            para(x, lo[k], hi[k]);
        }
    }
}

// x3 faces (phi, the contiguous direction) with each zone reconstructed once.
// The zones a row of x3 faces touches, z = ng3 - 1 .. ng3 + n3 (n3 + 2 of
// them for n3 + 1 faces), are numbered row after row as "slots"; CTA b takes
// slots b (BLK - 1) .. b (BLK - 1) + BLK - 1, one per thread, so consecutive
// CTAs share one slot. Phase 1: every thread reconstructs its slot's zone and
// leaves both edges in shared memory. Phase 2: thread l evaluates the face
// between slots l and l + 1 when both lie in the same row (left state: the
// upper edge of slot l, right state: the lower edge of slot l + 1). Every
// thread does the same work in each phase, so the barrier between them costs
// little. Same values as k_flux<3> face by face: the same para on the same
// five zones.
__host__ __device__ __forceinline__ long n_x3_slots(const Dims &d) {
    return (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3);
}

// build options: resident blocks per SM for the double and float x3 slot
// kernels. Measured per 384 x 192 x 192 step: float 10 blocks (48 registers)
// 2.04 ms, 12: 2.09, 8: 2.14, 6 (80 registers, no spills): 2.54; double (with
// the shared-divisor quotients and the centre EMFs) 5 blocks 5.48 ms, 4:
// 5.52, 6: 5.62.
// The face-frame solvers (HLLC, HLLD) in the x3 slot kernel, which hold both
// frame states, their fluxes and (HLLD) the wave fan in thread-local arrays:
// on the 384 x 192 x 192 torus, FP64, per step, 4 blocks per SM (128
// registers) HLLC 8.63 ms / HLLD 9.68 ms, 5: 8.66 / 11.98, 6: 9.80 / 14.91,
// 3: 9.50 / 9.87
#ifndef HAMR_FLUX_FT_X3_MINB
#define HAMR_FLUX_FT_X3_MINB 4
#endif
#ifndef HAMR_FLUX_FT_X3_MINB_F   // float: 7 blocks, HLLC 3.83 -> 3.69 ms, HLLD 6.19 -> 3.96 (5: 4.01 / 4.22)
#define HAMR_FLUX_FT_X3_MINB_F 7
#endif
#ifndef HAMR_FLUX_X3_MINB
#define HAMR_FLUX_X3_MINB 5
#endif
#ifndef HAMR_FLUX_X3_MINB_F
#define HAMR_FLUX_X3_MINB_F 10
#endif

template <typename T>
__device__ __forceinline__ void emf_centre_eval(const Dims &d, const Geom &m, const double *__restrict__ pv, int i,
                                                int j, long c, T *e);

// With Ec non-null the kernel also computes the centre EMFs (k_emf_centre's
// work): its slots are exactly k_emf_centre's zones, and the slot's
// primitives are already in L1 from its reconstruction stencil. A slot that
// two CTAs share is done by the first. Same values as k_emf_centre.
// The body of CTA `blk` of the block's slot range; returns the thread's
// face signal speed (0 without a face) for the CTA's CFL reduction.
template <typename T, int REC>
__device__ __forceinline__ double flux_x3_slots(const Dims &d, const Geom &m, const double *__restrict__ pv,
                                                const double *__restrict__ ps, T *__restrict__ F,
                                                T *__restrict__ Ec, long blk) {
    __shared__ T slo[NPR - 1][BLK], shi[NPR - 1][BLK];   // zone edges per slot (B3 skipped)
    const int l = threadIdx.x;
    const long nslot = n_x3_slots(d);
    const int rz = d.n3 + 2 * d.d3;   // slots per row
    const int nj = d.n2 + 2 * d.d2;
    const long sl = blk * (BLK - 1) + l;
    const int zl = (int)(sl % rz);
    const long row = sl / rz;
    const int j = (d.ng2 - 1) * d.d2 + (int)(row % nj);
    const int i = (d.ng1 - 1) * d.d1 + (int)(row / nj);
    const long c = cix(d, i, j, d.ng3 - 1 + zl);   // the slot's zone
    if (sl < nslot) {
        T lo[NPR], hi[NPR];
        zone_edges<3, T, REC>(d, pv, c, 1, lo, hi);
#pragma unroll
        for (int k = 0, q = 0; k < NPR; k++)
            if (k != B3) {
                slo[q][l] = lo[k];
                shi[q++][l] = hi[k];
            }
        if (Ec && (l < BLK - 1 || sl == nslot - 1)) {
            T e[3];
            emf_centre_eval(d, m, pv, i, j, c, e);
            Ec[1 * d.ks + c] = e[0];
            Ec[2 * d.ks + c] = e[1];
            Ec[3 * d.ks + c] = e[2];
        }
    }
    __syncthreads();
    double cmx = 0.0;
    // the face above this slot's zone: zone c + 1 is the next slot of the row
    if (l < BLK - 1 && sl + 1 < nslot && zl + 1 < rz) {
        T pl[NPR], pr[NPR];
#pragma unroll
        for (int k = 0, q = 0; k < NPR; k++)
            if (k != B3) {
                pl[k] = shi[q][l];
                pr[k] = slo[q++][l + 1];
            }
        Geo<T> gm;
        load_geo_t(d, m, i, j, FACE3, gm);
        cmx = flux_eval<3, T, REC>(d, gm, ps, pl, pr, F, c + 1, j);
    }
    return cmx;
}

// CTAs of the slot range: CTA b takes slots b (BLK - 1) .. b (BLK - 1) + BLK - 1
__host__ __device__ __forceinline__ long n_x3_slot_ctas(const Dims &d) {
    return (n_x3_slots(d) - 1 + BLK - 2) / (BLK - 1);
}

template <typename T, int REC>
__global__ void __launch_bounds__(BLK, sizeof(T) == 8 ? ((REC & 2) != 0 ? HAMR_FLUX_FT_X3_MINB : HAMR_FLUX_X3_MINB)
                                                         : ((REC & 2) != 0 ? HAMR_FLUX_FT_X3_MINB_F : HAMR_FLUX_X3_MINB_F))
    k_flux_x3(const Dims d, const Geom m, const double *__restrict__ pv, const double *__restrict__ ps,
              T *__restrict__ F, unsigned long long *__restrict__ dtbits, int calc_dt, T *__restrict__ Ec) {
    const double cmx = flux_x3_slots<T, REC>(d, m, pv, ps, F, Ec, blockIdx.x);
    if (calc_dt) cta_max_ctop(d, 3, cmx, &dtbits[3]);
}

// Faces of direction DIR (1 or 2) by rows: a thread walks FLUX_ROW
// consecutive faces along DIR at fixed transverse indices, reconstructing
// each zone once (its upper edge is the left state of the next face) where
// the face-by-face kernel reconstructs every zone twice; neighbouring
// threads take neighbouring z, so the loads stay coalesced. Same values as
// k_flux face by face.
// build options: faces per row, and minimum resident blocks of 128 threads
// per SM for the row kernels (FP64, float). Measured on the 384 x 192 x 192
// torus: rows of 12 beat 6, 8, 24 and 48 (shorter rows: more threads in
// flight, longer: fewer extra reconstructions); 7 float blocks beat 6 and 8,
// 5 double blocks beat 4. The stencil window (RowWindow) took the float x1 +
// x2 fluxes from 4.48 to 3.77 ms per step (FP64 13.49 -> 13.36).
#ifndef HAMR_FLUX_ROW
#define HAMR_FLUX_ROW 12
#endif
constexpr int FLUX_ROW = HAMR_FLUX_ROW;
#ifndef HAMR_FLUX_ROWS_MINB   // FP64: 4 blocks (128 registers) x2 + x1 9.18 -> 8.79 ms per step (5: 96)
#define HAMR_FLUX_ROWS_MINB 4
#endif
#ifndef HAMR_FLUX_ROWS_MINB_F
#define HAMR_FLUX_ROWS_MINB_F 7
#endif
template <int DIR>
__host__ __device__ __forceinline__ long n_flux_rows(const Dims &d) {
    static_assert(DIR == 1 || DIR == 2, "rows along x1 or x2");
    const long nf = DIR == 1 ? d.n1 + 2 * d.d1 - 1 : d.n2 + 2 * d.d2 - 1;
    const long nt = DIR == 1 ? (long)(d.n2 + 2 * d.d2) : (long)(d.n1 + 2 * d.d1);
    return ((nf + FLUX_ROW - 1) / FLUX_ROW) * nt * (d.n3 + 2 * d.d3);
}

// A thread's stencil window along its row, in shared memory: the NW zones
// (5 for PPM, 3 for MC) around the zone being reconstructed, each as its
// NPR - 1 reconstructed primitives (the normal field component is not
// reconstructed), converted to T once when loaded. Slot of zone index q along
// the row: q mod NW. Each thread touches only its own column (threadIdx.x), so
// no barrier is needed, and consecutive threads hit consecutive banks. Moving
// to the next face loads one new zone (NPR - 1 values) instead of the whole
// stencil (NW (NPR - 1) values); the reconstruction sees the same values as
// zone_edges.
template <int DIR, typename T, int REC>
struct RowWindow {
    static constexpr int NW = (REC & 1) == HAMR_RECON_MC ? 3 : 5;
    static constexpr int H = NW / 2;
    static constexpr int NK = NPR - 1;
    T *w;
    __device__ __forceinline__ T &at(int slot, int kk) const { return w[(slot * NK + kk) * BLK]; }
    __device__ __forceinline__ void load(const Dims &d, const double *__restrict__ pv, long cz, int slot) const {
        int kk = 0;
#pragma unroll
        for (int k = 0; k < NPR; k++) {
            if (k == B1 + DIR - 1) continue;
            at(slot, kk++) = (T)__ldg(pv + (long)k * d.ks + cz);
        }
    }
    // edges of the zone whose stencil starts in slot s0 (the zone q - H)
    __device__ __forceinline__ void edges(int s0, T *lo, T *hi) const {
        int kk = 0;
#pragma unroll
        for (int k = 0; k < NPR; k++) {
            if (k == B1 + DIR - 1) continue;
            T x[NW];
#pragma unroll
            for (int s = 0; s < NW; s++) {
                const int sl = s0 + s;
                x[s] = at(sl >= NW ? sl - NW : sl, kk);
            }
            if constexpr (NW == 3) {
                const T temp = T(0.5) * slope_lim(x[0], x[1], x[2]);
                lo[k] = x[1] - temp;
                hi[k] = x[1] + temp;
            } else {
                para(x, lo[k], hi[k]);
            }
            kk++;
        }
    }
};

// One row of FLUX_ROW faces along DIR (row t < n_flux_rows), reconstructed
// through the thread's stencil window in `wbuf` (a CTA's NW * NK * BLK
// values; column threadIdx.x); returns the row's largest signal-speed
// contribution (ctop_term)
template <int DIR, typename T, int REC>
__device__ __forceinline__ double flux_row(const Dims &d, const Geom &m, const double *__restrict__ pv,
                                           const double *__restrict__ ps, T *__restrict__ F, T *wbuf, const long t) {
    using Win = RowWindow<DIR, T, REC>;
    double cmx = 0.0;
    const int nz = d.n3 + 2 * d.d3, z = (d.ng3 - 1) * d.d3 + (int)(t % nz);
    const long r = t / nz;
    const int nt = DIR == 1 ? d.n2 + 2 * d.d2 : d.n1 + 2 * d.d1;
    const int a = (DIR == 1 ? (d.ng2 - 1) * d.d2 : (d.ng1 - 1) * d.d1) + (int)(r % nt);   // j or i
    const int seg = (int)(r / nt);
    const int nf = DIR == 1 ? d.n1 + 2 * d.d1 - 1 : d.n2 + 2 * d.d2 - 1;
    const int ng = DIR == 1 ? d.ng1 : d.ng2;
    const int f0 = ng + seg * FLUX_ROW;
    const int f1 = min(f0 + FLUX_ROW, ng + nf);
    const long stride = DIR == 1 ? (long)d.G2 * d.G3 : (long)d.G3;
    const int face = DIR == 1 ? FACE1 : FACE2;
    const Win win{wbuf + threadIdx.x};
    constexpr int NW = Win::NW, H = Win::H;
    T pl[NPR], lo[NPR], hi[NPR];
    // the stencil of the zone below the first face, zones f0 - 1 - H ..
    // f0 - 1 + H (f0 >= ng > H), then its upper edge: the first left state
    const long cf0 = DIR == 1 ? cix(d, f0, a, z) : cix(d, a, f0, z);
#pragma unroll
    for (int s = 0; s < NW; s++) win.load(d, pv, cf0 + (s - 1 - H) * stride, (f0 - 1 - H + s) % NW);
    win.edges((f0 - 1 - H) % NW, lo, hi);
#pragma unroll
    for (int k = 0; k < NPR; k++) pl[k] = hi[k];
    int s0 = (f0 - H) % NW;   // slot of zone f - H
    for (int f = f0; f < f1; f++) {
        const int i = DIR == 1 ? f : a, j = DIR == 1 ? a : f;
        const long c = cix(d, i, j, z);
        // zone f + H replaces zone f - H - 1 (slot s0 + 2H, mod NW)
        win.load(d, pv, c + H * stride, s0 == 0 ? NW - 1 : s0 - 1);
        win.edges(s0, lo, hi);
        s0 = s0 == NW - 1 ? 0 : s0 + 1;
        Geo<T> gm;
        load_geo_t(d, m, i, j, face, gm);
        T l[NPR];
#pragma unroll
        for (int k = 0; k < NPR; k++) l[k] = pl[k];
        cmx = d_max(cmx, flux_eval<DIR, T, REC>(d, gm, ps, l, lo, F, c, j));
#pragma unroll
        for (int k = 0; k < NPR; k++) pl[k] = hi[k];
    }
    return cmx;
}

template <int DIR, typename T, int REC>
__global__ void __launch_bounds__(BLK, sizeof(T) == 8 ? ((REC & 2) != 0 ? HAMR_FLUX_FT_ROWS_MINB : HAMR_FLUX_ROWS_MINB)
                                                         : ((REC & 2) != 0 ? HAMR_FLUX_FT_ROWS_MINB_F : HAMR_FLUX_ROWS_MINB_F))
    k_flux_rows(const Dims d, const Geom m, const double *__restrict__ pv, const double *__restrict__ ps,
                T *__restrict__ F, unsigned long long *__restrict__ dtbits, int calc_dt) {
    using Win = RowWindow<DIR, T, REC>;
    __shared__ T wbuf[Win::NW * Win::NK * BLK];
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const double cmx = t < n_flux_rows<DIR>(d) ? flux_row<DIR, T, REC>(d, m, pv, ps, F, wbuf, t) : 0.0;
    if (calc_dt) cta_max_ctop(d, DIR, cmx, &dtbits[DIR]);
}

// reflective polar axis and no-inflow radial edges (fix_flux, GPU_const_trans.h:3-61)
template <typename T>
__device__ __forceinline__ void fix_flux_at(const Dims &d, T *F1, T *F2, T *F3, const long t) {
    const long ks = d.ks;
    const long na = (long)d.G1 * d.G3;
    if (t < na) {
        const int z = (int)(t % d.G3), i = (int)(t / d.G3);
        if (!(i >= d.ng1 - d.d1 && z >= d.ng3 - d.d3 && i < d.n1 + d.ng1 + d.d1 && z < d.n3 + d.ng3 + d.d3)) return;
        if (d.pole1) {
            F1[B2 * ks + cix(d, i, d.ng2 - 1, z)] = -F1[B2 * ks + cix(d, i, d.ng2, z)];
            if (d.ng3 > 0) F3[B2 * ks + cix(d, i, d.ng2 - 1, z)] = -F3[B2 * ks + cix(d, i, d.ng2, z)];
            for (int k = 0; k < NPR; k++) F2[k * ks + cix(d, i, d.ng2, z)] = T(0.);
        }
        if (d.pole2) {
            F1[B2 * ks + cix(d, i, d.n2 + d.ng2, z)] = -F1[B2 * ks + cix(d, i, d.n2 + d.ng2 - 1, z)];
            if (d.ng3 > 0) F3[B2 * ks + cix(d, i, d.n2 + d.ng2, z)] = -F3[B2 * ks + cix(d, i, d.n2 + d.ng2 - 1, z)];
            for (int k = 0; k < NPR; k++) F2[k * ks + cix(d, i, d.n2 + d.ng2, z)] = T(0.);
        }
        return;
    }
    const long u = t - na;
    if (u >= (long)d.G2 * d.G3) return;
    const int z = (int)(u % d.G3), j = (int)(u / d.G3);
    if (!(j >= d.ng2 - d.d2 && z >= d.ng3 - d.d3 && j < d.n2 + d.ng2 + d.d2 && z < d.n3 + d.ng3 + d.d3)) return;
    // no inflow through the physical radial edges (not through a face shared
    // with a neighbouring block)
    const long ci = RHO * ks + cix(d, d.ng1, j, z);
    if (!(d.halo & 1) && F1[ci] > T(0.)) F1[ci] = T(0.);
    const long co = RHO * ks + cix(d, d.n1 + d.ng1, j, z);
    if (!(d.halo & 2) && F1[co] < T(0.)) F1[co] = T(0.);
}

// items of fix_flux: (i, z) on the polar rows, then (j, z) on the radial edges
__host__ __device__ __forceinline__ long n_fix_flux(const Dims &d) { return (long)d.G1 * d.G3 + (long)d.G2 * d.G3; }

template <typename T>
__global__ void k_fix_flux(const Dims d, T *F1, T *F2, T *F3) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_fix_flux(d)) fix_flux_at(d, F1, F2, F3, t);
}

// cell-centre EMF, -gdet (u x b), of zone (i, j, z): e[0..2] = E1, E2, E3
// (E1, E2 only in 3-D)
template <typename T>
__device__ __forceinline__ void emf_centre_eval(const Dims &d, const Geom &m, const double *__restrict__ pv, int i,
                                                int j, long c, T *e) {
    T pb[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pb[k] = (T)__ldg(&pv[k * d.ks + c]);
    Geo<T> gm;
    load_geo_t(d, m, i, j, CENT, gm);
    T ucon[4], ucov[4], bcon[4];
    ucon_calc(pb, gm, ucon);
    lower4(ucon, gm.gcov, ucov);
    bcon_calc(pb, ucon, ucov, bcon);
    if (d.ng3 > 0) {
        e[0] = -gm.g * (ucon[2] * bcon[3] - ucon[3] * bcon[2]);
        e[1] = -gm.g * (ucon[3] * bcon[1] - ucon[1] * bcon[3]);
    }
    e[2] = -gm.g * (ucon[1] * bcon[2] - ucon[2] * bcon[1]);
}

// on the active zones plus one ghost layer
template <typename T>
__device__ __forceinline__ void k_emf_centre_at(const Dims &d, const Geom &m, const double *__restrict__ pv,
                                                     T *__restrict__ Ec, const long t) {
    const int ni = d.n1 + 2 * d.d1, nj = d.n2 + 2 * d.d2, nz = d.n3 + 2 * d.d3;
    const int z = (d.ng3 - d.d3) * d.d3 + (int)(t % nz);
    const int j = (d.ng2 - d.d2) * d.d2 + (int)((t / nz) % nj);
    const int i = (d.ng1 - d.d1) * d.d1 + (int)(t / ((long)nz * nj));
    (void)ni;
    const long c = cix(d, i, j, z);
    T e[3];
    emf_centre_eval(d, m, pv, i, j, c, e);
    if (d.ng3 > 0) {
        Ec[1 * d.ks + c] = e[0];
        Ec[2 * d.ks + c] = e[1];
    }
    Ec[3 * d.ks + c] = e[2];
}

template <typename T>
__global__ void __launch_bounds__(BLK) k_emf_centre(const Dims d, const Geom m, const double *__restrict__ pv,
                                                     T *__restrict__ Ec) {
    const int ni = d.n1 + 2 * d.d1, nj = d.n2 + 2 * d.d2, nz = d.n3 + 2 * d.d3;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj * nz) return;
    k_emf_centre_at(d, m, pv, Ec, t);
}

template <typename T> __device__ __forceinline__ T up(T f) { return (T)(f <= T(0.0)); }
template <typename T> __device__ __forceinline__ T dn(T f) { return (T)(f > T(0.0)); }

// edge EMFs: average of the four face EMFs plus, when ct_upwind, the
// centre-minus-face corrections from the upwind side of each face, chosen by
// the sign of its mass flux (consttransport2, GPU_const_trans.h:121-338), for
// the edge at cell index c (row j): ec(k, di, dj, dz) is centre EMF k (1..3)
// of the zone offset by (di, dj, dz) in {-1, 0}^3 from the edge's cell
// (times the direction flags d1..d3); e[0..2] = E1, E2, E3
template <typename T, class EC>
__device__ __forceinline__ void emf_edge_eval(const Dims &d, EC ec, const T *__restrict__ F1,
                                              const T *__restrict__ F2, const T *__restrict__ F3, long c, int j,
                                              T *e) {
    const long ks = d.ks, jsize = d.G3, isize = (long)d.G2 * d.G3;
    const long D1 = d.d1, D2 = d.d2, D3 = d.d3;
    const T *F1r = F1 + RHO * ks, *F2r = F2 + RHO * ks, *F3r = F3 + RHO * ks;
    const bool w = d.ct_upwind != 0;
    // in the non-upwind build every correction is an exact 0.0
#define CORR(expr) (w ? (expr) : T(0.0))
    const T dE_LEFT_13_1 = CORR(ec(1, 0, 0, 0) - F3[B2 * ks + c]);
    const T dE_LEFT_13_2 = CORR(ec(1, 0, -1, 0) - F3[B2 * ks + c - jsize * D2]);
    const T dE_RIGHT_13_1 = CORR(F3[B2 * ks + c] - ec(1, 0, 0, -1));
    const T dE_RIGHT_13_2 = CORR(F3[B2 * ks + c - jsize * D2] - ec(1, 0, -1, -1));
    const T dE_LEFT_12_1 = CORR(ec(1, 0, 0, 0) + F2[B3 * ks + c]);
    const T dE_LEFT_12_2 = CORR(ec(1, 0, 0, -1) + F2[B3 * ks + c - D3]);
    const T dE_RIGHT_12_1 = CORR(-F2[B3 * ks + c] - ec(1, 0, -1, 0));
    const T dE_RIGHT_12_2 = CORR(-F2[B3 * ks + c - D3] - ec(1, 0, -1, -1));
    const T dE_LEFT_21_1 = CORR(ec(2, 0, 0, 0) - F1[B3 * ks + c]);
    const T dE_LEFT_21_2 = CORR(ec(2, 0, 0, -1) - F1[B3 * ks + c - D3]);
    const T dE_RIGHT_21_1 = CORR(F1[B3 * ks + c] - ec(2, -1, 0, 0));
    const T dE_RIGHT_21_2 = CORR(F1[B3 * ks + c - D3] - ec(2, -1, 0, -1));
    const T dE_LEFT_23_1 = CORR(ec(2, 0, 0, 0) + F3[B1 * ks + c]);
    const T dE_LEFT_23_2 = CORR(ec(2, -1, 0, 0) + F3[B1 * ks + c - D1 * isize]);
    const T dE_RIGHT_23_1 = CORR(-F3[B1 * ks + c] - ec(2, 0, 0, -1));
    const T dE_RIGHT_23_2 = CORR(-F3[B1 * ks + c - isize * D1] - ec(2, -1, 0, -1));
    const T dE_LEFT_31_1 = CORR(ec(3, 0, 0, 0) + F1[B2 * ks + c]);
    const T dE_LEFT_31_2 = CORR(ec(3, 0, -1, 0) + F1[B2 * ks + c - D2 * jsize]);
    const T dE_RIGHT_31_1 = CORR(-F1[B2 * ks + c] - ec(3, -1, 0, 0));
    const T dE_RIGHT_31_2 = CORR(-F1[B2 * ks + c - D2 * jsize] - ec(3, -1, -1, 0));
    const T dE_LEFT_32_1 = CORR(ec(3, 0, 0, 0) - F2[B1 * ks + c]);
    const T dE_LEFT_32_2 = CORR(ec(3, -1, 0, 0) - F2[B1 * ks + c - D1 * isize]);
    const T dE_RIGHT_32_1 = CORR(F2[B1 * ks + c] - ec(3, 0, -1, 0));
    const T dE_RIGHT_32_2 = CORR(F2[B1 * ks + c - D1 * isize] - ec(3, -1, -1, 0));
#undef CORR
    T e1 = T(0.25) * ((-F2[B3 * ks + c] - (dE_LEFT_13_1 * up(F2r[c]) + dE_LEFT_13_2 * dn(F2r[c])))
        + (-F2[B3 * ks + c - D3] + (dE_RIGHT_13_1 * up(F2r[c - D3]) + dE_RIGHT_13_2 * dn(F2r[c - D3]))) +
        +(F3[B2 * ks + c] - (dE_LEFT_12_1 * up(F3r[c]) + dE_LEFT_12_2 * dn(F3r[c])))
        + (F3[B2 * ks + c - D2 * jsize] + (dE_RIGHT_12_1 * up(F3r[c - D2 * jsize]) + dE_RIGHT_12_2 * dn(F3r[c - D2 * jsize]))));
    const T e2 = T(0.25) * ((-F3[B1 * ks + c] - (dE_LEFT_21_1 * up(F3r[c]) + dE_LEFT_21_2 * dn(F3r[c])))
        + (-F3[B1 * ks + c - D1 * isize] + (dE_RIGHT_21_1 * up(F3r[c - D1 * isize]) + dE_RIGHT_21_2 * dn(F3r[c - D1 * isize])))
        + (F1[B3 * ks + c] - (dE_LEFT_23_1 * up(F1r[c]) + dE_LEFT_23_2 * dn(F1r[c])))
        + (F1[B3 * ks + c - D3] + (dE_RIGHT_23_1 * up(F1r[c - D3]) + dE_RIGHT_23_2 * dn(F1r[c - D3]))));
    T e3 = T(0.25) * ((F2[B1 * ks + c] - (dE_LEFT_31_1 * up(F2r[c]) + dE_LEFT_31_2 * dn(F2r[c])))
        + (F2[B1 * ks + c - D1 * isize] + (dE_RIGHT_31_1 * up(F2r[c - D1 * isize]) + dE_RIGHT_31_2 * dn(F2r[c - D1 * isize])))
        + (-F1[B2 * ks + c] - (dE_LEFT_32_1 * up(F1r[c]) + dE_LEFT_32_2 * dn(F1r[c])))
        + (-F1[B2 * ks + c - D2 * jsize] + (dE_RIGHT_32_1 * up(F1r[c - D2 * jsize]) + dE_RIGHT_32_2 * dn(F1r[c - D2 * jsize]))));
    if ((d.pole1 && j == d.ng2) || (d.pole2 && j == d.n2 + d.ng2)) {
        e3 = T(0.);
        e1 = T(-0.5) * (F2[B3 * ks + c] + F2[B3 * ks + c - D3]);
    }
    e[0] = e1;
    e[1] = e2;
    e[2] = e3;
}

template <typename T>
__device__ __forceinline__ void k_emf_edge_at(const Dims &d, const T *__restrict__ Ec,
                                                   const T *__restrict__ F1, const T *__restrict__ F2,
                                                   const T *__restrict__ F3, T *__restrict__ emf, const long t) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2, nz = d.n3 + d.d3;
    const int z = d.ng3 * d.d3 + (int)(t % nz);
    const int j = d.ng2 * d.d2 + (int)((t / nz) % nj);
    const int i = d.ng1 * d.d1 + (int)(t / ((long)nz * nj));
    (void)ni;
    const long c = cix(d, i, j, z);
    const long ks = d.ks, jsize = d.G3, isize = (long)d.G2 * d.G3;
    auto ec = [&](int k, int di, int dj, int dz) {
        return Ec[k * ks + c + di * d.d1 * isize + dj * d.d2 * jsize + dz * d.d3];
    };
    T e[3];
    emf_edge_eval<T>(d, ec, F1, F2, F3, c, j, e);
    emf[1 * ks + c] = e[0];
    emf[2 * ks + c] = e[1];
    emf[3 * ks + c] = e[2];
}

// (two z edges per thread, as k_face_update takes two face triples, measured
// slower: 0.58 -> 0.63 ms per mixed 384 x 192 x 192 step, 1.03 -> 1.07 FP64)
template <typename T>
__global__ void __launch_bounds__(BLK) k_emf_edge(const Dims d, const T *__restrict__ Ec,
                                                   const T *__restrict__ F1, const T *__restrict__ F2,
                                                   const T *__restrict__ F3, T *__restrict__ emf) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2, nz = d.n3 + d.d3;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ni * nj * nz) return;
    k_emf_edge_at(d, Ec, F1, F2, F3, emf, t);
}

// phi-average of the x1-EMF on the polar edges of a block that holds every
// phi zone (E_average, const_trans.c:268-503): dt-scaled sum over active z,
// divided by n3, unscaled; x3-EMF zeroed there. One thread per (side, i).
template <typename T>
__device__ __forceinline__ void k_pole_average_at(const Dims &d, T *emf, StepSize st, const long t) {
    const int ni = d.n1 + d.ng1;
    const int side = t / ni, i = d.ng1 + t % ni;
    if ((side == 0 && !d.pole1) || (side == 1 && !d.pole2)) return;
    const int jp = side == 0 ? d.ng2 : d.n2 + d.ng2;
    const double dt = st.full();
    double avg = 0.;
    for (int z = d.ng3; z < d.n3 + d.ng3; z++) avg += dt * (double)emf[1 * d.ks + cix(d, i, jp, z)];
    avg /= (double)(d.n3);
    const double avg_new = avg / ((double)1);
    for (int z = d.ng3; z < d.n3 + 2 * d.ng3; z++) {
        emf[1 * d.ks + cix(d, i, jp, z)] = (T)(avg_new / dt);
        emf[3 * d.ks + cix(d, i, jp, z)] = T(0.);
    }
}

// The same average with one warp per (pole, i) row: the lanes load 32
// consecutive phi values at a time and lane 0 adds them in order (shuffled
// to it one by one), so the sum is the row-by-row one above, bit for bit;
// the row is written back by all lanes.
template <typename T>
__global__ void k_pole_average(const Dims d, T *emf, StepSize st) {
    const int ni = d.n1 + d.ng1;
    const int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (t >= 2 * ni) return;   // whole warps leave together (t is per warp)
    const int side = t / ni, i = d.ng1 + t % ni;
    if ((side == 0 && !d.pole1) || (side == 1 && !d.pole2)) return;
    const int jp = side == 0 ? d.ng2 : d.n2 + d.ng2;
    const double dt = st.full();
    const T *row = emf + 1 * d.ks + cix(d, i, jp, 0);
    double avg = 0.;
    for (int z0 = d.ng3; z0 < d.n3 + d.ng3; z0 += 32) {
        const int z = z0 + lane;
        const double x = z < d.n3 + d.ng3 ? (double)row[z] : 0.;
        const int m = min(32, d.n3 + d.ng3 - z0);
        for (int k = 0; k < m; k++) {
            const double xk = __shfl_sync(0xffffffffu, x, k);
            if (lane == 0) avg += dt * xk;
        }
    }
    avg = __shfl_sync(0xffffffffu, avg, 0);
    avg /= (double)(d.n3);
    const double avg_new = avg / ((double)1);
    for (int z = d.ng3 + lane; z < d.n3 + 2 * d.ng3; z += 32) {
        emf[1 * d.ks + cix(d, i, jp, z)] = (T)(avg_new / dt);
        emf[3 * d.ks + cix(d, i, jp, z)] = T(0.);
    }
}

// staggered field update from the edge EMFs (consttransport3,
// GPU_const_trans.h:426-529) of the face triple at cell (i, j, z): E(k, di,
// dj, dz) is edge EMF k (1..3) at the offset (di, dj, dz) in {0, 1}^3 (times
// the direction flags); `rows` selects which faces to write (bit 0: x1, bit 1:
// x2, bit 2: x3) on top of the range checks.
template <class EF>
__device__ __forceinline__ void face_update_eval(const Dims &d, const Geom &m, const double *psi, double *psf,
                                                 EF E, double Dt, int i, int j, int z, long c, long gi, int faces) {
    const long ks = d.ks;
    if ((faces & 1) && i < d.n1 + d.ng1 + d.d1 && j < d.n2 + d.ng2 && z < d.n3 + d.ng3) {
        const double gdf = __ldg(&m.gdet[FACE1 * d.gs + gi]);
        double temp = 0.;
        temp += 1.0 / ((double)1) * psi[c] * gdf;
        temp += div_rcp(-Dt, d.dx2, d.rdx2) * (E(3, 0, 1, 0) - E(3, 0, 0, 0));
        if (d.ng3 > 0) temp += div_rcp(Dt, d.dx3, d.rdx3) * (E(2, 0, 0, 1) - E(2, 0, 0, 0));
        psf[c] = div_face_volume(d, m, temp, gdf, 3, gi);
    }
    if ((faces & 4) && d.ng3 > 0 && i < d.n1 + d.ng1 && j < d.n2 + d.ng2 && z < d.n3 + d.ng3 + d.d3) {
        const double gdf = __ldg(&m.gdet[FACE3 * d.gs + gi]);
        double temp = psi[2 * ks + c] * gdf;
        temp += div_rcp(-Dt, d.dx1, d.rdx1) * (E(2, 1, 0, 0) - E(2, 0, 0, 0));
        temp += div_rcp(Dt, d.dx2, d.rdx2) * (E(1, 0, 1, 0) - E(1, 0, 0, 0));
        psf[2 * ks + c] = div_face_volume(d, m, temp, gdf, 5, gi);
    }
    if ((faces & 2) && i < d.n1 + d.ng1 && j < d.n2 + d.ng2 + d.d2 && z < d.n3 + d.ng3) {
        const double gdf = __ldg(&m.gdet[FACE2 * d.gs + gi]);
        double temp = 0.;
        temp += 1.0 / ((double)1) * psi[1 * ks + c] * gdf;
        temp += div_rcp(Dt, d.dx1, d.rdx1) * (E(3, 1, 0, 0) - E(3, 0, 0, 0));
        if (d.ng3 > 0) temp += div_rcp(-Dt, d.dx3, d.rdx3) * (E(1, 0, 0, 1) - E(1, 0, 0, 0));
        psf[1 * ks + c] = div_face_volume(d, m, temp, gdf, 4, gi);
    }
}

template <typename T>
__device__ __forceinline__ void k_face_update_at(const Dims &d, const Geom &m, const double *psi, double *psf,
                                                      const T *__restrict__ Et, StepSize st, const long t) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2, nz = d.n3 + d.d3;
    const int z = d.ng3 * d.d3 + (int)(t % nz);
    const int j = d.ng2 * d.d2 + (int)((t / nz) % nj);
    const int i = d.ng1 * d.d1 + (int)(t / ((long)nz * nj));
    (void)ni;
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    const long ks = d.ks, isize = (long)d.G2 * d.G3, jsz = d.G3;
    auto E = [&](int k, int di, int dj, int dz) {
        return (double)Et[k * ks + c + di * isize + dj * jsz + dz * d.d3];
    };
    face_update_eval(d, m, psi, psf, E, st.sub(), i, j, z, c, gi, 7);
}

// threads of k_face_update: two z face triples each
__host__ __device__ __forceinline__ long n_face_threads(const Dims &d) {
    return (long)(d.n1 + d.d1) * (d.n2 + d.d2) * ((d.n3 + d.d3 + 1) / 2);
}

// Two consecutive z face triples per thread (ZP = 2), so that the edge-EMF
// loads of both are in flight together; each triple is the one-item body.
template <typename T, int ZP = 2>
__global__ void __launch_bounds__(BLK) k_face_update(const Dims d, const Geom m, const double *psi, double *psf,
                                                      const T *__restrict__ Et, StepSize st) {
    const int ni = d.n1 + d.d1, nj = d.n2 + d.d2, nz = d.n3 + d.d3;
    const int nzp = (nz + ZP - 1) / ZP;
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (long)ni * nj * nzp) return;
    const long row = u / nzp;
    const int z0 = (int)(u % nzp) * ZP;
#pragma unroll
    for (int q = 0; q < ZP; q++)
        if (z0 + q < nz) k_face_update_at(d, m, psi, psf, Et, st, row * nz + z0 + q);
}

// ---------------------------------------------------------------- fused CT
// Constrained transport of a 3-D block in one kernel: centre EMFs, edge EMFs
// and the face update, with the centre and edge EMFs kept in shared memory
// instead of two HBM round trips. A CTA owns a tile of CT_TJ x CT_TZ (j, z)
// columns and marches along i over a chunk of planes, with two-plane rings:
// for plane i it builds the centre EMFs of plane i (tile plus a one-zone halo
// on the low j and z sides, which the edges need), then the edge EMFs of
// plane i (tile plus one edge on the high sides, which the faces need), then
// updates the faces of plane i - 1 (their upper edges lie in plane i). A
// chunk recomputes the centre and edge EMFs of the plane before it. Same
// expressions as k_emf_centre, k_emf_edge and k_face_update (the shared
// evaluators above), so the same values.
//
// With transmissive poles the polar x1-EMFs are replaced by their phi average
// over the whole ring (k_pole_average) before the faces next to the poles
// are updated: the kernel writes the edge EMFs of the two rows at each pole
// to the global array and leaves the faces of rows ng2, n2 + ng2 - 1 and
// n2 + ng2 to k_face_update_polar, which runs after the average.
//
// Measured on the 384 x 192 x 192 torus, per step: 4.0-5.0 ms (FP64) and
// 2.2-3.2 ms (float) over chunks of 4-24 planes and 2-4 CTAs per SM, against
// 2.7 and 1.9 ms for the three separate kernels: CTAs marching plane by plane
// with two barriers per plane keep too few loads in flight. The stage
// therefore runs the three kernels; HAMR_CT_FUSED=1 selects this one.
constexpr int CT_TZ = 32, CT_TJ = 8, CT_THREADS = CT_TZ * CT_TJ;
// build option: x1 planes per CTA of the fused CT kernel (more planes: less
// recomputed plane per chunk, fewer CTAs in flight)
#ifndef HAMR_CT_CHUNK
#define HAMR_CT_CHUNK 24
#endif

__device__ __forceinline__ bool ct_polar_row(const Dims &d, int j) {
    return d.bc2 == HAMR_BC_POLE_TRANS && (j == d.ng2 || j == d.n2 + d.ng2 - 1 || j == d.n2 + d.ng2);
}

template <typename T>
__global__ void __launch_bounds__(CT_THREADS, 2)
    k_ct_fused(const Dims d, const Geom m, const double *__restrict__ pv, const T *__restrict__ F1,
               const T *__restrict__ F2, const T *__restrict__ F3, const double *psi, double *psf,
               T *__restrict__ emf_g, StepSize st) {
    constexpr int EJ = CT_TJ + 2, EZ = CT_TZ + 2;   // centre-EMF tile with its low-side halo
    constexpr int GJ = CT_TJ + 1, GZ = CT_TZ + 1;   // edge tile with its high-side edge
    __shared__ T sEc[2][3][EJ][EZ];
    __shared__ T sE[2][3][GJ][GZ];
    const int tid = threadIdx.x;
    const int j0 = d.ng2 + blockIdx.y * CT_TJ, z0 = d.ng3 + blockIdx.x * CT_TZ;
    const int ia = d.ng1 + blockIdx.z * HAMR_CT_CHUNK;
    const int ib = min(ia + HAMR_CT_CHUNK, d.n1 + d.ng1 + 1);   // face planes [ia, ib)
    const int ie = min(ib, d.n1 + d.ng1);                        // last edge plane
    const long ks = d.ks, isize = (long)d.G2 * d.G3, jsz = d.G3;
    const double Dt = st.sub();
    const bool polar = d.bc2 == HAMR_BC_POLE_TRANS;
    // the faces of plane i from the edge rings (plane i in slot i & 1)
    auto faces = [&](int i) {
        const int jj = tid / CT_TZ, zz = tid % CT_TZ;
        const int j = j0 + jj, z = z0 + zz;
        if (j > d.n2 + d.ng2 || z > d.n3 + d.ng3 || ct_polar_row(d, j)) return;
        auto E = [&](int k, int di, int dj, int dz) { return (double)sE[(i + di) & 1][k - 1][jj + dj][zz + dz]; };
        face_update_eval(d, m, psi, psf, E, Dt, i, j, z, cix(d, i, j, z), gix(d, i, j), 7);
    };
    for (int i = ia - 1; i <= ie; i++) {
        // centre EMFs of plane i: zones j0-1 .. j0+CT_TJ, z0-1 .. z0+CT_TZ
        for (int e = tid; e < EJ * EZ; e += CT_THREADS) {
            const int jj = e / EZ, zz = e % EZ;
            const int j = j0 - 1 + jj, z = z0 - 1 + zz;
            if (j <= d.n2 + d.ng2 && z <= d.n3 + d.ng3) {
                T ec[3];
                emf_centre_eval(d, m, pv, i, j, cix(d, i, j, z), ec);
                sEc[i & 1][0][jj][zz] = ec[0];
                sEc[i & 1][1][jj][zz] = ec[1];
                sEc[i & 1][2][jj][zz] = ec[2];
            }
        }
        __syncthreads();
        if (i < ia) continue;
        // edge EMFs of plane i: edges j0 .. j0+CT_TJ, z0 .. z0+CT_TZ
        for (int e = tid; e < GJ * GZ; e += CT_THREADS) {
            const int jj = e / GZ, zz = e % GZ;
            const int j = j0 + jj, z = z0 + zz;
            if (j <= d.n2 + d.ng2 && z <= d.n3 + d.ng3) {
                const long c = cix(d, i, j, z);
                auto ec = [&](int k, int di, int dj, int dz) { return sEc[(i + di) & 1][k - 1][jj + 1 + dj][zz + 1 + dz]; };
                T ed[3];
                emf_edge_eval<T>(d, ec, F1, F2, F3, c, j, ed);
                sE[i & 1][0][jj][zz] = ed[0];
                sE[i & 1][1][jj][zz] = ed[1];
                sE[i & 1][2][jj][zz] = ed[2];
                if (polar && (j == d.ng2 || j == d.ng2 + 1 || j == d.n2 + d.ng2 - 1 || j == d.n2 + d.ng2)) {
                    emf_g[1 * ks + c] = ed[0];
                    emf_g[2 * ks + c] = ed[1];
                    emf_g[3 * ks + c] = ed[2];
                }
            }
        }
        __syncthreads();
        if (i - 1 >= ia) faces(i - 1);
    }
    // the last x1-face plane has no edge plane above it (x1 faces only)
    if (ib == d.n1 + d.ng1 + 1) {
        const int i = d.n1 + d.ng1;
        const int jj = tid / CT_TZ, zz = tid % CT_TZ;
        const int j = j0 + jj, z = z0 + zz;
        if (j <= d.n2 + d.ng2 && z <= d.n3 + d.ng3 && !ct_polar_row(d, j)) {
            auto E = [&](int k, int di, int dj, int dz) { return (double)sE[(i + di) & 1][k - 1][jj + dj][zz + dz]; };
            face_update_eval(d, m, psi, psf, E, Dt, i, j, z, cix(d, i, j, z), gix(d, i, j), 1);
        }
    }
    (void)isize;
    (void)jsz;
}

// the faces k_ct_fused leaves for after the polar average: rows ng2,
// n2 + ng2 - 1 and n2 + ng2, from the global edge EMFs
template <typename T>
__global__ void k_face_update_polar(const Dims d, const Geom m, const double *psi, double *psf,
                                    const T *__restrict__ Et, StepSize st) {
    const int ni = d.n1 + 1, nz = d.n3 + 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3L * ni * nz) return;
    const int z = d.ng3 + (int)(t % nz);
    const int i = d.ng1 + (int)((t / nz) % ni);
    const int r = (int)(t / ((long)nz * ni));
    const int j = r == 0 ? d.ng2 : (r == 1 ? d.n2 + d.ng2 - 1 : d.n2 + d.ng2);
    const long c = cix(d, i, j, z);
    const long ks = d.ks, isize = (long)d.G2 * d.G3, jsz = d.G3;
    auto E = [&](int k, int di, int dj, int dz) { return (double)Et[k * ks + c + di * isize + dj * jsz + dz]; };
    face_update_eval(d, m, psi, psf, E, st.sub(), i, j, z, c, gix(d, i, j), 7);
}

// geometric source gdet T^k_l Gamma^l_{jk} (source, GPU_phys_mhd.h:34-175)
// conn(s, k): the connection coefficient of symmetric pair s and index k at
// the zone's (i, j) column (from the tables, or staged in shared memory)
template <class Conn>
__device__ __forceinline__ void source_c(double gam, const double *ph, const Geo<double> &gm, Conn conn, double *dU,
                                         const State<double> &q) {
    double mhd[4][4];
    const double P = (gam - 1.) * ph[UU];
    const double u = ph[UU];
    const double w = P + ph[RHO] + u;
    const double bsq = dot4(q.bcon, q.bcov);
    const double eta = w + bsq;
    const double ptot = P + 0.5 * bsq;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
            mhd[a][b] = eta * q.ucon[a] * q.ucov[b] + ptot * (a == b ? 1. : 0.) - q.bcon[a] * q.bcov[b];
#pragma unroll
    for (int k = 0; k < NPR; k++) dU[k] = 0.;
#define CONN(s, k) conn((s), (k))
#pragma unroll
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

// connection accessors: from the tables (one (i, j) column: base pointer and
// plane stride), or from a column staged in shared memory
struct ConnTable {
    const double *conn;
    long gs, gi;
    __device__ __forceinline__ double operator()(int s, int k) const {
        return __ldg(&conn[(long)(s * 4 + k) * gs + gi]);
    }
};
struct ConnStaged {
    const double *g;   // 40 values, (s, k) at s * 4 + k
    __device__ __forceinline__ double operator()(int s, int k) const { return g[s * 4 + k]; }
};

// the same with the connection read from the tables (kept as its own body:
// the batched update spills less with it than through the accessor)
__device__ __forceinline__ void source(double gam, const double *ph, const Geo<double> &gm, const Dims &d,
                                       const Geom &m, long gi, double *dU, const State<double> &q) {
    double mhd[4][4];
    const long gs = d.gs;
    const double P = (gam - 1.) * ph[UU];
    const double u = ph[UU];
    const double w = P + ph[RHO] + u;
    const double bsq = dot4(q.bcon, q.bcov);
    const double eta = w + bsq;
    const double ptot = P + 0.5 * bsq;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
            mhd[a][b] = eta * q.ucon[a] * q.ucov[b] + ptot * (a == b ? 1. : 0.) - q.bcon[a] * q.bcov[b];
#pragma unroll
    for (int k = 0; k < NPR; k++) dU[k] = 0.;
#define CONN(s, k) __ldg(&m.conn[(long)((s) * 4 + (k)) * gs + gi])
#pragma unroll
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

// Conserved update of one active zone (fixup, GPU_fixup.h:5-424, up to the
// inversion): U(p^n) computed and cached by the half sub-step or read back by
// the full one, minus the flux divergence, plus the geometric source at the
// stage's primitives; U[B] from the face-averaged staggered field. pf returns
// the stage's primitives (the inversion's initial guess).
// FX(dir, k, up): flux k of direction dir on the zone's lower face (up = 0)
// or upper face (up = 1).
template <typename T, class Conn, class FX>
__device__ __forceinline__ void cons_update_fx(const Dims &d, const Geom &m, const double *__restrict__ pin,
                                               const double *__restrict__ pb, double *__restrict__ Ucache, FX FX_,
                                               int full, double Dt, int i, int j, long c, long gi,
                                               const Geo<double> &gm, Conn conn, double *pf, double *U) {
    const long ks = d.ks;
    State<double> q;
    double dU[NPR];
    if (!full) {
#pragma unroll
        for (int k = 0; k < NPR; k++) { pf[k] = 0.0; pf[k] += (1.0 / ((double)1)) * pin[k * ks + c]; }
        get_state(pf, gm, q);
        double vd;
        primtoflux(d.gam, pf, q, 0, gm, entropy(d.gam, pf), U, &vd, &vd);
#pragma unroll
        for (int k = 0; k < NPR; k++) Ucache[k * ks + c] = U[k];
    } else {
#pragma unroll
        for (int k = 0; k < NPR; k++) U[k] = Ucache[k * ks + c];
#pragma unroll
        for (int k = 0; k < NPR; k++) { pf[k] = 0.0; pf[k] += (1.0 / ((double)1)) * pb[k * ks + c]; }
        get_state(pf, gm, q);
    }
    if constexpr (sizeof(T) == sizeof(double)) {
#pragma unroll
        for (int k = 0; k < NPR; k++) {
            if (d.ng1 > 0) U[k] -= div_rcp(Dt * (FX_(1, k, 1) - FX_(1, k, 0)), d.dx1, d.rdx1);
            if (d.ng2 > 0) U[k] -= div_rcp(Dt * (FX_(2, k, 1) - FX_(2, k, 0)), d.dx2, d.rdx2);
            if (d.ng3 > 0) U[k] -= div_rcp(Dt * (FX_(3, k, 1) - FX_(3, k, 0)), d.dx3, d.rdx3);
        }
        if constexpr (std::is_same<Conn, ConnTable>::value) source(d.gam, pf, gm, d, m, gi, dU, q);
        else source_c(d.gam, pf, gm, conn, dU, q);
#pragma unroll
        for (int k = 0; k < NPR; k++) U[k] += Dt * (dU[k]);
    } else {
        // float fluxes: differences taken in double (exact for two floats of
        // similar size) and the four increments added to U^n with Neumaier
        // compensated summation
        if constexpr (std::is_same<Conn, ConnTable>::value) source(d.gam, pf, gm, d, m, gi, dU, q);
        else source_c(d.gam, pf, gm, conn, dU, q);
#pragma unroll
        for (int k = 0; k < NPR; k++) {
            double sum = U[k], comp = 0.;
            auto add = [&](double x) {
                const double tt = sum + x;
                comp += fabs(sum) >= fabs(x) ? (sum - tt) + x : (x - tt) + sum;
                sum = tt;
            };
            if (d.ng1 > 0) add(div_rcp(-Dt * ((double)FX_(1, k, 1) - (double)FX_(1, k, 0)), d.dx1, d.rdx1));
            if (d.ng2 > 0) add(div_rcp(-Dt * ((double)FX_(2, k, 1) - (double)FX_(2, k, 0)), d.dx2, d.rdx2));
            if (d.ng3 > 0) add(div_rcp(-Dt * ((double)FX_(3, k, 1) - (double)FX_(3, k, 0)), d.dx3, d.rdx3));
            add(Dt * dU[k]);
            U[k] = sum + comp;
        }
    }
}

// the same with the fluxes read from the global arrays
template <typename T, class Conn>
__device__ __forceinline__ void cons_update(const Dims &d, const Geom &m, const double *__restrict__ pin,
                                            const double *__restrict__ pb, double *__restrict__ Ucache,
                                            const T *__restrict__ F1, const T *__restrict__ F2,
                                            const T *__restrict__ F3, int full, double Dt, int i, int j,
                                            long c, long gi, const Geo<double> &gm, Conn conn, double *pf,
                                            double *U) {
    const long ks = d.ks, isize = (long)d.G2 * d.G3;
    auto fx = [&](int dir, int k, int up) -> T {
        return dir == 1 ? F1[k * ks + c + up * isize] : (dir == 2 ? F2[k * ks + c + up * d.G3] : F3[k * ks + c + up]);
    };
    cons_update_fx<T>(d, m, pin, pb, Ucache, fx, full, Dt, i, j, c, gi, gm, conn, pf, U);
}

// U[B] from the face-averaged staggered field (fixup, GPU_fixup.h:330-345)
__device__ __forceinline__ void face_average_b(const Dims &d, const Geom &m, const double *__restrict__ psf, int i,
                                               int j, long c, long gi, double *U) {
    const long ks = d.ks, isize = (long)d.G2 * d.G3;
    U[B1] = 0.0;
    U[B2] = 0.0;
    U[B1] += (psf[0 * ks + c] * m.gdet[FACE1 * d.gs + gi] + psf[0 * ks + c + isize] * m.gdet[FACE1 * d.gs + gix(d, i + d.d1, j)]) / (2.0 * (double)1);
    U[B2] += (psf[1 * ks + c] * m.gdet[FACE2 * d.gs + gi] + psf[1 * ks + c + d.G3] * m.gdet[FACE2 * d.gs + gix(d, i, j + d.d2)]) / (2.0 * (double)1);
    if (d.ng3 > 0)
        U[B3] = (psf[2 * ks + c] * m.gdet[FACE3 * d.gs + gi] + psf[2 * ks + c + 1 * d.d3] * m.gdet[FACE3 * d.gs + gi]) / 2.0;
}

// Opt-in work after the inversion (template bits of the inversion kernel):
// FIX_FLOORS the drift-frame floors (fixup_cell's body, GPU_fixup.h:1025-1800,
// compiled out in the reference) with the gamma-failure flag -333 and
// counter 3 of the fixup kernel (GPU_fixup.h:398-415); FIX_RESET the reset of
// failed zones to the floor state (fixuputoprim, GPU_fixup.h:735-852, whose
// call is commented out at step_ch.c:1281), fused here because it reads only
// the zone's own flag and primitives.
enum { FIX_FLOORS = 1, FIX_RESET = 2 };

// The entropy fallbacks 1dvsq2fix1 then 1dfix1 of a zone whose primary
// solver failed, counting each failure (fixup, GPU_fixup.h:360-382); returns
// the final flag. Works on copies so that the caller's U and pf can stay in
// registers.
__device__ __forceinline__ int invert_fallbacks(const Dims &d, const Geo<double> &gm, long c, const double *U,
                                                double *pf, int *__restrict__ failimage) {
    const long ks = d.ks;
    double Uc[NPR], pc[NPR], gcv[10], gcn[10];
#pragma unroll
    for (int k = 0; k < NPR; k++) { Uc[k] = U[k]; pc[k] = pf[k]; }
#pragma unroll
    for (int k = 0; k < 10; k++) { gcv[k] = gm.gcov[k]; gcn[k] = gm.gcon[k]; }
    failimage[c]++;
    int flag = utoprim_1dvsq2fix1(d.gam, Uc, gcv, gcn, gm.g, pc);
    if (flag) {
        failimage[1 * ks + c]++;
        flag = utoprim_1dfix1(d.gam, Uc, gcv, gcn, gm.g, pc);
        if (flag) failimage[2 * ks + c]++;
    }
#pragma unroll
    for (int k = 0; k < NPR; k++) pf[k] = pc[k];
    return flag;
}

// The opt-in floors and reset after the inversion chain, then the zone's
// flag and primitives written out.
template <int FIX>
__device__ __forceinline__ void invert_epilogue(const Dims &d, const Geo<double> &gm, long c, int flag, double *pf,
                                                double *__restrict__ pout, int *__restrict__ pflag,
                                                int *__restrict__ failimage) {
    const long ks = d.ks;
    if constexpr ((FIX & FIX_FLOORS) != 0) {
        if (floor_may_apply(pf, gm) && floor_zone(d.gam, pf, gm)) {
            flag = -333;
            failimage[3 * ks + c]++;
        }
    }
    if constexpr ((FIX & FIX_RESET) != 0) {
        if (flag != 0) {
            pf[RHO] = RHOMINLIMIT;
            pf[UU] = UUMINLIMIT;
            pf[U1] = 0.0;
            pf[U2] = 0.0;
            pf[U3] = 0.0;
            if constexpr ((FIX & FIX_FLOORS) != 0) (void)floor_zone(d.gam, pf, gm);
        }
    }
    pflag[c] = flag;
#pragma unroll
    for (int k = 0; k < NPR; k++) pout[k * ks + c] = pf[k];
}

// the inversion's per-zone constants, from the column table when there is one
__device__ __forceinline__ InvK inv_k(const Dims &d, const Geom &m, long gi, const Geo<double> &gm) {
    if (m.itab)
        return InvK{d.gam, d.rgam, gm.g, __ldg(&m.itab[gi]), __ldg(&m.itab[d.gs + gi]),
                    __ldg(&m.itab[2 * d.gs + gi])};
    return inv_consts(d.gam, d.rgam, gm.g, gm.gcon);
}

// the column table: at the zone centre of every (i, j), with the operations
// of inv_consts, so that a tabulated value equals the one computed in place
__global__ void k_inv_tab(const Dims d, const double *__restrict__ gcon, const double *__restrict__ gdet,
                          double *__restrict__ itab) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d.gs) return;
    const double g = gdet[(long)CENT * d.gs + idx];
    const double g00 = gcon[(long)CENT * d.gs + idx];   // component 0, location CENT
    itab[idx] = 1.0 / g;
    itab[d.gs + idx] = 1.0 / sqrt(-g00);
    itab[2 * d.gs + idx] = -sqrt(-1. / g00);
    itab[3 * d.gs + idx] = 1.0 / gdet[(long)FACE1 * d.gs + idx];
    itab[4 * d.gs + idx] = 1.0 / gdet[(long)FACE2 * d.gs + idx];
    itab[5 * d.gs + idx] = 1.0 / gdet[(long)FACE3 * d.gs + idx];
    for (int loc = 0; loc < 5; loc++) {
        const double a = 1. / sqrt(-gcon[(long)loc * d.gs + idx]);   // g^tt at loc (component 0)
        itab[(long)(6 + loc) * d.gs + idx] = a;
        itab[(long)(11 + loc) * d.gs + idx] = 1. / a;
    }
}


// primary solver: Noble 2D, or Newman-Hamlin in its place (NEWMAN builds)
template <int INV>
__device__ __forceinline__ int invert_primary(const Dims &d, const InvK &k, const Geo<double> &gm, const double *U,
                                              double *pf) {
    return INV == HAMR_INV_NM ? utoprim_nm(d.gam, U, gm.gcov, gm.gcon, gm.g, pf)
                              : utoprim_2d_k(k, U, gm.gcov, gm.gcon, pf);
}

// Primary inversion with the 1dvsq2fix1 and 1dfix1 fallbacks, recording the
// outcome in pflag and the failure counters (fixup, GPU_fixup.h:346-382),
// all in one pass (the batched inversion's per-item body)
template <int INV, int FIX = 0>
__device__ __forceinline__ void invert_zone(const Dims &d, const InvK &k, const Geo<double> &gm, long c, double *U,
                                            double *pf,
                                            double *__restrict__ pout, int *__restrict__ pflag,
                                            int *__restrict__ failimage) {
    int flag = invert_primary<INV>(d, k, gm, U, pf);
    if (flag) flag = invert_fallbacks(d, gm, c, U, pf, failimage);
    invert_epilogue<FIX>(d, gm, c, flag, pf, pout, pflag, failimage);
}

// build option: minimum resident blocks of 128 threads per SM for the
// inversion kernels (caps their registers per thread; on the 384 x 192 x 192
// torus, per step, for the primary-solver kernel: 8 blocks 3.18 ms (mixed
// step) / 3.07 ms (FP64), 7: 3.34 / 3.21, 6: 3.36 / 3.21)
#ifndef HAMR_UPD_MINB
#define HAMR_UPD_MINB 8
#endif

// The update in two kernels, so that each holds fewer registers and more
// zones are in flight: k_cons writes the six non-magnetic conserved variables
// and U[B3] to seven scratch planes W; k_invert reads them back, sets U[B]
// from the faces and inverts.
// build option: minimum resident blocks of 128 threads per SM for the
// conserved update (memory-latency bound: more zones in flight pay for the
// spills of a 64-register cap)
#ifndef HAMR_CONS_MINB
#define HAMR_CONS_MINB 8
#endif
template <typename T>
__device__ __forceinline__ void k_cons_at(const Dims &d, const Geom &m, const double *__restrict__ pin,
                                               const double *__restrict__ pb, double *__restrict__ Ucache,
                                               const T *__restrict__ F1, const T *__restrict__ F2,
                                               const T *__restrict__ F3, double *__restrict__ W, int full,
                                               StepSize st, const long t) {
    const int z = d.ng3 + (int)(t % d.n3);
    const int j = d.ng2 + (int)((t / d.n3) % d.n2);
    const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    Geo<double> gm;
    load_geo(d, m, i, j, CENT, gm);
    double pf[NPR], U[NPR];
    cons_update<T>(d, m, pin, pb, Ucache, F1, F2, F3, full, st.sub(), i, j, c, gi, gm, ConnTable{m.conn, d.gs, gi},
                   pf, U);
    W[0 * d.ks + c] = U[RHO];
    W[1 * d.ks + c] = U[UU];
    W[2 * d.ks + c] = U[U1];
    W[3 * d.ks + c] = U[U2];
    W[4 * d.ks + c] = U[U3];
    W[5 * d.ks + c] = U[KTOT];
    W[6 * d.ks + c] = U[B3];   // kept in 2-D, where the faces do not set it
}

template <typename T>
__global__ void __launch_bounds__(BLK, HAMR_CONS_MINB) k_cons(const Dims d, const Geom m, const double *__restrict__ pin,
                                               const double *__restrict__ pb, double *__restrict__ Ucache,
                                               const T *__restrict__ F1, const T *__restrict__ F2,
                                               const T *__restrict__ F3, double *__restrict__ W, int full,
                                               StepSize st, int *__restrict__ nfail) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *nfail = 0;   // the inversion's failed-zone list starts empty
    if (t >= (long)d.n1 * d.n2 * d.n3) return;
    k_cons_at(d, m, pin, pb, Ucache, F1, F2, F3, W, full, st, t);
}

// The same update with the zones' metric and connection staged in shared
// memory: the zones of a CTA lie in at most three (i, j) columns when
// n3 >= 64 (z runs fastest), whose 61 metric and connection values each are
// loaded once per CTA instead of once per zone.
constexpr int COL_VALS = 61;   // gcov 10, gcon 10, gdet 1 (centre), conn 40
template <typename T>
__global__ void __launch_bounds__(BLK, HAMR_CONS_MINB) k_cons_cols(const Dims d, const Geom m,
                                               const double *__restrict__ pin, const double *__restrict__ pb,
                                               double *__restrict__ Ucache, const T *__restrict__ F1,
                                               const T *__restrict__ F2, const T *__restrict__ F3,
                                               double *__restrict__ W, int full, StepSize st,
                                               int *__restrict__ nfail) {
    __shared__ double sg[3][COL_VALS];
    if (blockIdx.x == 0 && threadIdx.x == 0) *nfail = 0;   // the inversion's failed-zone list starts empty
    const long nzone = (long)d.n1 * d.n2 * d.n3;
    const long t0 = (long)blockIdx.x * blockDim.x;
    const long tl = (t0 + blockDim.x < nzone ? t0 + blockDim.x : nzone) - 1;
    const long col0 = t0 / d.n3, ncol = tl / d.n3 - col0 + 1;   // <= 3 for n3 >= 64
    const long gs = d.gs;
    for (int e = threadIdx.x; e < ncol * COL_VALS; e += blockDim.x) {
        const long col = col0 + e / COL_VALS;
        const int v = e % COL_VALS;
        const long gi = gix(d, d.ng1 + (int)(col / d.n2), d.ng2 + (int)(col % d.n2));
        double x;
        if (v < 10) x = m.gcov[(long)(v * 5 + CENT) * gs + gi];
        else if (v < 20) x = m.gcon[(long)((v - 10) * 5 + CENT) * gs + gi];
        else if (v == 20) x = m.gdet[(long)CENT * gs + gi];
        else x = m.conn[(long)(v - 21) * gs + gi];
        sg[e / COL_VALS][v] = x;
    }
    __syncthreads();
    const long t = t0 + threadIdx.x;
    if (t >= nzone) return;
    const int z = d.ng3 + (int)(t % d.n3);
    const int j = d.ng2 + (int)((t / d.n3) % d.n2);
    const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    const double *g = sg[t / d.n3 - col0];
    Geo<double> gm;
#pragma unroll
    for (int q = 0; q < 10; q++) { gm.gcov[q] = g[q]; gm.gcon[q] = g[10 + q]; }
    gm.g = g[20];
    geo_lapse(gm);
    double pf[NPR], U[NPR];
    cons_update<T>(d, m, pin, pb, Ucache, F1, F2, F3, full, st.sub(), i, j, c, gi, gm, ConnStaged{g + 21}, pf, U);
    W[0 * d.ks + c] = U[RHO];
    W[1 * d.ks + c] = U[UU];
    W[2 * d.ks + c] = U[U1];
    W[3 * d.ks + c] = U[U2];
    W[4 * d.ks + c] = U[U3];
    W[5 * d.ks + c] = U[KTOT];
    W[6 * d.ks + c] = U[B3];
}

// the inversion's inputs of one zone: the stage's primitives as the initial
// guess, the updated conserved variables, U[B] from the faces
__device__ __forceinline__ void invert_inputs(const Dims &d, const Geom &m, const double *__restrict__ pg,
                                              const double *__restrict__ W, const double *__restrict__ psf,
                                              int i, int j, long c, long gi, double *pf, double *U) {
#pragma unroll
    for (int k = 0; k < NPR; k++) pf[k] = pg[k * d.ks + c];
    U[RHO] = W[0 * d.ks + c];
    U[UU] = W[1 * d.ks + c];
    U[U1] = W[2 * d.ks + c];
    U[U2] = W[3 * d.ks + c];
    U[U3] = W[4 * d.ks + c];
    U[KTOT] = W[5 * d.ks + c];
    U[B3] = W[6 * d.ks + c];
    face_average_b(d, m, psf, i, j, c, gi, U);
}

// ------------------------------------------- TMA-staged conserved update
// The conserved update of one (i, j) row of zones (or an equal piece of it)
// per CTA, with the 45 flux operands of every zone -- the x1 fluxes on both
// faces, the x2 fluxes on both faces, the x3 fluxes of the row and one more
// -- brought into shared memory by bulk asynchronous copies (TMA,
// cp.async.bulk) before any arithmetic: 45 copies per row, completion
// counted on one mbarrier, all in flight at once, where a thread of the
// one-zone-per-thread kernel can only keep as many loads in flight as its
// registers hold. A bulk copy must start and end on 16-byte boundaries: each
// copied segment is widened to them and indexed from its offset. Same
// expressions as k_cons / k_cons_cols (cons_update_fx), so the same values.
//
// The wait on the barrier is bounded: a CTA that gives up sets *kerr and
// waits again, also bounded, for its copies before it returns without
// computing; the host reports the flag as an error.
__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    for (int it = 0; it < (1 << 20); it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completion counted on the barrier
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// shared-memory layout of one CTA of k_cons_tma, in bytes
struct ConsTmaLayout {
    int cap;       // elements per staged segment (a piece of lpiece zones, widened)
    int seg_bytes; // cap * sizeof(T), a multiple of 16
    int f_off;     // first segment (after the barrier and the metric column)
    int total;
};
template <typename T>
__host__ __device__ __forceinline__ ConsTmaLayout cons_tma_layout(int lpiece) {
    constexpr int A = 16 / (int)sizeof(T);
    ConsTmaLayout L;
    L.cap = ((lpiece + 1 + 2 * (A - 1)) + A - 1) / A * A;
    L.seg_bytes = L.cap * (int)sizeof(T);
    L.f_off = 16 + ((COL_VALS * 8 + 15) / 16) * 16;
    L.total = L.f_off + 5 * NPR * L.seg_bytes;
    return L;
}

// build option: resident CTAs per SM of the TMA-staged update (caps its
// registers; measured on the 384 x 192 x 192 torus, per step: float 3 (2.86
// ms; 2: 4.05, 4: 2.88), double 4 (3.67 ms; 2: 4.05, 3: 3.86))
#ifndef HAMR_CONS_TMA_MINB_F
#define HAMR_CONS_TMA_MINB_F 3
#endif
#ifndef HAMR_CONS_TMA_MINB
#define HAMR_CONS_TMA_MINB 4
#endif
// FUSE: 0 writes the seven planes of W for the inversion kernels; HAMR_INV_2D
// + 1 or HAMR_INV_NM + 1 runs the primary inversion of each zone right after
// its update (no floors or repair): the guess is pb (the state the update
// read), the face field psf, the output pout, and only a zone whose primary
// solver fails writes W and goes to the list for k_invert_fallback (*nfail
// cleared before the launch). The W round trip and the inversion's reload of
// the guess disappear; same values as the update followed by
// k_invert_primary.
#ifndef HAMR_CONS_INV_TMA_MINB   // the same kernel with the primary inversion inside (FUSE != 0);
#define HAMR_CONS_INV_TMA_MINB 3    // FP64 at 4 blocks spills 0.6 KB a thread (measured C3 update+inversion
#endif                              // 5.35 ms at 3 blocks, 6.0 at 4, 5.43 at 2)
#ifndef HAMR_CONS_INV_TMA_MINB_F
#define HAMR_CONS_INV_TMA_MINB_F HAMR_CONS_TMA_MINB_F
#endif
// The body of one CTA: row piece `blk` (row * npiece + piece) of the block,
// `smem` the CTA's dynamic shared memory (cons_tma_layout(lpiece).total bytes).
template <typename T, int FUSE>
__device__ __forceinline__ void cons_tma_row(const Dims &d, const Geom &m, const double *__restrict__ pin,
                                             const double *__restrict__ pb, double *__restrict__ Ucache,
                                             const T *__restrict__ F1, const T *__restrict__ F2,
                                             const T *__restrict__ F3, double *__restrict__ W, int full,
                                             const StepSize &st, int *__restrict__ nfail, int *__restrict__ kerr,
                                             int npiece, int lpiece, int blk, unsigned char *smem,
                                             const double *__restrict__ psf, double *__restrict__ pout,
                                             int *__restrict__ pflag, int *__restrict__ failimage,
                                             int *__restrict__ flist) {
    constexpr int A = 16 / (int)sizeof(T);
    const ConsTmaLayout lay = cons_tma_layout<T>(lpiece);
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(smem);
    double *sg = reinterpret_cast<double *>(smem + 16);
    T *sf = reinterpret_cast<T *>(smem + lay.f_off);   // [kind][plane][cap]
    const unsigned bar_a = smem_addr(bar);
    const int row = blk / npiece, piece = blk % npiece;
    const int i = d.ng1 + row / d.n2, j = d.ng2 + row % d.n2;
    const int za = d.ng3 + piece * lpiece;
    const int L = min(lpiece, d.n3 - piece * lpiece);
    const long ks = d.ks, isize = (long)d.G2 * d.G3;
    const long c0 = cix(d, i, j, za), gi = gix(d, i, j);
    if (!FUSE && blk == 0 && threadIdx.x == 0) *nfail = 0;   // the inversion's failed-zone list starts empty
    // the five segment kinds: start cell, length, source array
    auto seg_start = [&](int q) -> long { return q == 1 ? c0 + isize : (q == 3 ? c0 + d.G3 : c0); };
    auto seg_len = [&](int q) -> int { return q == 4 ? L + 1 : L; };
    auto seg_src = [&](int q) -> const T * { return q < 2 ? F1 : (q < 4 ? F2 : F3); };
    if (threadIdx.x == 0) mbar_init(bar_a, 1);
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned total = 0;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const long s0 = seg_start(q), sa = s0 & ~(long)(A - 1);
            const long se = (s0 + seg_len(q) + A - 1) & ~(long)(A - 1);
            total += (unsigned)((se - sa) * (long)sizeof(T)) * NPR;
        }
        if (threadIdx.x == 0) mbar_expect_tx(bar_a, total);
        __syncwarp();
        for (int e = threadIdx.x; e < 5 * NPR; e += 32) {
            const int q = e / NPR, k = e % NPR;
            const long s0 = seg_start(q), sa = s0 & ~(long)(A - 1);
            const long se = (s0 + seg_len(q) + A - 1) & ~(long)(A - 1);
            bulk_g2s(smem_addr(sf + (long)e * lay.cap), seg_src(q) + (long)k * ks + sa,
                     (unsigned)((se - sa) * (long)sizeof(T)), bar_a);
        }
    }
    // the row's metric and connection column, while the copies fly
    for (int v = threadIdx.x; v < COL_VALS; v += blockDim.x) {
        double x;
        if (v < 10) x = m.gcov[(long)(v * 5 + CENT) * d.gs + gi];
        else if (v < 20) x = m.gcon[(long)((v - 10) * 5 + CENT) * d.gs + gi];
        else if (v == 20) x = m.gdet[(long)CENT * d.gs + gi];
        else x = m.conn[(long)(v - 21) * d.gs + gi];
        sg[v] = x;
    }
    __syncthreads();
    if (!mbar_wait(bar_a, 0)) {
        atomicExch(kerr, 1);
        (void)mbar_wait(bar_a, 0);   // let the copies land before the CTA's shared memory goes
        return;
    }
    const int l = threadIdx.x;
    if (l >= L) return;
    const long c = c0 + l;
    int off[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const long s0 = seg_start(q);
        off[q] = (int)(s0 - (s0 & ~(long)(A - 1))) + l;
    }
    auto fx = [&](int dir, int k, int up) -> T {
        const int q = dir == 1 ? up : (dir == 2 ? 2 + up : 4);
        return sf[(long)(q * NPR + k) * lay.cap + off[q] + (dir == 3 ? up : 0)];
    };
    Geo<double> gm;
#pragma unroll
    for (int q = 0; q < 10; q++) { gm.gcov[q] = sg[q]; gm.gcon[q] = sg[10 + q]; }
    gm.g = sg[20];
    geo_lapse(gm);
    double pf[NPR], U[NPR];
    cons_update_fx<T>(d, m, pin, pb, Ucache, fx, full, st.sub(), i, j, c, gi, gm, ConnStaged{sg + 21}, pf, U);
    auto write_w = [&]() {
        W[0 * d.ks + c] = U[RHO];
        W[1 * d.ks + c] = U[UU];
        W[2 * d.ks + c] = U[U1];
        W[3 * d.ks + c] = U[U2];
        W[4 * d.ks + c] = U[U3];
        W[5 * d.ks + c] = U[KTOT];
        W[6 * d.ks + c] = U[B3];
    };
    if constexpr (FUSE == 0) {
        write_w();
    } else {
        constexpr int INV = FUSE - 1;
        const double Uw[7] = {U[RHO], U[UU], U[U1], U[U2], U[U3], U[KTOT], U[B3]};
        // the inversion's inputs as k_invert_primary reads them: the guess
        // straight from pb, U[B] from the updated faces
#pragma unroll
        for (int k = 0; k < NPR; k++) pf[k] = pb[k * ks + c];
        face_average_b(d, m, psf, i, j, c, gi, U);
        const int flag = invert_primary<INV>(d, inv_k(d, m, gi, gm), gm, U, pf);
        if (flag) {
            U[RHO] = Uw[0]; U[UU] = Uw[1]; U[U1] = Uw[2]; U[U2] = Uw[3]; U[U3] = Uw[4]; U[KTOT] = Uw[5];
            U[B3] = Uw[6];
            write_w();
            const long t = ((long)(i - d.ng1) * d.n2 + (j - d.ng2)) * d.n3 + (za - d.ng3 + l);
            flist[atomicAdd(nfail, 1)] = (int)t;
            return;
        }
        invert_epilogue<0>(d, gm, c, flag, pf, pout, pflag, failimage);
    }
}

template <typename T, int FUSE = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? (FUSE ? HAMR_CONS_INV_TMA_MINB : HAMR_CONS_TMA_MINB)
                                                       : (FUSE ? HAMR_CONS_INV_TMA_MINB_F : HAMR_CONS_TMA_MINB_F))
    k_cons_tma(const Dims d, const Geom m, const double *__restrict__ pin, const double *__restrict__ pb,
               double *__restrict__ Ucache, const T *__restrict__ F1, const T *__restrict__ F2,
               const T *__restrict__ F3, double *__restrict__ W, int full, StepSize st, int *__restrict__ nfail,
               int *__restrict__ kerr, int npiece, int lpiece, const double *__restrict__ psf = nullptr,
               double *__restrict__ pout = nullptr, int *__restrict__ pflag = nullptr,
               int *__restrict__ failimage = nullptr, int *__restrict__ flist = nullptr) {
    extern __shared__ __align__(16) unsigned char smem[];
    cons_tma_row<T, FUSE>(d, m, pin, pb, Ucache, F1, F2, F3, W, full, st, nfail, kerr, npiece, lpiece, blockIdx.x,
                          smem, psf, pout, pflag, failimage, flist);
}

template <int INV, int FIX = 0>
__device__ __forceinline__ void k_invert_at(const Dims &d, const Geom &m, const double *__restrict__ pg,
                                                 const double *__restrict__ W, const double *__restrict__ psf,
                                                 double *__restrict__ pout, int *__restrict__ pflag,
                                                 int *__restrict__ failimage, const long t) {
    const int z = d.ng3 + (int)(t % d.n3);
    const int j = d.ng2 + (int)((t / d.n3) % d.n2);
    const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    Geo<double> gm;
    load_geo(d, m, i, j, CENT, gm);
    double pf[NPR], U[NPR];
    invert_inputs(d, m, pg, W, psf, i, j, c, gi, pf, U);
    invert_zone<INV, FIX>(d, inv_k(d, m, gi, gm), gm, c, U, pf, pout, pflag, failimage);
}

// The single-block inversion in two passes, so that the common path carries
// none of the fallbacks' state: k_invert_primary runs the primary solver
// and, for the zones it solves, the epilogue; a zone it fails goes to a list
// (its active-zone index) and is finished by k_invert_fallback, which
// rebuilds the zone's U from the same inputs, restores what the failed
// primary solver left in pf (U[B]/gdet, written by its prologue unless
// U[RHO] <= 0) and runs the fallback chain and the epilogue. Same results
// as the one-pass invert_zone; *nfail must be zero on entry (the conserved
// update clears it).
template <int INV, int FIX = 0>
__global__ void __launch_bounds__(BLK, HAMR_UPD_MINB)
    k_invert_primary(const Dims d, const Geom m, const double *__restrict__ pg, const double *__restrict__ W,
                     const double *__restrict__ psf, double *__restrict__ pout, int *__restrict__ pflag,
                     int *__restrict__ failimage, int *__restrict__ flist, int *__restrict__ nfail) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)d.n1 * d.n2 * d.n3) return;
    const int z = d.ng3 + (int)(t % d.n3);
    const int j = d.ng2 + (int)((t / d.n3) % d.n2);
    const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    Geo<double> gm;
    load_geo(d, m, i, j, CENT, gm);
    double pf[NPR], U[NPR];
    invert_inputs(d, m, pg, W, psf, i, j, c, gi, pf, U);
    const int flag = invert_primary<INV>(d, inv_k(d, m, gi, gm), gm, U, pf);
    if (flag) {
        flist[atomicAdd(nfail, 1)] = (int)t;
        return;
    }
    invert_epilogue<FIX>(d, gm, c, flag, pf, pout, pflag, failimage);
}

// the fallback chain and epilogue of one listed zone (active-zone index t)
template <int FIX>
__device__ __forceinline__ void invert_fallback_at(const Dims &d, const Geom &m, const double *__restrict__ pg,
                                                   const double *__restrict__ W, const double *__restrict__ psf,
                                                   double *__restrict__ pout, int *__restrict__ pflag,
                                                   int *__restrict__ failimage, const long t) {
    const int z = d.ng3 + (int)(t % d.n3);
    const int j = d.ng2 + (int)((t / d.n3) % d.n2);
    const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
    const long c = cix(d, i, j, z), gi = gix(d, i, j);
    Geo<double> gm;
    load_geo(d, m, i, j, CENT, gm);
    double pf[NPR], U[NPR];
    invert_inputs(d, m, pg, W, psf, i, j, c, gi, pf, U);
    if (!(U[RHO] <= 0.)) {
#pragma unroll
        for (int k = B1; k <= B3; k++) pf[k] = U[k] / gm.g;   // the primary solver's prologue
    }
    const int flag = invert_fallbacks(d, gm, c, U, pf, failimage);
    invert_epilogue<FIX>(d, gm, c, flag, pf, pout, pflag, failimage);
}

template <int INV, int FIX = 0>
__global__ void __launch_bounds__(BLK)
    k_invert_fallback(const Dims d, const Geom m, const double *__restrict__ pg, const double *__restrict__ W,
                      const double *__restrict__ psf, double *__restrict__ pout, int *__restrict__ pflag,
                      int *__restrict__ failimage, const int *__restrict__ flist, const int *__restrict__ nfail) {
    const int n = *nfail;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        invert_fallback_at<FIX>(d, m, pg, W, psf, pout, pflag, failimage, flist[q]);
}

// ------------------------------------------------ neighbour repair (opt-in)
// fixup_utoprim (fixup.c:764-827): every failed active zone, in (i, j, z)
// order, takes the average of the first usable stencil of good neighbours
// (x1-x2 plane numbered 1 2 3 / 8 x 4 / 7 6 5 with 1 at (i-1, j+1); 9 and 10
// at z+1 and z-1), and then counts as good for the zones after it; only RHO
// .. U3 change. The two-point x1 and x2 stencils are chosen by the flags of
// the other direction, as the reference writes them.
//
// The order only matters between failed zones within each other's stencil.
// k_repair_scan repairs at once every failed zone with no failed active zone
// in its stencil (nothing else reads or writes what it touches) and lists
// the others; k_repair_chain, one CTA, repairs the listed zones in waves: a
// zone is ready once no failed active zone with a smaller index is left in
// its stencil, and ready zones never neighbour each other, so each wave runs
// in parallel and the result is the sequential one. Every wave repairs at
// least the smallest pending zone, so at most as many waves as listed zones.
struct RepairStencil {
    long si, sj, sz;
};

__device__ __forceinline__ bool active_zone(const Dims &d, long c) {
    const int z = (int)(c % d.G3), j = (int)((c / d.G3) % d.G2), i = (int)(c / ((long)d.G3 * d.G2));
    return i >= d.ng1 && i < d.ng1 + d.n1 && j >= d.ng2 && j < d.ng2 + d.n2 && z >= d.ng3 && z < d.ng3 + d.n3;
}

// the ten stencil offsets in the reference's numbering 1..10 (index 0 unused)
__device__ __forceinline__ long stencil_offset(const RepairStencil &o, int q) {
    switch (q) {
        case 1: return -o.si + o.sj;
        case 2: return o.sj;
        case 3: return o.si + o.sj;
        case 4: return o.si;
        case 5: return o.si - o.sj;
        case 6: return -o.sj;
        case 7: return -o.si - o.sj;
        case 8: return -o.si;
        case 9: return o.sz;
        default: return -o.sz;
    }
}

// a failed active zone among the stencil of c (before c only, when `before`)
__device__ __forceinline__ bool failed_neighbour(const Dims &d, const RepairStencil &o, const int *pflag, long c,
                                                 bool before) {
    for (int q = 1; q <= 10; q++) {
        const long off = stencil_offset(o, q);
        if (off == 0 || (before && off > 0)) continue;
        if (pflag[c + off] != 0 && active_zone(d, c + off)) return true;
    }
    return false;
}

__device__ void repair_zone(const RepairStencil &o, long ks, double *pv, int *pflag, int *failimage, long c) {
    bool pf[11];
#pragma unroll
    for (int q = 1; q <= 10; q++) pf[q] = !pflag[c + stencil_offset(o, q)];
    const long si = o.si, sj = o.sj;
#define P(off) pv[k * ks + c + (off)]
    if (pf[2] && pf[4] && pf[6] && pf[8] && pf[9] && pf[10]) {
        for (int k = 0; k < B1; k++) P(0) = 1. / 6. * (P(sj) + P(-sj) + P(-si) + P(si) + P(1) + P(-1));
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
        // no usable stencil: density and energy from both four-point
        // averages, velocity zero
        failimage[4 * ks + c]++;
        for (int k = RHO; k <= UU; k++)
            P(0) = 0.5 * (0.25 * (P(sj) + P(-sj) + P(-si) + P(si))
                          + 0.25 * (P(si + sj) + P(si - sj) + P(-si + sj) + P(-si - sj)));
        pv[U1 * ks + c] = 0.;
        pv[U2 * ks + c] = 0.;
        pv[U3 * ks + c] = 0.;
    }
#undef P
    pflag[c] = 0;
}

// (one thread per cell of the ghosted block: the flag test is one coalesced
// load, and only a failed zone pays for its (i, j, z))
__global__ void k_repair_scan(const Dims d, double *__restrict__ pv, int *__restrict__ pflag,
                              int *__restrict__ failimage, int *__restrict__ list, int *__restrict__ count) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long)d.G1 * d.G2 * d.G3) return;
    if (pflag[c] == 0 || !active_zone(d, c)) return;
    const RepairStencil o{(long)d.G2 * d.G3, d.G3, d.d3};
    if (failed_neighbour(d, o, pflag, c, false))
        list[atomicAdd(count, 1)] = (int)c;
    else
        repair_zone(o, d.ks, pv, pflag, failimage, c);
}

constexpr int REPAIR_THREADS = 1024;
__global__ void __launch_bounds__(REPAIR_THREADS) k_repair_chain(const Dims d, double *__restrict__ pv,
                                                                 int *__restrict__ pflag, int *__restrict__ failimage,
                                                                 int *__restrict__ list, int *__restrict__ count) {
    const int n = *count;
    const RepairStencil o{(long)d.G2 * d.G3, d.G3, d.d3};
    // entries: c >= 1 pending, ~c (<= -2) ready in this wave, -1 repaired
    for (int wave = 0; wave <= n; wave++) {
        int pending = 0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int e = list[k];
            if (e < 0) continue;
            pending = 1;
            if (!failed_neighbour(d, o, pflag, e, true)) list[k] = ~e;
        }
        if (!__syncthreads_or(pending)) break;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int e = list[k];
            if (e <= -2) {
                repair_zone(o, d.ks, pv, pflag, failimage, ~e);
                list[k] = -1;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = 0;
}

// ------------------------------------------------------------ ghost fills
// no-inflow check on a ghost zone (inflow_check, GPU_bounds.h:1368-1410)
__device__ void inflow_check(double *pr, const Geo<double> &gm, int type) {
    double ucon[4], gamma;
    ucon_calc(pr, gm, ucon);
    if (((ucon[1] > 0.) && (type == 0)) || ((ucon[1] < 0.) && (type == 1))) {
        gamma_calc(pr, gm, &gamma);
        pr[U1] /= gamma;
        pr[U2] /= gamma;
        pr[U3] /= gamma;
        const double alpha = 1. / sqrt(-gm.gcon[0]);
        const double beta1 = gm.gcon[1] * alpha * alpha;
        pr[U1] = beta1 / alpha;
        double vsq = gm.gcov[4] * pr[U1] * pr[U1];
        vsq += 2. * gm.gcov[5] * pr[U2] * pr[U1];
        vsq += 2. * gm.gcov[6] * pr[U3] * pr[U1];
        vsq += gm.gcov[7] * pr[U2] * pr[U2];
        vsq += 2 * gm.gcov[8] * pr[U3] * pr[U2];
        vsq += gm.gcov[9] * pr[U3] * pr[U3];
        vsq = d_max(1.e-13, vsq);
        if (vsq >= 1.) vsq = 1. - 1. / (80. * 80.);
        gamma = 1. / sqrt(1. - vsq);
        pr[U1] *= gamma;
        pr[U2] *= gamma;
        pr[U3] *= gamma;
    }
}

__device__ __forceinline__ void copy_cell(const Dims &d, double *pv, long dst, long src) {
#pragma unroll
    for (int k = 0; k < NPR; k++) pv[k * d.ks + dst] = pv[k * d.ks + src];
}

// x1 ghosts over every (j, z): periodic copy, or outflow copy + no-inflow
__device__ __forceinline__ void k_bound_x1_at(const Dims &d, const Geom &m, double *pv, double *ps, const long t) {
    const int z = (int)(t % d.G3), j = (int)((t / d.G3) % d.G2), g = (int)(t / ((long)d.G3 * d.G2));
    const int ilo = g, ihi = d.n1 + d.ng1 + g;
    const long ks = d.ks;
    if (d.bc1 == HAMR_BC_PERIODIC) {
        copy_cell(d, pv, cix(d, ilo, j, z), cix(d, ilo + d.n1, j, z));
        copy_cell(d, pv, cix(d, ihi, j, z), cix(d, ihi - d.n1, j, z));
        for (int k = 0; k < 3; k++) {
            ps[k * ks + cix(d, ilo, j, z)] = ps[k * ks + cix(d, ilo + d.n1, j, z)];
            ps[k * ks + cix(d, ihi, j, z)] = ps[k * ks + cix(d, ihi - d.n1, j, z)];
        }
        return;
    }
    double pr[NPR];
    Geo<double> gm;
    long src, dst;
    if (!(d.halo & 1)) {   // a side shared with a neighbouring block is filled by the exchange
        src = cix(d, d.ng1, j, z);
        dst = cix(d, ilo, j, z);
        for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + src];
        load_geo(d, m, ilo, j, CENT, gm);
        inflow_check(pr, gm, 0);
        for (int k = 0; k < NPR; k++) pv[k * ks + dst] = pr[k];
        ps[1 * ks + dst] = ps[1 * ks + src];
        ps[2 * ks + dst] = ps[2 * ks + src];
    }
    if (!(d.halo & 2)) {
        src = cix(d, d.n1 + d.ng1 - 1, j, z);
        dst = cix(d, ihi, j, z);
        for (int k = 0; k < NPR; k++) pr[k] = pv[k * ks + src];
        load_geo(d, m, ihi, j, CENT, gm);
        inflow_check(pr, gm, 1);
        for (int k = 0; k < NPR; k++) pv[k * ks + dst] = pr[k];
        ps[1 * ks + dst] = ps[1 * ks + src];
        ps[2 * ks + dst] = ps[2 * ks + src];
    }
}

__global__ void k_bound_x1(const Dims d, const Geom m, double *pv, double *ps) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)d.ng1 * d.G2 * d.G3) return;
    k_bound_x1_at(d, m, pv, ps, t);
}

// x3 ghosts (periodic) over every (i, j): one item per (component, i, j,
// ghost layer), the components being the NPR primitives and then the 3
// face-field planes, so that each thread copies one value to each end of a
// row (one item per (i, j, layer) copying all 12 left the launch at a fifth
// of a wave, bound by the latency of its 24 dependent copies)
constexpr int X3_COMPS = NPR + 3;
__host__ __device__ __forceinline__ long n_bound_x3(const Dims &d) { return (long)X3_COMPS * d.ng3 * d.G1 * d.G2; }

__device__ __forceinline__ void k_bound_x3_at(const Dims &d, double *pv, double *ps, const long t) {
    const int g = (int)(t % d.ng3);
    const long r = t / d.ng3;
    const int j = (int)(r % d.G2), i = (int)((r / d.G2) % d.G1), comp = (int)(r / ((long)d.G2 * d.G1));
    double *a = comp < NPR ? pv + (long)comp * d.ks : ps + (long)(comp - NPR) * d.ks;
    a[cix(d, i, j, g)] = a[cix(d, i, j, g + d.n3)];
    a[cix(d, i, j, d.n3 + d.ng3 + g)] = a[cix(d, i, j, d.ng3 + g)];
}

__global__ void k_bound_x3(const Dims d, double *pv, double *ps) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_bound_x3(d)) return;
    k_bound_x3_at(d, pv, ps, t);
}

// x2 ghosts: periodic, transmissive or reflective polar axis, or plain
// outflow copy. One item per (component, i, z), components being the NPR
// primitives and then the 3 face-field planes: every rule acts on one
// component at a time, so the items are independent, and the two poles of a
// column are filled in order by the same item (with very few rows the
// reflective-axis rows of one pole feed the other's).
constexpr int X2_COMPS = NPR + 3;
__host__ __device__ __forceinline__ long n_bound_x2(const Dims &d) { return (long)X2_COMPS * d.G1 * d.G3; }

__device__ __forceinline__ void k_bound_x2_at(const Dims &d, double *pv, double *ps, const long t) {
    const int z = (int)(t % d.G3), i = (int)((t / d.G3) % d.G1), comp = (int)(t / ((long)d.G3 * d.G1));
    const int n2 = d.n2, ng = d.ng2;
    const bool face = comp >= NPR;
    const int k = face ? comp - NPR : comp;
    double *a = (face ? ps : pv) + (long)k * d.ks;
    auto C = [&](int j, int zz) { return cix(d, i, j, zz); };
    if (d.bc2 == HAMR_BC_PERIODIC) {
        for (int g = 0; g < ng; g++) {
            a[C(g, z)] = a[C(g + n2, z)];
            a[C(n2 + ng + g, z)] = a[C(ng + g, z)];
        }
    } else if (d.bc2 == HAMR_BC_POLE_TRANS) {
        if (face && k == 1) return;
        const int zs = d.d3 ? (z - d.ng3 + d.n3 / 2) % d.n3 + d.ng3 : z;
        const double sg = face ? (k == 2 ? -1. : 1.) : ((k == U2 || k == U3 || k == B2 || k == B3) ? -1. : 1.);
        if (d.pole1)
            for (int jj = -ng; jj < 0; jj++) a[C(jj + ng, z)] = sg * a[C(-jj - 1 + ng, zs)];
        if (d.pole2)
            for (int jj = n2; jj < n2 + ng; jj++) a[C(jj + ng, z)] = sg * a[C(2 * n2 - jj - 1 + ng, zs)];
    } else if (d.bc2 == HAMR_BC_POLE_REFL) {
        if (face && k == 1) return;
        const int jref = 2;  // POLEFIX, config.h:490
        const bool fixrow = !face && (k == RHO || k == UU || k == U1 || k == U3 || k == KTOT);
        const bool fixu2 = !face && k == U2;
        const double sg = (!face && (k == U2 || k == B2)) ? -1. : 1.;
        if (d.pole1) {
            const double vr = a[C(jref + ng, z)];
            for (int jj = 0; jj < jref; jj++) {
                if (fixu2) a[C(jj + ng, z)] = (jj + 0.5) / (jref + 0.5) * vr;
                else if (fixrow) a[C(jj + ng, z)] = vr;
            }
            for (int g = 1; g <= ng; g++) a[C(ng - g, z)] = sg * a[C(ng + g - 1, z)];
        }
        if (d.pole2) {
            const double vr = a[C(n2 + ng - 1 - jref, z)];
            for (int jj = 0; jj < jref; jj++) {
                if (fixu2) a[C(n2 + ng - 1 - jj, z)] = (jj + 0.5) / (jref + 0.5) * vr;
                else if (fixrow) a[C(n2 + ng - 1 - jj, z)] = vr;
            }
            for (int g = 0; g < ng; g++) a[C(n2 + ng + g, z)] = sg * a[C(n2 + ng - 1 - g, z)];
        }
    } else {
        if (face && k == 1) return;
        for (int g = 0; g < ng; g++) {
            if (!(d.halo & 4)) a[C(g, z)] = a[C(ng, z)];
            if (!(d.halo & 8)) a[C(n2 + ng + g, z)] = a[C(n2 + ng - 1, z)];
        }
    }
}

__global__ void k_bound_x2(const Dims d, double *pv, double *ps) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_bound_x2(d)) return;
    k_bound_x2_at(d, pv, ps, t);
}

// ------------------------------------------------------------ halos
// A block of a domain decomposed along x1 (or x2) exchanges ng layers with
// each neighbour: the layers next to a shared side (its last ng active layers
// on the upper side, its first ng on the lower) become the neighbour's ghost
// layers on the facing side, over the whole ghost-inclusive cross section
// ((x2, x3) for an x1 side, (x1, x3) for an x2 side), for the NPR primitives
// and the 3 face-field planes. Buffer layout [component][layer][j][z] for x1
// sides (side 0, 1), [component][layer][i][z] for x2 sides (side 2, 3) (the
// boundprim slabs of boundcomP.c, one contiguous message per side).
constexpr int HALO_COMPS = NPR + 3;
__host__ __device__ __forceinline__ long n_halo_side(const Dims &d, int side) {
    return side < 2 ? (long)HALO_COMPS * d.ng1 * d.G2 * d.G3 : (long)HALO_COMPS * d.ng2 * d.G1 * d.G3;
}
__host__ __device__ __forceinline__ long n_halo(const Dims &d) {
    const long a = n_halo_side(d, 0), b = n_halo_side(d, 2);
    return a > b ? a : b;
}

template <bool PACK>
__global__ void k_halo(const Dims d, double *pv, double *ps, int side, double *buf) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_halo_side(d, side)) return;
    const bool upper = side & 1;
    const int z = (int)(t % d.G3);
    int i, j, comp;
    if (side < 2) {
        j = (int)((t / d.G3) % d.G2);
        const long r = t / ((long)d.G3 * d.G2);
        const int g = (int)(r % d.ng1);
        comp = (int)(r / d.ng1);
        // packed: active layers next to the side; unpacked: the ghosts beyond it
        i = PACK ? (upper ? d.n1 + g : d.ng1 + g) : (upper ? d.ng1 + d.n1 + g : g);
    } else {
        i = (int)((t / d.G3) % d.G1);
        const long r = t / ((long)d.G3 * d.G1);
        const int g = (int)(r % d.ng2);
        comp = (int)(r / d.ng2);
        j = PACK ? (upper ? d.n2 + g : d.ng2 + g) : (upper ? d.ng2 + d.n2 + g : g);
    }
    double *a = comp < NPR ? pv + (long)comp * d.ks : ps + (long)(comp - NPR) * d.ks;
    const long c = cix(d, i, j, z);
    if (PACK) buf[t] = a[c];
    else a[c] = buf[t];
}

// --------------------------------------------------------- step size logic
constexpr unsigned long long BITS_1E9 = 0x41CDCD6500000000ULL;  // 1.0e9

__global__ void k_dt_reset(unsigned long long *dtbits) {
    if (threadIdx.x < 4) dtbits[threadIdx.x] = BITS_1E9;
}

// CFL step 1/(1/dt1 + 1/dt2 + 1/dt3) of the last full sub-step
// (step_ch.c:1320-1331). In advance mode (dt_state != NULL) the device step
// size follows min(ndt, 1.3 dt) every `interval` steps (step_ch.c:973-975).
__global__ void k_dt_finalize(unsigned long long *dtbits, double *ndt_out, double *dt_state, int *counter, int interval) {
    if (threadIdx.x != 0) return;
    const double d1 = __longlong_as_double((long long)dtbits[1]);
    const double d2 = __longlong_as_double((long long)dtbits[2]);
    const double d3 = __longlong_as_double((long long)dtbits[3]);
    const double ndt = 1. / (1. / d1 + 1. / d2 + 1. / d3);
    *ndt_out = ndt;
    if (dt_state) {
        const int n = ++(*counter);
        if (interval <= 1 || n % interval == 0) {
            double dt = *dt_state;
            *dt_state = ndt > 1.3 * dt ? 1.3 * dt : ndt;
        }
    }
    dtbits[0] = dtbits[1] = dtbits[2] = dtbits[3] = BITS_1E9;
}

// |div B| max over active zones (divb_calc, diag.c:153-199)
__global__ void k_divb(const Dims d, const Geom m, const double *ps, unsigned long long *out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.;
    if (t < (long)d.n1 * d.n2 * d.n3) {
        const int z = d.ng3 + (int)(t % d.n3);
        const int j = d.ng2 + (int)((t / d.n3) % d.n2);
        const int i = d.ng1 + (int)(t / ((long)d.n3 * d.n2));
        const long c = cix(d, i, j, z), ks = d.ks;
        double divb = 0.;
        if (d.d1) divb += 0.25 * (ps[0 * ks + c + (long)d.G2 * d.G3] * m.gdet[FACE1 * d.gs + gix(d, i + 1, j)] - ps[0 * ks + c] * m.gdet[FACE1 * d.gs + gix(d, i, j)]) / d.dx1;
        if (d.d2) divb += 0.25 * (ps[1 * ks + c + d.G3] * m.gdet[FACE2 * d.gs + gix(d, i, j + 1)] - ps[1 * ks + c] * m.gdet[FACE2 * d.gs + gix(d, i, j)]) / d.dx2;
        if (d.d3) divb += 0.25 * (ps[2 * ks + c + 1] * m.gdet[FACE3 * d.gs + gix(d, i, j)] - ps[2 * ks + c] * m.gdet[FACE3 * d.gs + gix(d, i, j)]) / d.dx3;
        v = fabs(divb);
    }
    for (int o = 16; o > 0; o >>= 1) v = d_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

inline unsigned nblk(long n) { return (unsigned)((n + BLK - 1) / BLK); }

}  // namespace

// ===========================================================================
// The CFL bookkeeping constants of a block (Dims::cfl_c0, ctop_lim): c0 =
// cour dx per direction, as the device computes it, and the largest double
// x with c0 / x > 1e-6, found from c0 / 1e-6 by stepping one ulp at a time
// (IEEE division on the host, as on the device).
static void set_cfl_limits(Dims &d) {
    const double dx[4] = {0., d.dx1, d.dx2, d.dx3};
    d.cfl_c0[0] = 0.;
    d.ctop_lim[0] = -1.;
    for (int k = 1; k < 4; k++) {
        const double c0 = d.cour * dx[k];
        d.cfl_c0[k] = c0;
        double x = c0 / 1.e-6;
        if (!(c0 > 0.) || !std::isfinite(x) || !(x > 0.)) {
            d.ctop_lim[k] = -1.;   // no face counts
            continue;
        }
        for (int it = 0; it < 64 && !(c0 / x > 1.e-6); it++) x = std::nextafter(x, 0.);
        for (int it = 0; it < 64 && c0 / std::nextafter(x, INFINITY) > 1.e-6; it++) x = std::nextafter(x, INFINITY);
        d.ctop_lim[k] = x;
    }
}

struct hamr_ctx {
    hamr_params prm;
    Dims d;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool have_geom = false;
    long rows_min = 0;   // threads the row flux kernels need before they pay (several waves of the device)
    bool cons_cols = true;   // column-staged conserved update where n3 >= 64
    bool ct_fused = false;   // one constrained-transport kernel for 3-D blocks (slower: off)
    bool cons_tma = true;    // conserved update with TMA-staged fluxes (3-D, n3 >= 32, aligned planes)
    int *kerr = nullptr;     // set by kernels whose bounded waits gave up
    // independent kernels of a sub-step on two side streams, forked from and
    // joined back into `stream` by events (the x1/x2 fluxes and the centre
    // EMFs beside the x3 fluxes; the rest of the CT chain beside the conserved
    // update); off for the per-kernel profile and the allocation-free step.
    // Measured on the 384 x 192 x 192 torus: 14.44 ms per mixed step with the
    // side streams, 14.35 without (FP64 31.40, 31.32): off by default,
    // HAMR_CONCURRENT=1 turns it on
    bool concurrent = false;
    // 3-D blocks: the centre EMFs computed by the x3 flux kernel instead of
    // k_emf_centre (HAMR_EMF_IN_X3=0 keeps the separate kernel)
    bool emf_in_x3 = true;
    // the primary inversion inside the TMA-staged update kernel (no floors or
    // repair; HAMR_FUSE_INV=0 keeps the separate inversion kernel)
    bool fuse_inv = true;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev[5] = {};
    std::string err;
    // device state
    double *p = nullptr, *ph = nullptr, *ps = nullptr, *psh = nullptr, *U = nullptr;
    double *F1 = nullptr, *F2 = nullptr, *F3 = nullptr, *Ec = nullptr, *emf = nullptr;
    double *W = nullptr;  // updated conserved variables between k_cons and k_invert
    int *pflag = nullptr, *failimage = nullptr;
    double *gcov = nullptr, *gcon = nullptr, *gdet = nullptr, *conn = nullptr;
    double *itab = nullptr;   // the column table of reciprocals (k_inv_tab), 16 planes of gs
    unsigned long long *dtbits = nullptr;
    double *ndt = nullptr, *dt_state = nullptr;
    int *counter = nullptr;
    unsigned long long *divb = nullptr;
    int *rlist = nullptr, *rcount = nullptr;   // neighbour repair: listed zones and their count
    int *flist = nullptr, *nfail = nullptr;    // zones the primary inversion failed, and their count
    // captured advance graphs
    cudaGraphExec_t graph = nullptr;
    int graph_steps = -1, graph_interval = -1;
};

namespace {

int fail_cuda(hamr_ctx *c, cudaError_t e, const char *what) {
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return HAMR_E_CUDA;
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return fail_cuda(ctx, e_, #call); \
    } while (0)

Geom geom_of(const hamr_ctx *c) { return Geom{c->gcov, c->gcon, c->gdet, c->conn, c->itab}; }

// the error word kernels set when a bounded wait gave up (read after a
// synchronisation the caller already makes; cleared once reported)
int check_kerr(hamr_ctx *ctx) {
    if (!ctx->kerr) return HAMR_OK;
    int v = 0;
    CK(cudaMemcpyAsync(&v, ctx->kerr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!v) return HAMR_OK;
    CK(cudaMemsetAsync(ctx->kerr, 0, sizeof(int), ctx->stream));
    ctx->err = "a kernel's wait for its bulk copies timed out (the step's results are invalid)";
    return HAMR_E_CUDA;
}

// kernel groups timed by hamr_profile_step
enum { PROF_FLUX3, PROF_FLUX2, PROF_FLUX1, PROF_FIXFLUX, PROF_EMF_CENTRE, PROF_EMF_EDGE, PROF_POLE_AVG,
       PROF_FACE, PROF_UPDATE, PROF_INVERT, PROF_BOUND, PROF_NSLOT };

struct Prof {
    cudaEvent_t ev[PROF_NSLOT + 1];
    bool on = false;
};

inline void prof_mark(Prof *pf, int slot, cudaStream_t s) {
    if (pf && pf->on) cudaEventRecord(pf->ev[slot + 1], s);
}

// ghost fill of the state written by a sub-step (full: p, ps; else ph, psh)
// in direction dim (1, 2, 3), on the block's physical sides; dim 0: all
// three, in the order x1, x3, x2
int launch_bound_dim(hamr_ctx *ctx, int full, int dim) {
    const Dims &d = ctx->d;
    cudaStream_t s = ctx->stream;
    double *pw = full ? ctx->p : ctx->ph;
    double *psw = full ? ctx->ps : ctx->psh;
    if ((dim == 0 || dim == 1) && d.d1)
        k_bound_x1<<<nblk((long)d.ng1 * d.G2 * d.G3), BLK, 0, s>>>(d, geom_of(ctx), pw, psw);
    if ((dim == 0 || dim == 3) && d.d3) k_bound_x3<<<nblk(n_bound_x3(d)), BLK, 0, s>>>(d, pw, psw);
    if ((dim == 0 || dim == 2) && d.d2) k_bound_x2<<<nblk(n_bound_x2(d)), BLK, 0, s>>>(d, pw, psw);
    CK(cudaGetLastError());
    return HAMR_OK;
}

// n faces of direction DIR, one thread per face, with the block's reconstruction
// flux kernel variant: bit 0 MC reconstruction, bit 1 the face-frame
// Riemann solvers (HLLC), bit 2 HLLD there
inline int rec_key(const Dims &d) {
    return d.recon | (d.riemann != HAMR_RIEMANN_HLL ? 2 : 0) | (d.riemann == HAMR_RIEMANN_HLLD ? 4 : 0);
}

template <int DIR, typename T>
void launch_flux(long n, cudaStream_t s, const Dims &d, const Geom &m, const double *pin, const double *psin, T *F,
                 unsigned long long *dtbits, int cd, long rows_min, T *Ec = nullptr) {
    // x1 and x2 faces by rows, each zone reconstructed once, where the rows
    // still fill the device several times over; small blocks (2-D, ensemble
    // members) keep one thread per face
    if (DIR == 3) {   // each zone reconstructed once, edges through shared memory
        const long nb = n_x3_slot_ctas(d);
        switch (rec_key(d)) {
        case 1: k_flux_x3<T, 1><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        case 2: k_flux_x3<T, 2><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        case 3: k_flux_x3<T, 3><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        case 6: k_flux_x3<T, 6><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        case 7: k_flux_x3<T, 7><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        default: k_flux_x3<T, 0><<<nb, BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd, Ec); break;
        }
        return;
    }
    if (n_flux_rows<DIR == 3 ? 1 : DIR>(d) >= rows_min) {
        constexpr int RD = DIR == 3 ? 1 : DIR;
        const long nr = n_flux_rows<RD>(d);
        switch (rec_key(d)) {
        case 1: k_flux_rows<RD, T, 1><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        case 2: k_flux_rows<RD, T, 2><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        case 3: k_flux_rows<RD, T, 3><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        case 6: k_flux_rows<RD, T, 6><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        case 7: k_flux_rows<RD, T, 7><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        default: k_flux_rows<RD, T, 0><<<nblk(nr), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
        }
        return;
    }
    switch (rec_key(d)) {
    case 1: k_flux<DIR, T, 1><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    case 2: k_flux<DIR, T, 2><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    case 3: k_flux<DIR, T, 3><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    case 6: k_flux<DIR, T, 6><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    case 7: k_flux<DIR, T, 7><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    default: k_flux<DIR, T, 0><<<nblk(n), BLK, 0, s>>>(d, m, pin, psin, F, dtbits, cd); break;
    }
}

// the bulk copies of k_cons_tma need 16-byte aligned flux planes
template <typename T>
bool cons_tma_aligned(const hamr_ctx *ctx, const Dims &d, const T *F1, const T *F2, const T *F3) {
    auto al = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
    return ctx->kerr && (d.ks * (long)sizeof(T)) % 16 == 0 && al(F1) && al(F2) && al(F3);
}

// one sub-step: fluxes, CT, update, ghost fill of the written state. T is the
// type of the fluxes and EMFs (double, or float in the mixed-precision step);
// the float arrays reuse the double allocations with the same plane stride.
template <typename T>
int launch_stage_t(hamr_ctx *ctx, int full, StepSize st, bool calc_dt, Prof *pf) {
    const Dims &d = ctx->d;
    T *F1 = reinterpret_cast<T *>(ctx->F1), *F2 = reinterpret_cast<T *>(ctx->F2);
    T *F3 = reinterpret_cast<T *>(ctx->F3), *Ec = reinterpret_cast<T *>(ctx->Ec);
    T *emf = reinterpret_cast<T *>(ctx->emf);
    const Geom m = geom_of(ctx);
    cudaStream_t s = ctx->stream;
    const double *pin = full ? ctx->ph : ctx->p;
    const double *psin = full ? ctx->psh : ctx->ps;
    const int cd = calc_dt ? 1 : 0;
    // the fluxes of the three directions (each with its own step-size slot)
    // and the centre EMFs read only the sub-step's input state: x3 on the
    // stage stream, x2 and x1 + centre EMFs on the side streams
    const bool conc = ctx->concurrent && !(pf && pf->on) && !(d.d3 && ctx->ct_fused);
    cudaStream_t s2 = conc ? ctx->side[0] : s, s3 = conc ? ctx->side[1] : s;
    // 3-D: the centre EMFs come out of the x3 flux kernel
    const bool ec_x3 = d.d3 && !ctx->ct_fused && ctx->emf_in_x3;
    if (conc) {
        CK(cudaEventRecord(ctx->ev[0], s));
        CK(cudaStreamWaitEvent(s2, ctx->ev[0], 0));
        CK(cudaStreamWaitEvent(s3, ctx->ev[0], 0));
    }
    if (d.d3) {
        long n = (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3 - 1);
        launch_flux<3, T>(n, s, d, m, pin, psin, F3, ctx->dtbits, cd, ctx->rows_min, ec_x3 ? Ec : nullptr);
    }
    prof_mark(pf, PROF_FLUX3, s);
    {
        long n = (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2 - 1) * (d.n3 + 2 * d.d3);
        launch_flux<2, T>(n, s2, d, m, pin, psin, F2, ctx->dtbits, cd, ctx->rows_min);
    }
    prof_mark(pf, PROF_FLUX2, s);
    {
        long n = (long)(d.n1 + 2 * d.d1 - 1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3);
        launch_flux<1, T>(n, s3, d, m, pin, psin, F1, ctx->dtbits, cd, ctx->rows_min);
    }
    prof_mark(pf, PROF_FLUX1, s);
    if (conc) {
        long n = (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3);
        if (!ec_x3) k_emf_centre<T><<<nblk(n), BLK, 0, s3>>>(d, m, pin, Ec);
        CK(cudaEventRecord(ctx->ev[1], s2));
        CK(cudaEventRecord(ctx->ev[2], s3));
        CK(cudaStreamWaitEvent(s, ctx->ev[1], 0));
        CK(cudaStreamWaitEvent(s, ctx->ev[2], 0));
    }
    if (d.bc2 == HAMR_BC_POLE_REFL) {
        long n = (long)d.G1 * d.G3 + (long)d.G2 * d.G3;
        k_fix_flux<T><<<nblk(n), BLK, 0, s>>>(d, F1, F2, F3);
    }
    prof_mark(pf, PROF_FIXFLUX, s);
    // the rest of the CT chain (edge EMFs, polar average, face update) writes
    // only EMFs and the face field, which the conserved update does not read:
    // on a side stream beside it, joined before the inversion
    if (conc) {
        CK(cudaEventRecord(ctx->ev[3], s));
        CK(cudaStreamWaitEvent(s2, ctx->ev[3], 0));
    }
    if (d.d3 && ctx->ct_fused) {
        // centre EMFs, edge EMFs and the face update in one kernel (polar
        // rows of transmissive poles after the phi average); timed as the
        // edge-EMF group
        prof_mark(pf, PROF_EMF_CENTRE, s);
        const dim3 grid((d.n3 + CT_TZ) / CT_TZ, (d.n2 + CT_TJ) / CT_TJ, (d.n1 + HAMR_CT_CHUNK) / HAMR_CT_CHUNK);
        k_ct_fused<T><<<grid, CT_THREADS, 0, s>>>(d, m, pin, F1, F2, F3, ctx->ps, full ? ctx->ps : ctx->psh, emf, st);
        prof_mark(pf, PROF_EMF_EDGE, s);
        if (d.bc2 == HAMR_BC_POLE_TRANS) {
            k_pole_average<T><<<nblk(64L * (d.n1 + d.ng1)), BLK, 0, s>>>(d, emf, st);   // a warp per row
            prof_mark(pf, PROF_POLE_AVG, s);
            k_face_update_polar<T><<<nblk(3L * (d.n1 + 1) * (d.n3 + 1)), BLK, 0, s>>>(
                d, m, ctx->ps, full ? ctx->ps : ctx->psh, emf, st);
        } else {
            prof_mark(pf, PROF_POLE_AVG, s);
        }
        prof_mark(pf, PROF_FACE, s);
    } else {
    if (!conc && !ec_x3) {
        long n = (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3);
        k_emf_centre<T><<<nblk(n), BLK, 0, s>>>(d, m, pin, Ec);
    }
    prof_mark(pf, PROF_EMF_CENTRE, s);
    {
        k_emf_edge<T><<<nblk((long)(d.n1 + d.d1) * (d.n2 + d.d2) * (d.n3 + d.d3)), BLK, 0, s2>>>(d, Ec, F1, F2, F3,
                                                                                          emf);
        prof_mark(pf, PROF_EMF_EDGE, s);
        if (d.bc2 == HAMR_BC_POLE_TRANS)
            k_pole_average<T><<<nblk(64L * (d.n1 + d.ng1)), BLK, 0, s2>>>(d, emf, st);   // a warp per row
        prof_mark(pf, PROF_POLE_AVG, s);
        k_face_update<T><<<nblk(n_face_threads(d)), BLK, 0, s2>>>(d, m, ctx->ps, full ? ctx->ps : ctx->psh, emf, st);
        prof_mark(pf, PROF_FACE, s);
    }
    }
    {
        long n = (long)d.n1 * d.n2 * d.n3;
        const bool tma = ctx->cons_tma && d.d3 && d.n3 >= 32 && cons_tma_aligned<T>(ctx, d, F1, F2, F3);
        const int fix = (ctx->prm.floors ? FIX_FLOORS : 0) | (ctx->prm.repair == 1 ? FIX_RESET : 0);
        double *pout = full ? ctx->p : ctx->ph;
        const double *pg = full ? ctx->ph : ctx->p;
        const double *psf = full ? ctx->ps : ctx->psh;
        const int nm = d.inversion == HAMR_INV_NM;
        // the primary inversion inside the update kernel (the face update, which
        // it reads, has run in this stream)
        const bool fuse = tma && ctx->fuse_inv && fix == 0 && ctx->prm.repair != 2 && !conc;
        if (tma) {   // one row of zones per CTA, flux operands staged by bulk copies
            const int npiece = (d.n3 + 255) / 256, lpiece = (d.n3 + npiece - 1) / npiece;
            const dim3 grid(d.n1 * d.n2 * npiece), block((lpiece + 31) / 32 * 32);
            const size_t sm = cons_tma_layout<T>(lpiece).total;
            if (fuse) {
                CK(cudaMemsetAsync(ctx->nfail, 0, sizeof(int), s));
                auto kf = nm ? k_cons_tma<T, HAMR_INV_NM + 1> : k_cons_tma<T, HAMR_INV_2D + 1>;
                kf<<<grid, block, sm, s>>>(d, m, ctx->p, pg, ctx->U, F1, F2, F3, ctx->W, full, st, ctx->nfail,
                                           ctx->kerr, npiece, lpiece, psf, pout, ctx->pflag, ctx->failimage,
                                           ctx->flist);
            } else {
                k_cons_tma<T><<<grid, block, sm, s>>>(d, m, ctx->p, pg, ctx->U, F1, F2, F3, ctx->W, full, st,
                                                      ctx->nfail, ctx->kerr, npiece, lpiece);
            }
        } else if (d.n3 >= 64 && ctx->cons_cols)   // metric and connection staged per CTA
            k_cons_cols<T><<<nblk(n), BLK, 0, s>>>(d, m, ctx->p, full ? ctx->ph : ctx->p, ctx->U, F1, F2, F3, ctx->W,
                                                   full, st, ctx->nfail);
        else
            k_cons<T><<<nblk(n), BLK, 0, s>>>(d, m, ctx->p, full ? ctx->ph : ctx->p, ctx->U, F1, F2, F3, ctx->W, full,
                                              st, ctx->nfail);
        prof_mark(pf, PROF_UPDATE, s);
        if (conc) {
            CK(cudaEventRecord(ctx->ev[4], s2));
            CK(cudaStreamWaitEvent(s, ctx->ev[4], 0));
        }
        // primary solver over every zone, then the fallback chain over the
        // zones it failed (usually none: the second launch reads the count
        // and returns)
        using InvP = void (*)(const Dims, const Geom, const double *, const double *, const double *, double *,
                              int *, int *, int *, int *);
        using InvF = void (*)(const Dims, const Geom, const double *, const double *, const double *, double *,
                              int *, int *, const int *, const int *);
        static const InvP inv_p[2][4] = {
            {k_invert_primary<HAMR_INV_2D, 0>, k_invert_primary<HAMR_INV_2D, 1>, k_invert_primary<HAMR_INV_2D, 2>,
             k_invert_primary<HAMR_INV_2D, 3>},
            {k_invert_primary<HAMR_INV_NM, 0>, k_invert_primary<HAMR_INV_NM, 1>, k_invert_primary<HAMR_INV_NM, 2>,
             k_invert_primary<HAMR_INV_NM, 3>}};
        static const InvF inv_f[2][4] = {
            {k_invert_fallback<HAMR_INV_2D, 0>, k_invert_fallback<HAMR_INV_2D, 1>, k_invert_fallback<HAMR_INV_2D, 2>,
             k_invert_fallback<HAMR_INV_2D, 3>},
            {k_invert_fallback<HAMR_INV_NM, 0>, k_invert_fallback<HAMR_INV_NM, 1>, k_invert_fallback<HAMR_INV_NM, 2>,
             k_invert_fallback<HAMR_INV_NM, 3>}};
        if (!fuse)
            inv_p[nm][fix]<<<nblk(n), BLK, 0, s>>>(d, m, pg, ctx->W, psf, pout, ctx->pflag, ctx->failimage,
                                                   ctx->flist, ctx->nfail);
        inv_f[nm][fix]<<<FALLBACK_CTAS, BLK, 0, s>>>(d, m, pg, ctx->W, psf, pout, ctx->pflag, ctx->failimage,
                                                     ctx->flist, ctx->nfail);
        if (ctx->prm.repair == 2) {
            k_repair_scan<<<nblk((long)d.G1 * d.G2 * d.G3), BLK, 0, s>>>(d, pout, ctx->pflag, ctx->failimage,
                                                                         ctx->rlist, ctx->rcount);
            k_repair_chain<<<1, REPAIR_THREADS, 0, s>>>(d, pout, ctx->pflag, ctx->failimage, ctx->rlist,
                                                        ctx->rcount);
        }
    }
    prof_mark(pf, PROF_INVERT, s);
    // ghost fill of the written state; a block of a decomposed domain leaves
    // it to the caller (hamr_bound_dim around the halo exchange)
    if (!d.halo) launch_bound_dim(ctx, full, 0);
    prof_mark(pf, PROF_BOUND, s);
    CK(cudaGetLastError());
    return HAMR_OK;
}

int launch_stage(hamr_ctx *ctx, int full, StepSize st, bool calc_dt, Prof *pf = nullptr) {
    if (ctx->prm.precision == HAMR_MIXED) return launch_stage_t<float>(ctx, full, st, calc_dt, pf);
    return launch_stage_t<double>(ctx, full, st, calc_dt, pf);
}

int launch_step(hamr_ctx *ctx, StepSize half, StepSize full, double *dt_state, int interval) {
    int rc = launch_stage(ctx, 0, half, false);
    if (rc) return rc;
    rc = launch_stage(ctx, 1, full, true);
    if (rc) return rc;
    k_dt_finalize<<<1, 32, 0, ctx->stream>>>(ctx->dtbits, ctx->ndt, dt_state, ctx->counter, interval);
    CK(cudaGetLastError());
    return HAMR_OK;
}

}  // namespace

extern "C" {

int hamr_ctx_create(const hamr_params *prm, hamr_ctx **out) {
    if (!prm || !out) return HAMR_E_ARG;
    *out = nullptr;
    if (prm->n1 < 2 || prm->n2 < 2 || prm->n3 < 1) return HAMR_E_ARG;
    if (prm->recon != HAMR_RECON_PPM && prm->recon != HAMR_RECON_MC) return HAMR_E_ARG;
    if (prm->riemann != HAMR_RIEMANN_HLL && prm->riemann != HAMR_RIEMANN_HLLC && prm->riemann != HAMR_RIEMANN_HLLD)
        return HAMR_E_ARG;
    if (!(prm->ng == 3 || (prm->ng == 2 && prm->recon == HAMR_RECON_MC))) return HAMR_E_ARG;
    if (prm->precision != HAMR_FP64 && prm->precision != HAMR_MIXED) return HAMR_E_ARG;
    if ((prm->halo & ~15) || ((prm->halo & 3) && (prm->bc1 == HAMR_BC_PERIODIC || prm->n1 < prm->ng))) return HAMR_E_ARG;
    // an x2 side shared with a neighbour is no pole and no periodic wrap
    if ((prm->halo & 12) && (prm->bc2 == HAMR_BC_PERIODIC || prm->n2 < prm->ng || ((prm->halo & 4) && prm->pole1) ||
                             ((prm->halo & 8) && prm->pole2)))
        return HAMR_E_ARG;
    if ((prm->floors & ~1) || prm->repair < 0 || prm->repair > 2) return HAMR_E_ARG;
    // the neighbour repair's order spans the whole domain: not on a slab of one
    if (prm->repair == 2 && prm->halo) return HAMR_E_ARG;
    if (prm->inversion != HAMR_INV_2D && prm->inversion != HAMR_INV_NM) return HAMR_E_ARG;
    if (prm->n3 > 1 && prm->bc3 != HAMR_BC_PERIODIC) return HAMR_E_ARG;
    if (prm->bc2 == HAMR_BC_POLE_TRANS && (prm->n3 < 2 || prm->n3 % 2)) return HAMR_E_ARG;
    if (!(prm->gam > 1.0) || !(prm->cour > 0.0) || !(prm->dx1 > 0) || !(prm->dx2 > 0) || !(prm->dx3 > 0)) return HAMR_E_ARG;
    hamr_ctx *ctx = new hamr_ctx();
    ctx->prm = *prm;
    Dims &d = ctx->d;
    d.n1 = prm->n1; d.n2 = prm->n2; d.n3 = prm->n3;
    d.d1 = d.n1 > 1; d.d2 = d.n2 > 1; d.d3 = d.n3 > 1;
    d.ng1 = d.d1 ? prm->ng : 0; d.ng2 = d.d2 ? prm->ng : 0; d.ng3 = d.d3 ? prm->ng : 0;
    d.G1 = d.n1 + 2 * d.ng1; d.G2 = d.n2 + 2 * d.ng2; d.G3 = d.n3 + 2 * d.ng3;
    const long ncell = (long)d.G1 * d.G2 * d.G3, ngeo = (long)d.G1 * d.G2;
    d.ks = prm->ksize ? prm->ksize : ncell + (64 - ncell % 64);
    d.gs = prm->gsize ? prm->gsize : ngeo + (64 - ngeo % 64);
    if (d.ks < ncell || d.gs < ngeo) { delete ctx; return HAMR_E_ARG; }
    d.dx1 = prm->dx1; d.dx2 = prm->dx2; d.dx3 = prm->dx3;
    d.rdx1 = 1.0 / d.dx1; d.rdx2 = 1.0 / d.dx2; d.rdx3 = 1.0 / d.dx3;
    d.rgam = 1.0 / prm->gam;
    d.gam = prm->gam; d.cour = prm->cour;
    set_cfl_limits(d);   // after dx and cour
    d.pole1 = prm->pole1; d.pole2 = prm->pole2;
    d.bc1 = prm->bc1; d.bc2 = prm->bc2; d.bc3 = prm->bc3;
    d.ct_upwind = prm->ct_upwind;
    d.inversion = prm->inversion;
    d.recon = prm->recon;
    d.riemann = prm->riemann;
    d.halo = prm->halo;
    if (prm->stream) {
        ctx->stream = (cudaStream_t)prm->stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete ctx; return HAMR_E_CUDA; }
        ctx->own_stream = true;
    }
    {
        // six waves of the row kernels' residency (blocks of 128 per SM: the
        // FP64 and float register caps)
        int dev = 0, nsm = 148;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int per_sm = prm->precision == HAMR_MIXED ? HAMR_FLUX_ROWS_MINB_F : HAMR_FLUX_ROWS_MINB;
        ctx->rows_min = 6L * nsm * per_sm * BLK;
        // tuning override (threads; 0: always by rows), read once per context
        if (const char *e = getenv("HAMR_FLUX_ROWS_MIN")) ctx->rows_min = atol(e);
        if (const char *e = getenv("HAMR_CONS_COLS")) ctx->cons_cols = atoi(e) != 0;
        if (const char *e = getenv("HAMR_CT_FUSED")) ctx->ct_fused = atoi(e) != 0;
        if (const char *e = getenv("HAMR_CONS_TMA")) ctx->cons_tma = atoi(e) != 0;
        if (const char *e = getenv("HAMR_CONCURRENT")) ctx->concurrent = atoi(e) != 0;
        if (const char *e = getenv("HAMR_EMF_IN_X3")) ctx->emf_in_x3 = atoi(e) != 0;
        if (const char *e = getenv("HAMR_FUSE_INV")) ctx->fuse_inv = atoi(e) != 0;
    }
    if (ctx->concurrent) {
        for (auto &st : ctx->side)
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) ctx->concurrent = false;
        for (auto &ev : ctx->ev)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) ctx->concurrent = false;
    }
    const size_t cb = sizeof(double) * d.ks;
    struct A { void **p; size_t n; } allocs[] = {
        {(void **)&ctx->p, NPR * cb}, {(void **)&ctx->ph, NPR * cb}, {(void **)&ctx->ps, 3 * cb},
        {(void **)&ctx->psh, 3 * cb}, {(void **)&ctx->U, NPR * cb}, {(void **)&ctx->F1, NPR * cb},
        {(void **)&ctx->F2, NPR * cb}, {(void **)&ctx->F3, NPR * cb}, {(void **)&ctx->Ec, 4 * cb},
        {(void **)&ctx->emf, 4 * cb}, {(void **)&ctx->W, 7 * cb}, {(void **)&ctx->pflag, sizeof(int) * d.ks},
        {(void **)&ctx->failimage, 5 * sizeof(int) * d.ks},
        {(void **)&ctx->gcov, 50 * sizeof(double) * d.gs}, {(void **)&ctx->gcon, 50 * sizeof(double) * d.gs},
        {(void **)&ctx->gdet, 5 * sizeof(double) * d.gs}, {(void **)&ctx->conn, 40 * sizeof(double) * d.gs},
        {(void **)&ctx->itab, 16 * sizeof(double) * d.gs},
        {(void **)&ctx->dtbits, 4 * sizeof(unsigned long long)}, {(void **)&ctx->ndt, sizeof(double)},
        {(void **)&ctx->dt_state, sizeof(double)}, {(void **)&ctx->counter, sizeof(int)},
        {(void **)&ctx->divb, sizeof(unsigned long long)},
        {(void **)&ctx->rlist, prm->repair == 2 ? sizeof(int) * d.n1 * d.n2 * d.n3 : 0},
        {(void **)&ctx->rcount, prm->repair == 2 ? sizeof(int) : 0},
        {(void **)&ctx->flist, sizeof(int) * d.n1 * d.n2 * d.n3}, {(void **)&ctx->nfail, sizeof(int)},
        {(void **)&ctx->kerr, sizeof(int)}};
    if (prm->repair == 2 && d.ks > 0x7fffffffL) { hamr_ctx_destroy(ctx); return HAMR_E_ARG; }
    for (auto &a : allocs) {
        if (a.n == 0) continue;
        if (cudaMalloc(a.p, a.n) != cudaSuccess) {
            hamr_ctx_destroy(ctx);
            return HAMR_E_NOMEM;
        }
        cudaMemsetAsync(*a.p, 0, a.n, ctx->stream);
    }
    k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
    // the TMA-staged update's shared memory for rows of up to 256 zones
    cudaFuncSetAttribute(k_cons_tma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<double>(256).total);
    cudaFuncSetAttribute(k_cons_tma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<float>(256).total);
    cudaFuncSetAttribute(k_cons_tma<double, HAMR_INV_2D + 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<double>(256).total);
    cudaFuncSetAttribute(k_cons_tma<double, HAMR_INV_NM + 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<double>(256).total);
    cudaFuncSetAttribute(k_cons_tma<float, HAMR_INV_2D + 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<float>(256).total);
    cudaFuncSetAttribute(k_cons_tma<float, HAMR_INV_NM + 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         cons_tma_layout<float>(256).total);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        hamr_ctx_destroy(ctx);
        return HAMR_E_CUDA;
    }
    *out = ctx;
    return HAMR_OK;
}

int hamr_ctx_destroy(hamr_ctx *ctx) {
    if (!ctx) return HAMR_E_ARG;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
    void *bufs[] = {ctx->p, ctx->ph, ctx->ps, ctx->psh, ctx->U, ctx->F1, ctx->F2, ctx->F3, ctx->Ec, ctx->emf,
                    ctx->W, ctx->pflag, ctx->failimage, ctx->gcov, ctx->gcon, ctx->gdet, ctx->conn, ctx->itab,
                    ctx->dtbits,
                    ctx->ndt, ctx->dt_state, ctx->counter, ctx->divb, ctx->rlist, ctx->rcount,
                    ctx->flist, ctx->nfail, ctx->kerr};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (auto st : ctx->side)
        if (st) cudaStreamDestroy(st);
    for (auto ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return HAMR_OK;
}

const char *hamr_last_error(const hamr_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int hamr_strides(const hamr_ctx *ctx, long *ksize, long *gsize) {
    if (!ctx) return HAMR_E_ARG;
    if (ksize) *ksize = ctx->d.ks;
    if (gsize) *gsize = ctx->d.gs;
    return HAMR_OK;
}

int hamr_set_geometry(hamr_ctx *ctx, const double *gcov, const double *gcon, const double *gdet, const double *conn) {
    if (!ctx || !gcov || !gcon || !gdet || !conn) return HAMR_E_ARG;
    const size_t g = sizeof(double) * ctx->d.gs;
    CK(cudaMemcpyAsync(ctx->gcov, gcov, 50 * g, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->gcon, gcon, 50 * g, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->gdet, gdet, 5 * g, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->conn, conn, 40 * g, cudaMemcpyHostToDevice, ctx->stream));
    k_inv_tab<<<nblk(ctx->d.gs), BLK, 0, ctx->stream>>>(ctx->d, ctx->gcon, ctx->gdet, ctx->itab);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_geom = true;
    return HAMR_OK;
}

int hamr_upload(hamr_ctx *ctx, const double *p, const double *ps) {
    if (!ctx || !p || !ps) return HAMR_E_ARG;
    const size_t cb = sizeof(double) * ctx->d.ks;
    CK(cudaMemcpyAsync(ctx->p, p, NPR * cb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->ps, ps, 3 * cb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HAMR_OK;
}

int hamr_download(hamr_ctx *ctx, double *p, double *ps) {
    if (!ctx) return HAMR_E_ARG;
    const size_t cb = sizeof(double) * ctx->d.ks;
    if (p) CK(cudaMemcpyAsync(p, ctx->p, NPR * cb, cudaMemcpyDeviceToHost, ctx->stream));
    if (ps) CK(cudaMemcpyAsync(ps, ctx->ps, 3 * cb, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HAMR_OK;
}

int hamr_download_flags(hamr_ctx *ctx, int *pflag, int *failimage) {
    if (!ctx) return HAMR_E_ARG;
    const size_t ib = sizeof(int) * ctx->d.ks;
    if (pflag) CK(cudaMemcpyAsync(pflag, ctx->pflag, ib, cudaMemcpyDeviceToHost, ctx->stream));
    if (failimage) CK(cudaMemcpyAsync(failimage, ctx->failimage, 5 * ib, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HAMR_OK;
}

int hamr_bound(hamr_ctx *ctx) {
    if (!ctx) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    return launch_bound_dim(ctx, 1, 0);
}

int hamr_bound_dim(hamr_ctx *ctx, int full, int dim) {
    if (!ctx || dim < 1 || dim > 3) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    return launch_bound_dim(ctx, full ? 1 : 0, dim);
}

long hamr_halo_count(const hamr_ctx *ctx) {
    if (!ctx) return -1;
    return n_halo(ctx->d);
}

int hamr_halo_pack(hamr_ctx *ctx, int full, int side, double *buf) {
    if (!ctx || !buf || side < 0 || side > 3) return HAMR_E_ARG;
    const Dims &d = ctx->d;
    k_halo<true><<<nblk(n_halo_side(d, side)), BLK, 0, ctx->stream>>>(
        d, full ? ctx->p : ctx->ph, full ? ctx->ps : ctx->psh, side, buf);
    CK(cudaGetLastError());
    return HAMR_OK;
}

int hamr_halo_unpack(hamr_ctx *ctx, int full, int side, const double *buf) {
    if (!ctx || !buf || side < 0 || side > 3) return HAMR_E_ARG;
    const Dims &d = ctx->d;
    k_halo<false><<<nblk(n_halo_side(d, side)), BLK, 0, ctx->stream>>>(
        d, full ? ctx->p : ctx->ph, full ? ctx->ps : ctx->psh, side, const_cast<double *>(buf));
    CK(cudaGetLastError());
    return HAMR_OK;
}

int hamr_cfl_dirs(hamr_ctx *ctx, double *dt3) {
    if (!ctx || !dt3) return HAMR_E_ARG;
    unsigned long long b[4];
    CK(cudaMemcpyAsync(b, ctx->dtbits, sizeof(b), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 3; k++) memcpy(&dt3[k], &b[k + 1], sizeof(double));
    return HAMR_OK;
}

int hamr_stage(hamr_ctx *ctx, int full, double Dt, double dt) {
    if (!ctx) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    if (!(Dt > 0) || !(dt > 0)) return HAMR_E_ARG;
    StepSize st{nullptr, 0., Dt, dt};
    if (full) k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
    return launch_stage(ctx, full ? 1 : 0, st, full != 0);
}

int hamr_step(hamr_ctx *ctx, double dt, double *dt_next) {
    if (!ctx) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    if (ctx->d.halo) {   // the halo exchange has to come between the sub-steps
        ctx->err = "a block with halo sides steps through hamr_stage, hamr_bound_dim and the halo exchange";
        return HAMR_E_STATE;
    }
    if (!(dt > 0)) return HAMR_E_ARG;
    k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
    int rc = launch_step(ctx, StepSize{nullptr, 0.5, 0.5 * dt, dt}, StepSize{nullptr, 1.0, dt, dt}, nullptr, 0);
    if (rc) return rc;
    if (dt_next) {
        CK(cudaMemcpyAsync(dt_next, ctx->ndt, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (int rc2 = check_kerr(ctx)) return rc2;
        if (!(*dt_next > 0) || !isfinite(*dt_next)) {
            ctx->err = "non-finite or non-positive CFL step";
            return HAMR_E_PHYSICS;
        }
    }
    return HAMR_OK;
}

int hamr_advance(hamr_ctx *ctx, int nsteps, int interval, double *dt_inout) {
    if (!ctx || !dt_inout || nsteps < 1 || interval < 1) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    if (ctx->d.halo) {   // the halo exchange has to come between the sub-steps
        ctx->err = "a block with halo sides steps through hamr_stage, hamr_bound_dim and the halo exchange";
        return HAMR_E_STATE;
    }
    if (!(*dt_inout > 0)) return HAMR_E_ARG;
    CK(cudaMemcpyAsync(ctx->dt_state, dt_inout, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->counter, 0, sizeof(int), ctx->stream));
    k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
    if (!ctx->graph || ctx->graph_steps != nsteps || ctx->graph_interval != interval) {
        if (ctx->graph) {
            cudaGraphExecDestroy(ctx->graph);
            ctx->graph = nullptr;
        }
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = HAMR_OK;
        for (int n = 0; n < nsteps && rc == HAMR_OK; n++)
            rc = launch_step(ctx, StepSize{ctx->dt_state, 0.5, 0., 0.}, StepSize{ctx->dt_state, 1.0, 0., 0.},
                             ctx->dt_state, interval);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail_cuda(ctx, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&ctx->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "cudaGraphInstantiate");
        ctx->graph_steps = nsteps;
        ctx->graph_interval = interval;
    }
    CK(cudaGraphLaunch(ctx->graph, ctx->stream));
    CK(cudaMemcpyAsync(dt_inout, ctx->dt_state, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_kerr(ctx);
}

int hamr_profile_step(hamr_ctx *ctx, double dt, int reps, double *ms, int nslots) {
    if (!ctx || !ms || reps < 1 || nslots < PROF_NSLOT) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    if (ctx->d.halo) {   // the halo exchange has to come between the sub-steps
        ctx->err = "a block with halo sides steps through hamr_stage, hamr_bound_dim and the halo exchange";
        return HAMR_E_STATE;
    }
    Prof pf;
    for (auto &e : pf.ev) CK(cudaEventCreate(&e));
    pf.on = true;
    for (int k = 0; k < nslots; k++) ms[k] = 0.;
    int rc = HAMR_OK;
    for (int r = 0; r < reps && rc == HAMR_OK; r++) {
        for (int stage = 0; stage < 2 && rc == HAMR_OK; stage++) {
            k_dt_reset<<<1, 32, 0, ctx->stream>>>(ctx->dtbits);
            StepSize st{nullptr, 0., stage ? dt : 0.5 * dt, dt};
            // every group records its end mark, launched or not, so
            // consecutive marks bracket exactly one group
            cudaEventRecord(pf.ev[0], ctx->stream);
            rc = launch_stage(ctx, stage, st, stage == 1, &pf);
            if (rc) break;
            if (cudaEventSynchronize(pf.ev[PROF_NSLOT]) != cudaSuccess) { rc = HAMR_E_CUDA; break; }
            for (int k = 0; k < PROF_NSLOT; k++) {
                float t = 0.f;
                cudaEventElapsedTime(&t, pf.ev[k], pf.ev[k + 1]);
                ms[k] += t / reps;
            }
        }
    }
    for (auto &e : pf.ev) cudaEventDestroy(e);
    return rc;
}

int hamr_device_state(hamr_ctx *ctx, double **p, double **ps, double **ph, double **psh) {
    if (!ctx) return HAMR_E_ARG;
    if (p) *p = ctx->p;
    if (ps) *ps = ctx->ps;
    if (ph) *ph = ctx->ph;
    if (psh) *psh = ctx->psh;
    return HAMR_OK;
}

int hamr_divb_max(hamr_ctx *ctx, double *out) {
    if (!ctx || !out) return HAMR_E_ARG;
    if (!ctx->have_geom) return HAMR_E_STATE;
    const Dims &d = ctx->d;
    CK(cudaMemsetAsync(ctx->divb, 0, sizeof(unsigned long long), ctx->stream));
    k_divb<<<nblk((long)d.n1 * d.n2 * d.n3), BLK, 0, ctx->stream>>>(d, geom_of(ctx), ctx->ps, ctx->divb);
    CK(cudaGetLastError());
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, ctx->divb, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    memcpy(out, &bits, sizeof(double));
    return HAMR_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free step (hamr_step_noalloc). All intermediate arrays of one RK2
// step -- half-step state, cached conserved variables, face fluxes, EMFs,
// inversion flags, CFL minima -- live in file-scope device arrays sized for at
// most HAMR_NOALLOC_MAX_CELLS zones per plane. Every GPU that loads the library
// holds these arrays (about 17 MB) until the process exits; every call shares
// them, so calls that overlap on the GPU race.
namespace {

constexpr long NA_DPLANES = 9 + 3 + 9 + 27 + 4 + 4 + 7;  // ph, psh, U, F1-F3, E_cent, emf, W
constexpr long NA_IPLANES = 1 + 4 + 1;               // pflag, failimage, failed-zone list
static __device__ __align__(256) double na_scratch[NA_DPLANES * HAMR_NOALLOC_MAX_CELLS];
static __device__ __align__(256) int na_iscratch[NA_IPLANES * HAMR_NOALLOC_MAX_CELLS];
static __device__ __align__(256) unsigned long long na_dtbits[4];
static __device__ __align__(256) double na_ndt[1];
static __device__ __align__(256) int na_nfail[1];

constexpr int NA_MAX_DEVICES = 64;
struct NaPtrs {
    double *scratch = nullptr;
    int *iscratch = nullptr;
    unsigned long long *dtbits = nullptr;
    double *ndt = nullptr;
    int *nfail = nullptr;
};
NaPtrs na_ptrs[NA_MAX_DEVICES];
// set (release) after na_ptrs[dev] is written; a reader that sees it set
// (acquire) also sees the pointers
std::atomic<bool> na_ready[NA_MAX_DEVICES];
std::mutex na_mutex;

// Device addresses of the scratch arrays on the current device, looked up once
// per device: in host code the array names are host-side stand-ins.
int na_setup(int dev) {
    std::lock_guard<std::mutex> lock(na_mutex);
    if (na_ready[dev].load(std::memory_order_acquire)) return HAMR_OK;
    NaPtrs q;
    if (cudaGetSymbolAddress((void **)&q.scratch, na_scratch) != cudaSuccess) return HAMR_E_CUDA;
    if (cudaGetSymbolAddress((void **)&q.iscratch, na_iscratch) != cudaSuccess) return HAMR_E_CUDA;
    if (cudaGetSymbolAddress((void **)&q.dtbits, na_dtbits) != cudaSuccess) return HAMR_E_CUDA;
    if (cudaGetSymbolAddress((void **)&q.ndt, na_ndt) != cudaSuccess) return HAMR_E_CUDA;
    if (cudaGetSymbolAddress((void **)&q.nfail, na_nfail) != cudaSuccess) return HAMR_E_CUDA;
    na_ptrs[dev] = q;
    na_ready[dev].store(true, std::memory_order_release);
    return HAMR_OK;
}

}  // namespace

extern "C" int hamr_step_noalloc(const hamr_params *prm, const double *gcov, const double *gcon,
                                 const double *gdet, const double *conn, double *p, double *ps,
                                 double dt, double *dt_next) {
    if (!prm || !gcov || !gcon || !gdet || !conn || !p || !ps || !(dt > 0)) return HAMR_E_ARG;
    if (prm->n1 < 2 || prm->n2 < 2 || prm->n3 < 1 || prm->precision != HAMR_FP64 || prm->halo) return HAMR_E_ARG;
    if (prm->floors || prm->repair) return HAMR_E_ARG;
    if (prm->recon != HAMR_RECON_PPM && prm->recon != HAMR_RECON_MC) return HAMR_E_ARG;
    if (prm->riemann != HAMR_RIEMANN_HLL && prm->riemann != HAMR_RIEMANN_HLLC) return HAMR_E_ARG;
    if (!(prm->ng == 3 || (prm->ng == 2 && prm->recon == HAMR_RECON_MC))) return HAMR_E_ARG;
    if (prm->inversion != HAMR_INV_2D && prm->inversion != HAMR_INV_NM) return HAMR_E_ARG;
    if (prm->n3 > 1 && prm->bc3 != HAMR_BC_PERIODIC) return HAMR_E_ARG;
    if (prm->bc2 == HAMR_BC_POLE_TRANS && (prm->n3 < 2 || prm->n3 % 2)) return HAMR_E_ARG;
    if (!(prm->gam > 1.0) || !(prm->cour > 0.0) || !(prm->dx1 > 0) || !(prm->dx2 > 0) || !(prm->dx3 > 0)) return HAMR_E_ARG;
    // the same dimension bookkeeping as hamr_ctx_create
    hamr_ctx c{};   // value-initialised: every field not set below is zero
    c.rows_min = 1L << 60;   // blocks this small keep one thread per face
    c.cons_tma = false;      // the update without the bulk-copy staging (no error word here)
    c.concurrent = false;    // no side streams
    c.prm = *prm;
    Dims &d = c.d;
    d.n1 = prm->n1; d.n2 = prm->n2; d.n3 = prm->n3;
    d.d1 = d.n1 > 1; d.d2 = d.n2 > 1; d.d3 = d.n3 > 1;
    d.ng1 = d.d1 ? prm->ng : 0; d.ng2 = d.d2 ? prm->ng : 0; d.ng3 = d.d3 ? prm->ng : 0;
    d.G1 = d.n1 + 2 * d.ng1; d.G2 = d.n2 + 2 * d.ng2; d.G3 = d.n3 + 2 * d.ng3;
    const long ncell = (long)d.G1 * d.G2 * d.G3, ngeo = (long)d.G1 * d.G2;
    d.ks = prm->ksize ? prm->ksize : ncell + (64 - ncell % 64);
    d.gs = prm->gsize ? prm->gsize : ngeo + (64 - ngeo % 64);
    if (d.ks < ncell || d.gs < ngeo) return HAMR_E_ARG;
    if (d.ks > HAMR_NOALLOC_MAX_CELLS) return HAMR_E_ARG;   // beyond the static scratch
    d.dx1 = prm->dx1; d.dx2 = prm->dx2; d.dx3 = prm->dx3;
    d.rdx1 = 1.0 / d.dx1; d.rdx2 = 1.0 / d.dx2; d.rdx3 = 1.0 / d.dx3;
    d.rgam = 1.0 / prm->gam;
    d.gam = prm->gam; d.cour = prm->cour;
    set_cfl_limits(d);   // after dx and cour
    d.pole1 = prm->pole1; d.pole2 = prm->pole2;
    d.bc1 = prm->bc1; d.bc2 = prm->bc2; d.bc3 = prm->bc3;
    d.ct_upwind = prm->ct_upwind;
    d.inversion = prm->inversion;
    d.recon = prm->recon;
    d.riemann = prm->riemann;
    d.halo = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return HAMR_E_CUDA;
    if (!na_ready[dev].load(std::memory_order_acquire) && na_setup(dev) != HAMR_OK) return HAMR_E_CUDA;
    const NaPtrs &q = na_ptrs[dev];
    const long ks = d.ks;
    c.stream = (cudaStream_t)prm->stream;
    c.have_geom = true;
    c.p = p;
    c.ps = ps;
    c.ph = q.scratch;
    c.psh = c.ph + 9 * ks;
    c.U = c.psh + 3 * ks;
    c.F1 = c.U + 9 * ks;
    c.F2 = c.F1 + 9 * ks;
    c.F3 = c.F2 + 9 * ks;
    c.Ec = c.F3 + 9 * ks;
    c.emf = c.Ec + 4 * ks;
    c.W = c.emf + 4 * ks;
    c.pflag = q.iscratch;
    c.failimage = q.iscratch + ks;
    c.flist = q.iscratch + 5 * ks;   // cleared per sub-step by the conserved update
    c.nfail = q.nfail;
    c.gcov = const_cast<double *>(gcov);
    c.gcon = const_cast<double *>(gcon);
    c.gdet = const_cast<double *>(gdet);
    c.conn = const_cast<double *>(conn);
    c.dtbits = q.dtbits;
    c.ndt = q.ndt;
    c.counter = nullptr;
    // the arrays keep the previous call's contents: zero the failure counters
    // and, in 2-D, the x3 fluxes and centre EMFs the edge-EMF kernel reads
    if (cudaMemsetAsync(c.failimage, 0, 4 * sizeof(int) * ks, c.stream) != cudaSuccess) return HAMR_E_CUDA;
    if (!d.d3) {
        if (cudaMemsetAsync(c.F3, 0, 9 * sizeof(double) * ks, c.stream) != cudaSuccess) return HAMR_E_CUDA;
        if (cudaMemsetAsync(c.Ec, 0, 4 * sizeof(double) * ks, c.stream) != cudaSuccess) return HAMR_E_CUDA;
    }
    k_dt_reset<<<1, 32, 0, c.stream>>>(c.dtbits);
    int rc = launch_step(&c, StepSize{nullptr, 0.5, 0.5 * dt, dt}, StepSize{nullptr, 1.0, dt, dt}, nullptr, 0);
    c.p = c.ps = nullptr;  // caller-owned: not ours to release
    if (rc) return rc;
    if (dt_next) {
        if (cudaMemcpyAsync(dt_next, c.ndt, sizeof(double), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess) return HAMR_E_CUDA;
        if (cudaStreamSynchronize(c.stream) != cudaSuccess) return HAMR_E_CUDA;
        if (!(*dt_next > 0) || !isfinite(*dt_next)) return HAMR_E_PHYSICS;
    }
    return HAMR_OK;
}

#include "hamr_batch.cuh"
#include "hamr_adjoint.cuh"
