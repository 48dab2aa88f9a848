/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Forward-mode dual numbers for a tangent-linear build of the oracle
 * (oracle_dual.cpp): every double of hamr_oracle.c becomes a value with
 * HD_NT tangents, carried through the same arithmetic in the same order, so
 * the values are the oracle's own and each tangent is the directional
 * derivative of the step along one seeded direction, in the branch the
 * values take (an active min/max/clamp passes its argument's derivative;
 * Newton iterates are differentiated as iterated). The adjoint of the CUDA
 * library is checked against it: <gradient, v> must equal the tangent of the
 * objective along v.
 */
#pragma once
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef HD_NT
#define HD_NT 8
#endif

struct hd_dual {
    double v;
    double d[HD_NT];
    hd_dual() = default;
    hd_dual(double x) : v(x) {
        for (int q = 0; q < HD_NT; q++) d[q] = 0.0;
    }
    explicit operator int() const { return (int)v; }
    explicit operator long() const { return (long)v; }
    hd_dual &operator+=(const hd_dual &b) {
        for (int q = 0; q < HD_NT; q++) d[q] += b.d[q];
        v += b.v;
        return *this;
    }
    hd_dual &operator-=(const hd_dual &b) {
        for (int q = 0; q < HD_NT; q++) d[q] -= b.d[q];
        v -= b.v;
        return *this;
    }
    hd_dual &operator*=(const hd_dual &b) {
        for (int q = 0; q < HD_NT; q++) d[q] = d[q] * b.v + v * b.d[q];
        v *= b.v;
        return *this;
    }
    hd_dual &operator/=(const hd_dual &b) {
        const double r = v / b.v;
        for (int q = 0; q < HD_NT; q++) d[q] = (d[q] - r * b.d[q]) / b.v;
        v = r;
        return *this;
    }
};
// value f, derivative scale df: tangents df * a.d
static inline hd_dual hd_chain(double f, double df, const hd_dual &a) {
    hd_dual o;
    o.v = f;
    for (int q = 0; q < HD_NT; q++) o.d[q] = df * a.d[q];
    return o;
}
static inline hd_dual operator+(hd_dual a, const hd_dual &b) { return a += b; }
static inline hd_dual operator-(hd_dual a, const hd_dual &b) { return a -= b; }
static inline hd_dual operator-(const hd_dual &a) { return hd_chain(-a.v, -1.0, a); }
static inline hd_dual operator+(const hd_dual &a) { return a; }
static inline hd_dual operator*(hd_dual a, const hd_dual &b) { return a *= b; }
static inline hd_dual operator/(hd_dual a, const hd_dual &b) { return a /= b; }
static inline hd_dual operator+(hd_dual a, double b) { return a += hd_dual(b); }
static inline hd_dual operator+(double a, const hd_dual &b) { return hd_dual(a) += b; }
static inline hd_dual operator-(hd_dual a, double b) { return a -= hd_dual(b); }
static inline hd_dual operator-(double a, const hd_dual &b) { return hd_dual(a) -= b; }
static inline hd_dual operator*(const hd_dual &a, double b) { return hd_chain(a.v * b, b, a); }
static inline hd_dual operator*(double a, const hd_dual &b) { return hd_chain(a * b.v, a, b); }
static inline hd_dual operator/(const hd_dual &a, double b) {
    hd_dual o;
    o.v = a.v / b;
    for (int q = 0; q < HD_NT; q++) o.d[q] = a.d[q] / b;
    return o;
}
static inline hd_dual operator/(double a, const hd_dual &b) { return hd_dual(a) /= b; }
#define HD_CMP(op)                                                                        \
    static inline bool operator op(const hd_dual &a, const hd_dual &b) { return a.v op b.v; } \
    static inline bool operator op(const hd_dual &a, double b) { return a.v op b; }          \
    static inline bool operator op(double a, const hd_dual &b) { return a op b.v; }
HD_CMP(<) HD_CMP(>) HD_CMP(<=) HD_CMP(>=) HD_CMP(==) HD_CMP(!=)
#undef HD_CMP
static inline bool operator!(const hd_dual &a) { return !a.v; }

static inline hd_dual sqrt(const hd_dual &a) {
    const double s = sqrt(a.v);
    return hd_chain(s, s > 0.0 ? 0.5 / s : 0.0, a);
}
static inline hd_dual fabs(const hd_dual &a) { return a.v < 0.0 ? -a : a; }
static inline hd_dual exp(const hd_dual &a) { const double e = exp(a.v); return hd_chain(e, e, a); }
static inline hd_dual log(const hd_dual &a) { return hd_chain(log(a.v), 1.0 / a.v, a); }
static inline hd_dual sin(const hd_dual &a) { return hd_chain(sin(a.v), cos(a.v), a); }
static inline hd_dual cos(const hd_dual &a) { return hd_chain(cos(a.v), -sin(a.v), a); }
static inline hd_dual acos(const hd_dual &a) {
    const double s = sqrt(1.0 - a.v * a.v);
    return hd_chain(acos(a.v), s > 0.0 ? -1.0 / s : 0.0, a);
}
static inline hd_dual pow(const hd_dual &a, const hd_dual &b) {
    hd_dual o;
    o.v = pow(a.v, b.v);
    const double da = b.v * pow(a.v, b.v - 1.0);
    const double db = a.v > 0.0 ? o.v * log(a.v) : 0.0;
    for (int q = 0; q < HD_NT; q++) o.d[q] = (a.d[q] != 0.0 ? da * a.d[q] : 0.0) + (b.d[q] != 0.0 ? db * b.d[q] : 0.0);
    return o;
}
static inline hd_dual pow(const hd_dual &a, double b) { return pow(a, hd_dual(b)); }
static inline hd_dual pow(double a, const hd_dual &b) { return pow(hd_dual(a), b); }
static inline hd_dual fma(const hd_dual &a, const hd_dual &b, const hd_dual &c) {
    hd_dual o;
    o.v = fma(a.v, b.v, c.v);
    for (int q = 0; q < HD_NT; q++) o.d[q] = a.d[q] * b.v + a.v * b.d[q] + c.d[q];
    return o;
}
static inline hd_dual fmax(const hd_dual &a, const hd_dual &b) { return a.v >= b.v ? a : b; }
static inline hd_dual fmin(const hd_dual &a, const hd_dual &b) { return a.v <= b.v ? a : b; }
static inline int isfinite(const hd_dual &a) { return isfinite(a.v); }
static inline int isnan(const hd_dual &a) { return isnan(a.v); }

// OpenMP reductions of the oracle's parallel loops, on the values
#pragma omp declare reduction(min : hd_dual : omp_out = (omp_in.v < omp_out.v ? omp_in : omp_out)) \
    initializer(omp_priv = hd_dual(1.e300))
#pragma omp declare reduction(max : hd_dual : omp_out = (omp_in.v > omp_out.v ? omp_in : omp_out)) \
    initializer(omp_priv = hd_dual(-1.e300))
#pragma omp declare reduction(+ : hd_dual : omp_out += omp_in) initializer(omp_priv = hd_dual(0.0))

#define double hd_dual
