// Forward-mode dual numbers for local derivatives in the adjoint kernels:
// a value and N directional derivatives, propagated exactly (to rounding) by
// the chain rule. The physics routines are templates on their arithmetic
// type, so instantiating them with Dual<N> differentiates the very code the
// forward step runs, in the branch it takes at the point of evaluation.
#pragma once
#include <math.h>

namespace hamr {

template <int N>
struct Dual {
    double v;
    double d[N];
    __host__ __device__ Dual() {}
    __host__ __device__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; k++) d[k] = 0.;
    }
    __host__ __device__ explicit operator double() const { return v; }
};

template <int N>
__device__ __forceinline__ Dual<N> dual_var(double x, int dir) {
    Dual<N> r(x);
    if (dir >= 0 && dir < N) r.d[dir] = 1.;
    return r;
}

#define HAMR_DUAL_LOOP _Pragma("unroll") for (int k = 0; k < N; k++)

template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v + b.v; HAMR_DUAL_LOOP r.d[k] = a.d[k] + b.d[k]; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v - b.v; HAMR_DUAL_LOOP r.d[k] = a.d[k] - b.d[k]; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a) {
    Dual<N> r; r.v = -a.v; HAMR_DUAL_LOOP r.d[k] = -a.d[k]; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v * b.v; HAMR_DUAL_LOOP r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v / b.v;
    const double ib = 1. / b.v;
    HAMR_DUAL_LOOP r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, double b) { Dual<N> r = a; r.v += b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N> &b) { return b + a; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, double b) { Dual<N> r = a; r.v -= b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N> &b) { return -b + a; }
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, double b) {
    Dual<N> r; r.v = a.v * b; HAMR_DUAL_LOOP r.d[k] = a.d[k] * b; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N> &b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, double b) {
    Dual<N> r; r.v = a.v / b; const double ib = 1. / b; HAMR_DUAL_LOOP r.d[k] = a.d[k] * ib; return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N> &b) { return Dual<N>(a) / b; }
template <int N> __device__ __forceinline__ Dual<N> &operator+=(Dual<N> &a, const Dual<N> &b) { a = a + b; return a; }
template <int N> __device__ __forceinline__ Dual<N> &operator-=(Dual<N> &a, const Dual<N> &b) { a = a - b; return a; }
template <int N> __device__ __forceinline__ Dual<N> &operator*=(Dual<N> &a, const Dual<N> &b) { a = a * b; return a; }
template <int N> __device__ __forceinline__ Dual<N> &operator/=(Dual<N> &a, const Dual<N> &b) { a = a / b; return a; }
template <int N> __device__ __forceinline__ Dual<N> &operator*=(Dual<N> &a, double b) { a = a * b; return a; }

// comparisons look at the value: the branch the forward code takes
template <int N> __device__ __forceinline__ bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N> __device__ __forceinline__ bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }

// the elementary functions the physics routines call
template <int N> __device__ __forceinline__ Dual<N> d_sqrt(Dual<N> x) {
    Dual<N> r; r.v = sqrt(x.v);
    const double h = 0.5 / r.v;
    HAMR_DUAL_LOOP r.d[k] = x.d[k] * h;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> d_pow(Dual<N> x, Dual<N> y) {
    // x^y, d = x^y (y' ln x + y x'/x)
    Dual<N> r; r.v = pow(x.v, y.v);
    const double lx = log(x.v), yx = y.v / x.v;
    HAMR_DUAL_LOOP r.d[k] = r.v * (y.d[k] * lx + yx * x.d[k]);
    return r;
}

#undef HAMR_DUAL_LOOP

}  // namespace hamr
