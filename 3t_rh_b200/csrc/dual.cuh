// Forward-mode dual numbers with N tangent directions, for the local
// Jacobians the adjoint kernels need (the eigenvector matrices of a face as
// functions of its five Roe-averaged scalars, the CFL time step of a cell as
// a function of its state). Branches follow the values; the derivative of
// |x| at 0 is taken as +1, of max/min as that of the first argument on ties,
// the same conventions as the oracle's dual numbers.
#pragma once

namespace rh3t {

// the double versions stay visible beside the dual overloads below
using ::fabs;
using ::fmax;
using ::fmin;
using ::sqrt;

template <int N> struct DualN {
    double v;
    double d[N];
    __device__ __forceinline__ DualN() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    __device__ __forceinline__ DualN(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    // x with tangent e_k
    __device__ __forceinline__ static DualN var(double x, int k) {
        DualN r(x);
        r.d[k] = 1.0;
        return r;
    }
};

template <int N> __device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r(a.v + b.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r(a.v - b.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a) {
    DualN<N> r(-a.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator*(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r(a.v * b.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator/(const DualN<N>& a, const DualN<N>& b) {
    const double q = a.v / b.v, ib = 1.0 / b.v;
    DualN<N> r(q);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - q * b.d[k]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, double b) { return a + DualN<N>(b); }
template <int N> __device__ __forceinline__ DualN<N> operator+(double a, const DualN<N>& b) { return DualN<N>(a) + b; }
template <int N> __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a, double b) { return a - DualN<N>(b); }
template <int N> __device__ __forceinline__ DualN<N> operator-(double a, const DualN<N>& b) { return DualN<N>(a) - b; }
template <int N> __device__ __forceinline__ DualN<N> operator*(const DualN<N>& a, double b) {
    DualN<N> r(a.v * b);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator*(double a, const DualN<N>& b) {
    DualN<N> r(a * b.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a * b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator/(const DualN<N>& a, double b) {
    const double ib = 1.0 / b;
    DualN<N> r(a.v / b);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * ib;
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> operator/(double a, const DualN<N>& b) {
    const double q = a / b.v, f = -q / b.v;
    DualN<N> r(q);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = f * b.d[k];
    return r;
}

// at a.v = 0 a direction with zero tangent keeps a zero derivative (the
// local dt's discriminant is exactly 0 when both exchange coefficients are)
template <int N> __device__ __forceinline__ DualN<N> sqrt(const DualN<N>& a) {
    const double s = ::sqrt(a.v), h = 0.5 / s;
    DualN<N> r(s);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] == 0.0 ? 0.0 : a.d[k] * h;
    return r;
}
template <int N> __device__ __forceinline__ DualN<N> fabs(const DualN<N>& a) { return a.v < 0.0 ? -a : a; }
template <int N> __device__ __forceinline__ DualN<N> fmax(const DualN<N>& a, const DualN<N>& b) {
    return a.v >= b.v ? a : b;
}
template <int N> __device__ __forceinline__ DualN<N> fmin(const DualN<N>& a, const DualN<N>& b) {
    return a.v <= b.v ? a : b;
}

} // namespace rh3t
