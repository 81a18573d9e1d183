// Forward-mode dual numbers for the adjoint kernels: a value and N partial
// derivatives, carried through the same expressions as the value.  The
// adjoint passes evaluate each local term (one pair, one spin rotation) with
// its own inputs seeded and read the partials as that term's Jacobian row;
// the partials are exact derivatives of the rounded expression graph, in FP64.
#pragma once
#include <cuda_runtime.h>

template <int N>
struct Dual {
    double v;
    double d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(double v) {
    Dual<N> a;
    a.v = v;
#pragma unroll
    for (int k = 0; k < N; ++k) a.d[k] = 0.0;
    return a;
}

// v with unit partial k (k < 0 or k >= N: a constant)
template <int N>
__device__ __forceinline__ Dual<N> dseed(double v, int k) {
    Dual<N> a = dconst<N>(v);
    if (k >= 0 && k < N) a.d[k] = 1.0;
    return a;
}

__device__ __forceinline__ double val(double a) { return a; }
template <int N>
__device__ __forceinline__ double val(const Dual<N>& a) { return a.v; }

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> c;
    c.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] + b.d[k];
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> c;
    c.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] - b.d[k];
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> c;
    c.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = -a.d[k];
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> c;
    c.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> c;
    c.v = a.v / b.v;
    double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = (a.d[k] - c.v * b.d[k]) * ib;
    return c;
}
// mixed with plain doubles
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
    Dual<N> c = a;
    c.v += b;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double b, const Dual<N>& a) { return a + b; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
    Dual<N> c = a;
    c.v -= b;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double b, const Dual<N>& a) {
    Dual<N> c = -a;
    c.v += b;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> c;
    c.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] * b;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double b, const Dual<N>& a) { return a * b; }
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> c;
    c.v = a.v / b;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] / b;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
    Dual<N> c;
    c.v = a / b.v;
    double s = -c.v / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = s * b.d[k];
    return c;
}
template <int N, class B>
__device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const B& b) { return a = a + b; }
template <int N, class B>
__device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const B& b) { return a = a - b; }

// elementary functions: the value from CUDA's own function, the partials
// from its derivative
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dlog(double a) { return log(a); }
__device__ __forceinline__ double dexp(double a) { return exp(a); }
__device__ __forceinline__ double dsin(double a) { return sin(a); }
__device__ __forceinline__ double dcos(double a) { return cos(a); }

template <int N>
__device__ __forceinline__ Dual<N> chain(const Dual<N>& a, double v, double dv) {
    Dual<N> c;
    c.v = v;
#pragma unroll
    for (int k = 0; k < N; ++k) c.d[k] = a.d[k] * dv;
    return c;
}
template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
    double v = sqrt(a.v);
    return chain(a, v, 0.5 / v);
}
template <int N>
__device__ __forceinline__ Dual<N> dlog(const Dual<N>& a) { return chain(a, log(a.v), 1.0 / a.v); }
template <int N>
__device__ __forceinline__ Dual<N> dexp(const Dual<N>& a) {
    double v = exp(a.v);
    return chain(a, v, v);
}
template <int N>
__device__ __forceinline__ Dual<N> dsin(const Dual<N>& a) { return chain(a, sin(a.v), cos(a.v)); }
template <int N>
__device__ __forceinline__ Dual<N> dcos(const Dual<N>& a) { return chain(a, cos(a.v), -sin(a.v)); }
