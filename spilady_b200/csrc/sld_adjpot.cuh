// Parameterised forms of the potential for the adjoint (sld_adjoint.cu):
// the functional forms of DD05.cpp:6-164 and JijFe.cpp:5-43 with their 36
// constants as a parameter vector theta,
//   [0, 2)   F(rho) = -a sqrt(rho) - [rho < 1] b/ln2 (1 - sqrt(rho)) ln(2 - rho)
//   [2, 8)   f(r) coefficients a_k, [8, 14) knots r_k:  f = sum a_k (r_k - r)^3, r < r_k
//   [14, 22) phi(r) coefficients V_k, [22, 30) knots:   phi = sum V_k (r_k - r)^3, r > 2 A
//            (the ZBL core below 1.8 A, and between 1.8 and 2.0 A the quintic
//            with the value and first two derivatives of both at the ends)
//   [30, 32) J(r) = A (1 - r/rc)^3, r < rc
//   [32, 36) Landau A, B, C, D (constants in rho)
// Every form is a template over the number type (double, or Dual<N> for
// derivatives) and over a parameter accessor, so one expression serves the
// forward pass and every partial derivative the adjoint needs.
#pragma once
#include "sld_common.cuh"
#include "sld_dual.cuh"

#define ADJ_NTHETA 36
enum {
    TH_FA = 0, TH_FB = 1, TH_DA = 2, TH_DK = 8, TH_PV = 14, TH_PK = 22, TH_JA = 30, TH_JRC = 31,
    TH_LANDAU = 32
};

// parameter vector and the ZBL end of the 1.8-2.0 A join (the reference's
// finite-difference derivatives of its ZBL term, DD05.cpp:97-99, from the host)
struct AdjConst {
    double th[ADJ_NTHETA];
    double y1, dy1, d2y1;
    double zbl_as;
};

template <class T>
struct Num;
template <>
struct Num<double> {
    static __device__ __forceinline__ double c(double v) { return v; }
};
template <int N>
struct Num<Dual<N>> {
    static __device__ __forceinline__ Dual<N> c(double v) { return dconst<N>(v); }
};

// parameter accessors: plain values, or values with partial off + k seeded
// for the parameters k in [lo, hi)
struct ThPlain {
    const double* th;
    __device__ __forceinline__ double operator()(int k) const { return th[k]; }
};
template <int N>
struct ThSeed {
    const double* th;
    int off, lo, hi;
    __device__ __forceinline__ Dual<N> operator()(int k) const {
        return dseed<N>(th[k], (k >= lo && k < hi) ? off + k : -1);
    }
};

// F(rho), F'(rho)
template <class T, class P>
__device__ __forceinline__ void adj_emb(const T& rho, const P& th, T& F, T& dF) {
    auto a = th(TH_FA);
    auto b = th(TH_FB);
    T sq = dsqrt(rho);
    F = -(a * sq);
    dF = -(0.5 * a / sq);
    if (val(rho) < 1.0) {
        T l = dlog(2.0 - rho);
        auto bl = b / 0.69314718055994530942;
        F = F - bl * (1.0 - sq) * l;
        dF = dF - bl * ((-0.5 / sq) * l - (1.0 - sq) / (2.0 - rho));
    }
}

// f(r), f'(r)
template <class T, class P>
__device__ __forceinline__ void adj_dens(const T& r, const P& th, T& f, T& df) {
    f = Num<T>::c(0.0);
    df = Num<T>::c(0.0);
    for (int k = 0; k < 6; ++k) {
        auto kk = th(TH_DK + k);
        if (val(r) < val(kk)) {
            auto u = kk - r;
            auto a = th(TH_DA + k);
            f = f + a * u * u * u;
            df = df - 3.0 * a * u * u;
        }
    }
}

// ZBL core (DD05.cpp:31-47): value and first two derivatives in r
__device__ __forceinline__ void adj_zbl(double as, double r, double& v, double& dv, double& d2v) {
    const double z2 = 26e0 * 26e0 * 14.3992;
    const double b[4] = {0.1818, 0.5099, 0.2802, 0.02817}, k[4] = {3.2, 0.9423, 0.4029, 0.2016};
    double x = r / as, s = 0.0, ds = 0.0, d2s = 0.0;
    for (int q = 0; q < 4; ++q) {
        double e = b[q] * exp(-k[q] * x);
        s += e;
        ds -= k[q] / as * e;
        d2s += (k[q] / as) * (k[q] / as) * e;
    }
    v = z2 * s / r;
    dv = z2 * (ds * r - s) / (r * r);
    d2v = z2 * (d2s * r * r - 2.0 * (ds * r - s)) / (r * r * r);
}

// phi(r), phi'(r)
template <class T, class P>
__device__ __forceinline__ void adj_pair(const AdjConst& K, const T& r, const P& th, T& v, T& dv) {
    const double x1 = 1.8, x2 = 2.0;
    v = Num<T>::c(0.0);
    dv = Num<T>::c(0.0);
    if (val(r) > x2) {
        for (int k = 0; k < 8; ++k) {
            auto kk = th(TH_PK + k);
            if (val(r) < val(kk)) {
                auto u = kk - r;
                auto V = th(TH_PV + k);
                v = v + V * u * u * u;
                dv = dv - 3.0 * V * u * u;
            }
        }
    } else if (val(r) > x1) {
        // quintic in Hermite form: value, slope and curvature of the ZBL
        // core at x1 and of the knot cubics at x2
        auto y2 = Num<decltype(th(0))>::c(0.0), d2 = y2, c2 = y2;
        for (int k = 0; k < 8; ++k) {
            auto kk = th(TH_PK + k);
            if (x2 < val(kk)) {
                auto u = kk - x2;
                auto V = th(TH_PV + k);
                y2 = y2 + V * u * u * u;
                d2 = d2 - 3.0 * V * u * u;
                c2 = c2 + 6.0 * V * u;
            }
        }
        const double h = x2 - x1;
        T t = (r - x1) / h;
        T t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
        T h0 = 1.0 - 10.0 * t3 + 15.0 * t4 - 6.0 * t5;
        T h1 = t - 6.0 * t3 + 8.0 * t4 - 3.0 * t5;
        T h2 = 0.5 * t2 - 1.5 * t3 + 1.5 * t4 - 0.5 * t5;
        T h3 = 10.0 * t3 - 15.0 * t4 + 6.0 * t5;
        T h4 = -4.0 * t3 + 7.0 * t4 - 3.0 * t5;
        T h5 = 0.5 * t3 - t4 + 0.5 * t5;
        T g0 = -30.0 * t2 + 60.0 * t3 - 30.0 * t4;
        T g1 = 1.0 - 18.0 * t2 + 32.0 * t3 - 15.0 * t4;
        T g2 = t - 4.5 * t2 + 6.0 * t3 - 2.5 * t4;
        T g3 = 30.0 * t2 - 60.0 * t3 + 30.0 * t4;
        T g4 = -12.0 * t2 + 28.0 * t3 - 15.0 * t4;
        T g5 = 1.5 * t2 - 4.0 * t3 + 2.5 * t4;
        v = K.y1 * h0 + (h * K.dy1) * h1 + (h * h * K.d2y1) * h2 + y2 * h3 + (h * d2) * h4 +
            (h * h * c2) * h5;
        dv = (K.y1 * g0 + (h * K.dy1) * g1 + (h * h * K.d2y1) * g2 + y2 * g3 + (h * d2) * g4 +
              (h * h * c2) * g5) / h;
    } else {
        double z, dz, d2z;
        adj_zbl(K.zbl_as, val(r), z, dz, d2z);
        // the core has no parameters; its slope and curvature carry r's partials
        v = Num<T>::c(z) + (r - val(r)) * dz;
        dv = Num<T>::c(dz) + (r - val(r)) * d2z;
    }
}

// J(r), J'(r)
template <class T, class P>
__device__ __forceinline__ void adj_exch(const T& r, const P& th, T& J, T& dJ) {
    auto A = th(TH_JA);
    auto rc = th(TH_JRC);
    J = Num<T>::c(0.0);
    dJ = Num<T>::c(0.0);
    if (val(r) < val(rc)) {
        auto u = 1.0 - r / rc;
        J = A * u * u * u;
        dJ = -3.0 * A * u * u / rc;
    }
}

// FP32 twins of the pair forms for the split-precision forward pass (the
// parameters rounded to FP32; the 1.8-2.0 A join and the ZBL core, reached
// only in close collisions, in FP64)
__device__ __forceinline__ void adj_dens32(const AdjConst& K, float r, float& f, float& df) {
    f = 0.f;
    df = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float kk = (float)K.th[TH_DK + k];
        if (r < kk) {
            float u = kk - r, a = (float)K.th[TH_DA + k];
            f = fmaf(a * u * u, u, f);
            df = fmaf(-3.f * a, u * u, df);
        }
    }
}

__device__ __forceinline__ void adj_pair32(const AdjConst& K, double r64, float& v, float& dv) {
    float r = (float)r64;
    if (r64 > 2.0) {
        v = 0.f;
        dv = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float kk = (float)K.th[TH_PK + k];
            if (r < kk) {
                float u = kk - r, V = (float)K.th[TH_PV + k];
                v = fmaf(V * u * u, u, v);
                dv = fmaf(-3.f * V, u * u, dv);
            }
        }
    } else {
        double v64, dv64;
        adj_pair(K, r64, ThPlain{K.th}, v64, dv64);
        v = (float)v64;
        dv = (float)dv64;
    }
}

__device__ __forceinline__ void adj_exch32(const AdjConst& K, float r, float& J, float& dJ) {
    float A = (float)K.th[TH_JA], rc = (float)K.th[TH_JRC];
    J = 0.f;
    dJ = 0.f;
    if (r < rc) {
        float u = 1.f - r / rc;
        J = A * u * u * u;
        dJ = -3.f * A * u * u / rc;
    }
}

