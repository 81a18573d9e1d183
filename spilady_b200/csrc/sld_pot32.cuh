// Split-precision form: the potential evaluated analytically in FP32, and
// compensated FP32 sums.
//
// The FP64 form reads the reference's 10^6-point tables (built from the
// DD05.cpp / JijFe.cpp forms, with seven-point numerical derivatives); here
// the same functions are evaluated directly in FP32, which needs no table
// traffic.  The values are the functional forms themselves (linear
// interpolation between table entries 4.1e-6 A apart changes them by less
// than FP64 rounding).  The derivatives are the reference's: its derivative
// tables hold the seven-point central difference with step dx = x/1000
// (potential_CPU.cpp:159-170), which for a piecewise cubic equals the exact
// derivative except within 3 dx of a knot, where the stencil straddles the
// knot; there the one term a (k - x)^3_+ that changes form adds the
// stencil's difference from its exact derivative (knot_stencil32 below).
// The embedding function F(rho) and F'(rho) are read from the reference's
// tables per atom, in FP64.  The pair term between 1.8 and 2.0 A is the
// quintic that joins the ZBL core to the cubic knots (its Hermite data is
// computed on the host in FP64); below 1.8 A it is the ZBL screened Coulomb
// term itself.
#pragma once
#include "sld_common.cuh"

// offsets in the split form's potential table (potential.h: kDensKnots,
// kPairIv, kDensIv)
#define SLD_DENS_KNOTS 80
#define SLD_PAIR_IV 8
#define SLD_DENS_IV 88

// compensated (Kahan) FP32 accumulator
struct Kahan {
    float s, c;
    __device__ __forceinline__ Kahan() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float x) {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

__device__ __forceinline__ void zbl32(const Pot32& P, float r, float& v, float& dv) {
    const float z2 = 26.f * 26.f * 14.3992f;
    float x = r / P.zbl_as;
    float e0 = expf(-3.2f * x), e1 = expf(-0.9423f * x), e2 = expf(-0.4029f * x),
          e3 = expf(-0.2016f * x);
    float s = 0.1818f * e0 + 0.5099f * e1 + 0.2802f * e2 + 0.02817f * e3;
    float ds = -(0.1818f * 3.2f * e0 + 0.5099f * 0.9423f * e1 + 0.2802f * 0.4029f * e2 +
                 0.02817f * 0.2016f * e3) / P.zbl_as;
    v = z2 * s / r;
    dv = z2 * (ds * r - s) / (r * r);
}

// DD05 pair term phi(r) and phi'(r) at r <= 2 A: the ZBL core below 1.8 A
// and the quintic join between 1.8 and 2.0 A
__device__ __forceinline__ void pair32(const Pot32& P, float r, float& v, float& dv) {
    if (r <= 1.8f) {
        zbl32(P, r, v, dv);
        return;
    }
    const float w = 0.2f;
    float t = (r - 1.8f) / w, t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
    float h00 = 1 - 10 * t3 + 15 * t4 - 6 * t5, h01 = 10 * t3 - 15 * t4 + 6 * t5;
    float h10 = t - 6 * t3 + 8 * t4 - 3 * t5, h11 = -4 * t3 + 7 * t4 - 3 * t5;
    float h20 = 0.5f * t2 - 1.5f * t3 + 1.5f * t4 - 0.5f * t5, h21 = 0.5f * t3 - t4 + 0.5f * t5;
    float g00 = -30 * t2 + 60 * t3 - 30 * t4, g01 = -g00;
    float g10 = 1 - 18 * t2 + 32 * t3 - 15 * t4, g11 = -12 * t2 + 28 * t3 - 15 * t4;
    float g20 = t - 4.5f * t2 + 6 * t3 - 2.5f * t4, g21 = 1.5f * t2 - 4 * t3 + 2.5f * t4;
    v = h00 * P.zbl_y1 + h01 * P.knot_y2 + w * (h10 * P.zbl_d1 + h11 * P.knot_d2) +
        w * w * (h20 * P.zbl_c1 + h21 * P.knot_c2);
    dv = (g00 * P.zbl_y1 + g01 * P.knot_y2 + w * (g10 * P.zbl_d1 + g11 * P.knot_d2) +
          w * w * (g20 * P.zbl_c1 + g21 * P.knot_c2)) / w;
}

// The seven-point derivative (potential_CPU.cpp:159-170) of x -> (k - x)^3_+
// at x = r with step dx, less the exact derivative -3 (k - r)^2_+, for
// u = k - r.  Zero (up to rounding) for |u| >= 3 dx, where the stencil sees
// one cubic.  The terms are of size dx^3 and the result of size dx^2, so FP32
// keeps it to about 1e-7 relative.  i60dx = 1 / (60 dx), formed by the caller
// from the pair's 1/r (a few ulp; the stencil's own division would cost a
// division per knot).
__device__ __forceinline__ float cube_pos32(float x) { return x > 0.f ? x * x * x : 0.f; }
__device__ __forceinline__ float knot_stencil32(float u, float dx, float i60dx) {
    float s = 45.f * (cube_pos32(u - dx) - cube_pos32(u + dx)) -
              9.f * (cube_pos32(u - 2.f * dx) - cube_pos32(u + 2.f * dx)) +
              (cube_pos32(u - 3.f * dx) - cube_pos32(u + 3.f * dx));
    float up = fmaxf(u, 0.f);
    return s * i60dx + 3.f * up * up;
}
// 1 / (60 dx) for dx = r / 1000, from ir = 1/r
__device__ __forceinline__ float stencil_i60(float ir) { return ir * (1.f / 0.06f); }
// The knots of the pair term and of the density (ascending), held in
// registers by a thread for its whole pair loop.
struct Knots32 {
    float p[8], d[6];
};
__device__ __forceinline__ Knots32 knots32(const Dev& D) {
    Knots32 K;
#pragma unroll
    for (int i = 0; i < 8; ++i) K.p[i] = __ldg(D.cubic + i);
#pragma unroll
    for (int i = 0; i < 6; ++i) K.d[i] = __ldg(D.cubic + SLD_DENS_KNOTS + i);
    return K;
}

// One piecewise cubic at an FP32 distance r: the interval m (the number of
// knots <= r) from the knots in registers, then its 32-byte block {c0..c3,
// base, upper knot, amplitudes of the knots below and above} in two loads.
// t = r - base is exact in FP32 (r and the knot are within a factor of two).
// df is the reference's seven-point derivative: within 3 r/1000 of the knot
// below or above (knots are 0.1 A or more apart, the stencil spans
// 6 r/1000 < 0.025 A) that knot's stencil term is added.
template <int N>
__device__ __forceinline__ void cubic_iv(const float (&K)[N], const float* __restrict__ blocks,
                                         float r, float ir, float& f, float& df) {
    int m = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) m += r >= K[i] ? 1 : 0;
    const float4* b = reinterpret_cast<const float4*>(blocks) + 2 * m;
    const float4 c = __ldg(b), e = __ldg(b + 1);
    const float t = r - e.x;
    f = fmaf(fmaf(fmaf(c.w, t, c.z), t, c.y), t, c.x);
    df = fmaf(fmaf(3.f * c.w, t, 2.f * c.z), t, c.y);
    const float dx = r * 1e-3f, i60 = stencil_i60(ir);
    const float ub = e.x - r, ua = e.y - r;
    if (ub > -3.f * dx && e.z != 0.f) df = fmaf(e.z, knot_stencil32(ub, dx, i60), df);
    if (ua < 3.f * dx) df = fmaf(e.w, knot_stencil32(ua, dx, i60), df);
}

// density f and the reference's f' at an FP32 distance r (ir = 1/r)
__device__ __forceinline__ void dens32f(const Dev& D, const Knots32& K, float r, float ir,
                                        float& f, float& df) {
    cubic_iv<6>(K.d, D.cubic + SLD_DENS_IV, r, ir, f, df);
}

// pair term phi and the reference's phi' at an FP32 distance (ZBL core and
// join below 2 A; within 3 r/1000 of 1.8 and 2.0 A the reference's stencil
// also straddles the joins, which only close collisions reach: there the
// exact derivative of the join is used)
__device__ __forceinline__ void pair32f(const Dev& D, const Knots32& K, float r, float ir,
                                        float& v, float& dv) {
    if (r > 2.0f) {
        cubic_iv<8>(K.p, D.cubic + SLD_PAIR_IV, r, ir, v, dv);
        return;
    }
    pair32(D.pot32, r, v, dv);
}

// Fe exchange J(r) = 0.870 (1 - r/3.75)^3 = a (3.75 - r)^3 for r < 3.75, and
// the reference's J'(r) (its stencil straddles the knot for |r - 3.75| < 3 dx)
__device__ __forceinline__ void exch32f(float r, float ir, float& J, float& dJ) {
    const float A = 0.870f, rc = 3.75f, a = 0.870f / (3.75f * 3.75f * 3.75f);
    float u = 1.f - r * (1.f / 3.75f);
    if (u > 0.f) {
        J = A * u * u * u;
        dJ = -3.f * A / rc * u * u;
    } else {
        J = 0.f;
        dJ = 0.f;
    }
    const float dx = r * 1e-3f, uk = rc - r;
    if (fabsf(uk) < 3.f * dx) dJ = fmaf(a, knot_stencil32(uk, dx, stencil_i60(ir)), dJ);
}

// F(rho) and F'(rho) from the reference's FP64 tables (potential_CPU.cpp:172-179)
__device__ __forceinline__ void emb_tab(const Dev& D, double rho, double& F, double& dF) {
    F = interp(D.tF, rho, D.inv_rho, &D.ctl->err);
    dF = interp(D.tdF, rho, D.inv_rho, &D.ctl->err);
}

// ---- the analytic forms in FP64 with their exact derivatives ----
// (SLD_FP64_ANALYTIC: the model the adjoint differentiates; it differs from
// the reference's tables by the tables' seven-point derivatives near the
// knots, about 1e-4 of the forces)
__device__ __forceinline__ void cubic_eval64(const double* __restrict__ K, const double* __restrict__ C,
                                             int n, double r, double& f, double& df) {
    int m = 0;
    for (int i = 0; i < n; ++i) m += r >= __ldg(K + i);
    if (m == n) {
        f = 0.0;
        df = 0.0;
        return;
    }
    double t = r - __ldg(K + (m == 0 ? 0 : m - 1));
    const double* c = C + 4 * m;
    double c0 = __ldg(c), c1 = __ldg(c + 1), c2 = __ldg(c + 2), c3 = __ldg(c + 3);
    f = ((c3 * t + c2) * t + c1) * t + c0;
    df = (3.0 * c3 * t + 2.0 * c2) * t + c1;
}
__device__ __forceinline__ void emb64(double rho, double& F, double& dF) {
    const double a = 4.100199340884814, b_ln2 = 1.565647547483517 / 0.69314718055994531;
    double sq = sqrt(rho);
    F = -a * sq;
    dF = -0.5 * a / sq;
    if (rho < 1.0) {
        double l = log(2.0 - rho);
        F -= b_ln2 * (1.0 - sq) * l;
        dF -= b_ln2 * ((-0.5 / sq) * l - (1.0 - sq) / (2.0 - rho));
    }
}
__device__ __forceinline__ void exch64(double r, double& J, double& dJ) {
    const double A = 0.870, rc = 3.75;
    double u = 1.0 - r / rc;
    if (u > 0.0) {
        J = A * u * u * u;
        dJ = -3.0 * A / rc * u * u;
    } else {
        J = 0.0;
        dJ = 0.0;
    }
}
__device__ __forceinline__ void pair64(const Dev& D, double r, double& v, double& dv) {
    if (r > 2.0) {
        cubic_eval64(D.cubic64, D.cubic64 + 8, 8, r, v, dv);
        return;
    }
    float vf, dvf;
    pair32(D.pot32, (float)r, vf, dvf);
    v = vf;
    dv = dvf;
}
__device__ __forceinline__ void dens64(const Dev& D, double r, double& f, double& df) {
    cubic_eval64(D.cubic64 + 44, D.cubic64 + 50, 6, r, f, df);
}
