// Split-precision form: the potential evaluated analytically in FP32, and
// compensated FP32 sums.
//
// The FP64 form reads the reference's 10^6-point tables (built from the
// DD05.cpp / JijFe.cpp forms, with seven-point numerical derivatives); here
// the same functional forms and their exact derivatives are evaluated
// directly in FP32, which needs no table traffic.  The pair term between
// 1.8 and 2.0 A is the quintic that joins the ZBL core to the cubic knots
// (its Hermite data is computed on the host in FP64); below 1.8 A it is the
// ZBL screened Coulomb term itself.
#pragma once
#include "sld_common.cuh"

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

// DD05 density f(r) = sum a_i (r_i - r)^3 for r < r_i, and f'(r)
__device__ __forceinline__ void dens32(float r, float& f, float& df) {
    const float a[6] = {0.9332056681088162f, -1.162558782567700f, -0.3502026949249225f,
                        0.4287820835430028f, 4.907925057809273f, -5.307049068415304f};
    const float k[6] = {3.0f, 2.8666666666666666f, 2.7333333333333333f, 2.6f, 2.4f, 2.3f};
    f = 0.f;
    df = 0.f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float u = k[i] - r;
        if (u > 0.f) {
            float u2 = u * u;
            f = fmaf(a[i] * u2, u, f);
            df = fmaf(-3.f * a[i], u2, df);
        }
    }
}

// DD05 embedding F(rho) and F'(rho)
__device__ __forceinline__ void emb32(float rho, float& F, float& dF) {
    const float a = 4.100199340884814f, b = 1.565647547483517f;
    const float b_ln2 = 1.565647547483517f / 0.69314718055994531f;
    float sq = sqrtf(rho);
    F = -a * sq;
    dF = -0.5f * a / sq;
    if (rho < 1.f) {
        float l = logf(2.f - rho);
        F -= b_ln2 * (1.f - sq) * l;
        dF -= b_ln2 * ((-0.5f / sq) * l - (1.f - sq) / (2.f - rho));
    }
    (void)b;
}

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

// DD05 pair term phi(r) and phi'(r)
__device__ __forceinline__ void pair32(const Pot32& P, float r, float& v, float& dv) {
    const float V[8] = {-0.1960674387419232f, 0.3687525935422963f, -1.505333614924853f,
                        4.948907078156191f,   -4.894613262753399f, 3.468897724782442f,
                        -1.792218099820337f,  80.22069592246987f};
    const float K[8] = {4.1f, 3.8f, 3.5f, 3.2f, 2.9f, 2.6f, 2.4f, 2.3f};
    if (r > 2.0f) {
        v = 0.f;
        dv = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float u = K[i] - r;
            if (u > 0.f) {
                float u2 = u * u;
                v = fmaf(V[i] * u2, u, v);
                dv = fmaf(-3.f * V[i], u2, dv);
            }
        }
        return;
    }
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

// Fe exchange J(r) = 0.870 (1 - r/3.75)^3 for r < 3.75, and J'(r)
__device__ __forceinline__ void exch32(float r, float& J, float& dJ) {
    const float A = 0.870f, rc = 3.75f;
    float u = 1.f - r / rc;
    if (u > 0.f) {
        J = A * u * u * u;
        dJ = -3.f * A / rc * u * u;
    } else {
        J = 0.f;
        dJ = 0.f;
    }
}

// One piecewise cubic (knots K[0..n), coefficients C[4*(n+1)]) at r, with
// t = r - base formed in FP64 so that it carries FP32 relative precision.
__device__ __forceinline__ void cubic_eval(const float* __restrict__ K, const float* __restrict__ C,
                                           int n, double r, float& f, float& df) {
    int m = 0;
    for (int i = 0; i < n; ++i) m += r >= (double)__ldg(K + i);
    if (m == n) {
        f = 0.f;
        df = 0.f;
        return;
    }
    double base = (double)__ldg(K + (m == 0 ? 0 : m - 1));
    float t = (float)(r - base);
    const float* c = C + 4 * m;
    float c0 = __ldg(c), c1 = __ldg(c + 1), c2 = __ldg(c + 2), c3 = __ldg(c + 3);
    f = fmaf(fmaf(fmaf(c3, t, c2), t, c1), t, c0);
    df = fmaf(fmaf(3.f * c3, t, 2.f * c2), t, c1);
}

// density f and f' at an FP64 distance
__device__ __forceinline__ void dens32r(const Dev& D, double r, float& f, float& df) {
    cubic_eval(D.cubic + 44, D.cubic + 50, 6, r, f, df);
}

// pair term phi and phi' at an FP64 distance (ZBL core and join below 2 A)
__device__ __forceinline__ void pair32r(const Dev& D, double r, float& v, float& dv) {
    if (r > 2.0) {
        cubic_eval(D.cubic, D.cubic + 8, 8, r, v, dv);
        return;
    }
    pair32(D.pot32, (float)r, v, dv);
}

// exchange J and J' at an FP64 distance
__device__ __forceinline__ void exch32r(double r, float& J, float& dJ) {
    const float A = 0.870f, rc = 3.75f;
    float u = (float)(1.0 - r * (1.0 / 3.75));
    if (u > 0.f) {
        J = A * u * u * u;
        dJ = -3.f * A / rc * u * u;
    } else {
        J = 0.f;
        dJ = 0.f;
    }
}

// ---- the same forms in FP64 (the split form's error reference) ----
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
