// The electron heat-capacity model of core_dTe (heatcapacity_CPU.cpp:33-57):
// with u = b Te, b = 2e-4 / boltz, a = 3,
//     Ce = a tanh(u),  Ee = a/b log cosh(u),  Te = acosh(exp(b Ee / a)) / b.
// Two forms, chosen at compile time by the kernels of core_dTe:
//   FAST = false  the reference's expressions (the FP64 form);
//   FAST = true   polynomial forms fitted to these functions on
//                 u in [0, TE_U_MAX] (te_poly.h, from gen_te_poly.py), about
//                 1 ulp, with the reference's expressions outside it.  They
//                 are short FMA chains where the reference's compositions
//                 (log of cosh, acosh of exp) are long dependent chains of
//                 transcendental functions, and they avoid the cancellation
//                 of log(cosh u) and acosh(exp y) near u = 0.  Used by the
//                 split form and its FP64 twin.
#pragma once
#include "sld_common.cuh"
#include "te_poly.h"

#define TE_B (2e-4 / SLD_BOLTZ)
#define TE_A 3.0

// the reference's expressions, out of line: the fitted forms fall back to
// them only above TE_U_MAX (Te ~ 7500 K)
__device__ __noinline__ double te_to_Ee_far(double T) { return te_to_Ee(T); }
__device__ __noinline__ double Ee_to_te_far(double E) { return Ee_to_te(E); }
__device__ __noinline__ double te_coth_far(double u) { return 1.0 / tanh(u); }

__device__ __forceinline__ double te_to_Ee_fast(double T) {
    const double u = TE_B * T, v = u * u;
    if (!(v <= TE_V_MAX)) return te_to_Ee_far(T);
    const double t = (v - te_poly_logcosh_MID) * te_poly_logcosh_INV_HALF;
    return (TE_A / TE_B) * (v * te_poly_logcosh(t));
}

__device__ __forceinline__ double Ee_to_te_fast(double E) {
    const double y = (TE_B / TE_A) * E;
    if (!(y <= TE_Y_MAX)) return Ee_to_te_far(E);
    const double t = (y - te_poly_inv_logcosh_MID) * te_poly_inv_logcosh_INV_HALF;
    // y < 0 (no temperature has it) gives NaN, as acosh(exp(y)) does
    return sqrt(y * te_poly_inv_logcosh(t)) * (1.0 / TE_B);
}

// exp(x) - 1: the Taylor series through x^4/4! for |x| < 2^-14 (truncation
// below 2e-19 relative there), through x^8/8! for |x| < 2^-8 (below 2e-21),
// else expm1.  B's decay exponent is of order 1e-5 for femtosecond substeps.
__device__ __forceinline__ double te_expm1(double x) {
    if (fabs(x) < 6.103515625e-05) {
        double p = 1.0 / 24.0;
        p = fma(p, x, 1.0 / 6.0);
        p = fma(p, x, 0.5);
        return fma(x * x, p, x);
    }
    if (fabs(x) < 0.00390625) {
        double p = 1.0 / 40320.0;
        p = fma(p, x, 1.0 / 5040.0);
        p = fma(p, x, 1.0 / 720.0);
        p = fma(p, x, 1.0 / 120.0);
        p = fma(p, x, 1.0 / 24.0);
        p = fma(p, x, 1.0 / 6.0);
        p = fma(p, x, 0.5);
        return fma(x * x, p, x);
    }
    return expm1(x);
}

// exp(-g / Ce(Te)) - 1 = expm1(-(g / a) coth u)
__device__ __forceinline__ double te_decay_m1_fast(double g, double T) {
    const double u = TE_B * T, v = u * u;
    double coth;
    if (v <= TE_V_MAX) {
        const double t = (v - te_poly_coth_MID) * te_poly_coth_INV_HALF;
        coth = 1.0 / u + u * te_poly_coth(t);
    } else {
        coth = te_coth_far(u);
    }
    return te_expm1(-(g * (1.0 / TE_A)) * coth);
}

template <bool FAST>
__device__ __forceinline__ double te_E(double T) {
    if constexpr (FAST) return te_to_Ee_fast(T);
    else return te_to_Ee(T);
}

template <bool FAST>
__device__ __forceinline__ double te_T(double E) {
    if constexpr (FAST) return Ee_to_te_fast(E);
    else return Ee_to_te(E);
}

// B(hh): C dTe/dt = -(Ges + Gel) Te by the reference's RK4
// (core_dTe_CPU.cpp:105-124); g = (Gel + Ges) hh / boltz.  The fast form
// carries k hh instead of k, which removes the divisions by hh.
template <bool FAST>
__device__ __forceinline__ double te_rk4(double T, double g, double hh) {
    if constexpr (FAST) {
        const double m1 = T * te_decay_m1_fast(g, T);
        const double T1 = T + 0.5 * m1;
        const double m2 = T1 * te_decay_m1_fast(g, T1);
        const double T2 = T + 0.5 * m2;
        const double m3 = T2 * te_decay_m1_fast(g, T2);
        const double T3 = T + m3;
        const double m4 = T3 * te_decay_m1_fast(g, T3);
        return T + (m1 + 2.0 * m2 + 2.0 * m3 + m4) * (1.0 / 6.0);
    } else {
        double k1_ = T * (exp(-g / te_Ce(T)) - 1.0) / hh;
        double T1 = T + k1_ * hh / 2.0;
        double k2_ = T1 * (exp(-g / te_Ce(T1)) - 1.0) / hh;
        double T2 = T + k2_ * hh / 2.0;
        double k3_ = T2 * (exp(-g / te_Ce(T2)) - 1.0) / hh;
        double T3 = T + k3_ * hh;
        double k4_ = T3 * (exp(-g / te_Ce(T3)) - 1.0) / hh;
        return T + hh / 6.0 * (k1_ + 2.0 * k2_ + 2.0 * k3_ + k4_);
    }
}
