// Spin integrator of one visit (calculate_spin_CPU.cpp:33-199), FP64.
#pragma once
#include "sld_common.cuh"

// core_ds_CPU.cpp:90-127: exact rotation of s about -Heff/hbar by |w| dt
// sin x and 1 - cos x.  The rotation angle |w| dt of one visit is a small
// fraction of a radian, where the Taylor series of sin and of 1 - cos
// (truncated after x^15 and x^16: the next terms are below 1e-17 relative for
// |x| < 0.5) are far shorter than the general routine; larger angles use
// sincos.  1 - cos x from its own series also avoids the cancellation of
// 1 - cos(x) near zero.
__device__ __forceinline__ void sin_1mcos(double x, double& sn, double& omc) {
    if (fabs(x) < 0.5) {
        double x2 = x * x;
        // sin x = x (1 - x^2/3! + x^4/5! - ...)
        double p = -1.0 / 1307674368000.0;                 // -1/15!
        p = p * x2 + 1.0 / 6227020800.0;                   //  1/13!
        p = p * x2 - 1.0 / 39916800.0;                     // -1/11!
        p = p * x2 + 1.0 / 362880.0;                       //  1/9!
        p = p * x2 - 1.0 / 5040.0;                         // -1/7!
        p = p * x2 + 1.0 / 120.0;                          //  1/5!
        p = p * x2 - 1.0 / 6.0;                            // -1/3!
        sn = x + x * (x2 * p);
        // 1 - cos x = x^2 (1/2! - x^2/4! + x^4/6! - ...)
        double q = 1.0 / 20922789888000.0;                 //  1/16!
        q = q * x2 - 1.0 / 87178291200.0;                  // -1/14!
        q = q * x2 + 1.0 / 479001600.0;                    //  1/12!
        q = q * x2 - 1.0 / 3628800.0;                      // -1/10!
        q = q * x2 + 1.0 / 40320.0;                        //  1/8!
        q = q * x2 - 1.0 / 720.0;                          // -1/6!
        q = q * x2 + 1.0 / 24.0;                           //  1/4!
        q = q * x2 - 0.5;                                  // -1/2!
        omc = -(x2 * q);
        return;
    }
    double c;
    sincos(x, &sn, &c);
    omc = 1.0 - c;
}

// (w = -H/hbar is formed with one reciprocal and |w| with one reciprocal
// square root: the reference divides each component, which differs in the
// last bit at most)
//
// The rotation about -H/hbar by |w| dt depends only on H and dt, so its
// coefficients are formed once (RotCoef) and applied to any spin (rot_apply);
// the Langevin scheme's first and last parts share them.
struct RotCoef {
    double3 w;                      // unit axis
    double A, B;                    // sin, 1 - cos of the angle
    double w12, w23, w13, w1s, w2s, w3s;
};

__device__ __forceinline__ RotCoef rot_coef(double3 H, double dt) {
    const double k = -1.0 / SLD_HBAR;
    RotCoef c;
    double3 w = make_double3(H.x * k, H.y * k, H.z * k);
    double w2 = w.x * w.x + w.y * w.y + w.z * w.z;
    double iw = w2 > 0.0 ? rsqrt(w2) : 0.0;
    double w0 = w2 * iw;
    w = make_double3(w.x * iw, w.y * iw, w.z * iw);
    c.w = w;
    c.w12 = w.x * w.y; c.w23 = w.y * w.z; c.w13 = w.x * w.z;
    c.w1s = w.x * w.x; c.w2s = w.y * w.y; c.w3s = w.z * w.z;
    sin_1mcos(w0 * dt, c.A, c.B);
    return c;
}

__device__ __forceinline__ double3 rot_apply(const RotCoef& c, double3 s) {
    const double3 w = c.w;
    const double A = c.A, B = c.B;
    double3 o;
    o.x = s.x + (s.x * B * (-c.w2s - c.w3s) + s.y * (B * c.w12 - A * w.z) + s.z * (A * w.y + B * c.w13));
    o.y = s.y + (s.y * B * (-c.w1s - c.w3s) + s.z * (B * c.w23 - A * w.x) + s.x * (A * w.z + B * c.w12));
    o.z = s.z + (s.z * B * (-c.w1s - c.w2s) + s.x * (B * c.w13 - A * w.y) + s.y * (A * w.x + B * c.w23));
    return o;
}

__device__ __forceinline__ double3 spin_rotation(double3 H, double3 s, double dt) {
    return rot_apply(rot_coef(H, dt), s);
}

// Landau field plus the exchange correction (calculate_spin_CPU.cpp:127-136)
__device__ __forceinline__ double3 landau_field(const double L[4], double sumJ, double3 x) {
    double s_sq = x.x * x.x + x.y * x.y + x.z * x.z;
    double c = -(2.0 * L[0] + 4.0 * L[1] * s_sq + 6.0 * L[2] * (s_sq * s_sq) +
                 8.0 * L[3] * (s_sq * s_sq * s_sq));
    double3 HL = make_double3(c * x.x, c * x.y, c * x.z);
    if (s_sq > 0.0) {
        double k = -sumJ * rsqrt(s_sq);
        HL.x += k * x.x; HL.y += k * x.y; HL.z += k * x.z;
    }
    return HL;
}

// One visit with field H (and sum_j J |s_j|): NVE rotation, or the five-part
// Langevin Heisenberg-Landau scheme with the noise increment dS (eV/s, the
// normals times sqrt(2 T gamma_S / dt)).  Returns the new spin; HL receives
// the last Landau field.
__device__ __forceinline__ double3 spin_integrate_dS(const Dev& D, double3 s, double3 H,
                                                     double sumJ, double rho, double3 dS,
                                                     double dt, double3& HL) {
    HL = make_double3(0.0, 0.0, 0.0);
    if (!D.spinlang) return spin_rotation(H, s, dt);
    if (!D.hc) sumJ = 0.0;   // the exchange correction of the Landau field is SLDHL's
    double dt_half = dt / 2.0, dt_quad = dt / 4.0, g = D.gamma_S_HL;
    double L[4];
    for (int k = 0; k < 4; ++k) L[k] = interp_const(D.landau[k], rho, D.inv_rho);
    const RotCoef rc = rot_coef(H, dt_half);
    s = rot_apply(rc, s);                                               // part 1
    HL = landau_field(L, sumJ, s);                                      // part 2
    double a = g * dt_quad;
    double3 t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    HL = landau_field(L, sumJ, t);
    a = g * dt_half;
    s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    s = make_double3(s.x + dt * dS.x, s.y + dt * dS.y, s.z + dt * dS.z);    // part 3
    HL = landau_field(L, sumJ, s);                                      // part 4
    a = g * dt_quad;
    t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    HL = landau_field(L, sumJ, t);
    a = g * dt_half;
    s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    return rot_apply(rc, s);                                            // part 5
}

// The noise increment of one visit at temperature T (eV): the normals xi
// scaled by sqrt(2 T gamma_S_HL / dt) (calculate_spin_CPU.cpp:157-167), or
// for the Heisenberg scheme the random field sqrt(2 T gamma_S_H hbar / dt) xi
// (calculate_spin_CPU.cpp:78-87).
__device__ __forceinline__ double3 spin_noise_dS(const Dev& D, double T, double3 xi, double dt) {
    double amp = D.hint ? sqrt(2.0 * T * D.gamma_S_H * SLD_HBAR / dt) : sqrt(2.0 * T * D.gamma_S_HL / dt);
    return make_double3(amp * xi.x, amp * xi.y, amp * xi.z);
}

// The damped precession of a spin of length s0 about H over a half step, in
// closed form (calculate_spin_CPU.cpp:55-74): ca, sa = cos, sin of the
// precession angle, eb = the damping factor exp(-|H| s0 gamma_S_H dt/2 / hbar).
__device__ __forceinline__ double3 llg_half(double3 s, double3 H, double H0, double s0, double ca,
                                           double sa, double eb) {
    const double e2b = eb * eb;
    double3 x = make_double3(s.y * H.z - s.z * H.y, s.z * H.x - s.x * H.z, s.x * H.y - s.y * H.x);
    double n = 0.0;
    if (s0 > 0.0 && H0 > 0.0) n = (s.x * H.x + s.y * H.y + s.z * H.z) / s0 / H0;
    double den = (1e0 + e2b + n * (1e0 - e2b)) * H0;
    double fac = (1e0 - e2b + n * (1e0 + e2b - 2e0 * ca * eb)) * s0;
    double a = 2e0 * ca * eb * H0, b = 2e0 * sa * eb;
    return make_double3((a * s.x + b * x.x + fac * H.x) / den, (a * s.y + b * x.y + fac * H.y) / den,
                        (a * s.z + b * x.z + fac * H.z) / den);
}

// One visit of the Heisenberg Hamiltonians (SDH, SLDH): NVE rotation, or the
// three-part Langevin scheme (calculate_spin_CPU.cpp:49-101; P.-W. Ma and
// S. L. Dudarev, Phys. Rev. B 83, 134418 (2011)): damped precession for dt/2,
// a rotation about the random field dh for dt, damped precession for dt/2.
// s0 is the spin's stored length.
__device__ __forceinline__ double3 spin_integrate_H(const Dev& D, double3 s, double s0, double3 H,
                                                    double3 dh, double dt) {
    if (!D.spinlang) return spin_rotation(H, s, dt);
    const double dt_half = dt / 2e0;
    const double H0 = sqrt(H.x * H.x + H.y * H.y + H.z * H.z);
    double sa, ca;
    sincos(H0 * (dt_half / SLD_HBAR), &sa, &ca);
    const double eb = exp(-H0 * s0 * D.gamma_S_H * (dt_half / SLD_HBAR));
    s = llg_half(s, H, H0, s0, ca, sa, eb);
    s = spin_rotation(dh, s, dt);
    return llg_half(s, H, H0, s0, ca, sa, eb);
}
