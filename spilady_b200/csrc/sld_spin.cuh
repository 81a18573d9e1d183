// Spin integrator of one visit (calculate_spin_CPU.cpp:33-199), FP64.
#pragma once
#include "sld_common.cuh"

// core_ds_CPU.cpp:90-127: exact rotation of s about -Heff/hbar by |w| dt
__device__ __forceinline__ double3 spin_rotation(double3 H, double3 s, double dt) {
    double3 w = make_double3(H.x / -SLD_HBAR, H.y / -SLD_HBAR, H.z / -SLD_HBAR);
    double w0 = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
    if (w0 > 0.0) w = make_double3(w.x / w0, w.y / w0, w.z / w0);
    else w = make_double3(0.0, 0.0, 0.0);
    double w12 = w.x * w.y, w23 = w.y * w.z, w13 = w.x * w.z;
    double w1s = w.x * w.x, w2s = w.y * w.y, w3s = w.z * w.z;
    double A, cw;
    sincos(w0 * dt, &A, &cw);
    double B = 1.0 - cw;
    double3 o;
    o.x = s.x + (s.x * B * (-w2s - w3s) + s.y * (B * w12 - A * w.z) + s.z * (A * w.y + B * w13));
    o.y = s.y + (s.y * B * (-w1s - w3s) + s.z * (B * w23 - A * w.x) + s.x * (A * w.z + B * w12));
    o.z = s.z + (s.z * B * (-w1s - w2s) + s.x * (B * w13 - A * w.y) + s.y * (A * w.x + B * w23));
    return o;
}

// Landau field plus the exchange correction (calculate_spin_CPU.cpp:127-136)
__device__ __forceinline__ double3 landau_field(const double L[4], double sumJ, double3 x) {
    double s_sq = x.x * x.x + x.y * x.y + x.z * x.z;
    double c = -(2.0 * L[0] + 4.0 * L[1] * s_sq + 6.0 * L[2] * (s_sq * s_sq) +
                 8.0 * L[3] * (s_sq * s_sq * s_sq));
    double3 HL = make_double3(c * x.x, c * x.y, c * x.z);
    double s0 = sqrt(s_sq);
    if (s0 > 0.0) {
        double k = -sumJ / s0;
        HL.x += k * x.x; HL.y += k * x.y; HL.z += k * x.z;
    }
    return HL;
}

// One visit with field H (and sum_j J |s_j|): NVE rotation, or the five-part
// Langevin Heisenberg-Landau scheme with normal noise xi at temperature T (eV).
// Returns the new spin; HL receives the last Landau field.
__device__ __forceinline__ double3 spin_integrate(const Dev& D, double3 s, double3 H, double sumJ,
                                                  double rho, double T, double3 xi, double dt,
                                                  double3& HL) {
    HL = make_double3(0.0, 0.0, 0.0);
    if (!D.spinlang) return spin_rotation(H, s, dt);
    double dt_half = dt / 2.0, dt_quad = dt / 4.0, g = D.gamma_S_HL;
    double L[4];
    for (int k = 0; k < 4; ++k) L[k] = interp_const(D.landau[k], rho, D.inv_rho);
    s = spin_rotation(H, s, dt_half);                                   // part 1
    HL = landau_field(L, sumJ, s);                                      // part 2
    double a = g * dt_quad;
    double3 t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    HL = landau_field(L, sumJ, t);
    a = g * dt_half;
    s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    double amp = sqrt(2.0 * T * g / dt);                                // part 3
    double3 dS = make_double3(amp * xi.x, amp * xi.y, amp * xi.z);
    s = make_double3(s.x + dt * dS.x, s.y + dt * dS.y, s.z + dt * dS.z);
    HL = landau_field(L, sumJ, s);                                      // part 4
    a = g * dt_quad;
    t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    HL = landau_field(L, sumJ, t);
    a = g * dt_half;
    s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
    return spin_rotation(H, s, dt_half);                                // part 5
}
