// Potential tables for bcc Fe, built on the host at context creation.
//
// Functional forms and published parameters: the DD05 embedded-atom
// potential (Dudarev & Derlet 2005) as DD05.cpp:6-164 states it, the Fe
// exchange J(r) = 0.870 (1 - r/3.75)^3 and the constant Landau coefficients
// of JijFe.cpp:5-43.  Tables and derivatives follow potential_CPU.cpp:61-170:
// 10^6 points at x_n = (n+1) max / 10^6, derivatives by the seven-point
// central difference with dx = x/1000.  The arithmetic of each entry follows
// the reference's so the tables agree with its own to the last bit wherever
// the dynamics reads them (the pair term between 1.8 and 2.0 A, reached only
// in close collisions, is the same quintic written in Hermite form).
#include <cmath>
#include <thread>
#include <vector>

#include "potential.h"

namespace sld {

static const double kEmbA = 4.100199340884814, kEmbB = 1.565647547483517;
static const double kDensA[6] = {0.9332056681088162, -1.162558782567700, -0.3502026949249225,
                                 0.4287820835430028, 4.907925057809273,  -5.307049068415304};
static const double kDensK[6] = {3.0, 2.8666666666666666, 2.7333333333333333, 2.6, 2.4, 2.3};
static const double kJA = 0.870, kJRC = 3.75;

static double emb_F(double rho) {
    const double a = kEmbA, b = kEmbB;
    if (rho >= 1e0) return -a * std::sqrt(rho);
    return -a * std::sqrt(rho) - b / std::log(2e0) * (1e0 - std::sqrt(rho)) * std::log(2e0 - rho);
}

static double dens_f(double r) {
    const double* a = kDensA;
    const double* k = kDensK;
    double f = 0e0;
    for (int i = 0; i < 6; ++i)
        if (r < k[i]) f += a[i] * std::pow(k[i] - r, 3);
    return f;
}

static double zbl(double r) {
    const double z = 26e0, abohr = 0.52917720859e0;
    double as = 0.88535e0 * abohr / (2e0 * std::pow(z, 0.23));
    double x = r / as;
    double v = 0.1818e0 * std::exp(-3.2 * x) + 0.5099e0 * std::exp(-0.9423 * x) +
               0.2802e0 * std::exp(-0.4029 * x) + 0.02817e0 * std::exp(-0.2016 * x);
    return z * z * 14.3992 * v / r;
}

static const double kPV[8] = {-0.1960674387419232, 0.3687525935422963, -1.505333614924853,
                              4.948907078156191,   -4.894613262753399, 3.468897724782442,
                              -1.792218099820337,  80.22069592246987};
static const double kPK[8] = {4.1, 3.8, 3.5, 3.2, 2.9, 2.6, 2.4, 2.3};

static double pair_knots(double r, int deriv) {
    double v = 0e0;
    for (int i = 0; i < 8; ++i) {
        if (r < kPK[i]) {
            double u = kPK[i] - r;
            if (deriv == 0) v += kPV[i] * std::pow(u, 3);
            else if (deriv == 1) v -= 3e0 * kPV[i] * u * u;
            else v += 6e0 * kPV[i] * u;
        }
    }
    return v;
}

static double pair_phi(double r) {
    const double x1 = 1.8, x2 = 2.0;
    if (r <= x1) return zbl(r);
    if (r <= x2) {
        const double h = 1e-7;
        double y1 = zbl(x1);
        double d1 = (zbl(x1 + h) - zbl(x1 - h)) / 2e-7;
        double c1 = (zbl(x1 + h) + zbl(x1 - h) - 2e0 * zbl(x1)) / std::pow(h, 2);
        double y2 = pair_knots(x2, 0), d2 = pair_knots(x2, 1), c2 = pair_knots(x2, 2);
        double w = x2 - x1, t = (r - x1) / w;
        double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
        double h00 = 1 - 10 * t3 + 15 * t4 - 6 * t5, h01 = 10 * t3 - 15 * t4 + 6 * t5;
        double h10 = t - 6 * t3 + 8 * t4 - 3 * t5, h11 = -4 * t3 + 7 * t4 - 3 * t5;
        double h20 = 0.5 * t2 - 1.5 * t3 + 1.5 * t4 - 0.5 * t5;
        double h21 = 0.5 * t3 - t4 + 0.5 * t5;
        return h00 * y1 + h01 * y2 + w * (h10 * d1 + h11 * d2) + w * w * (h20 * c1 + h21 * c2);
    }
    return pair_knots(r, 0);
}

static double exch_J(double r) {
    const double A = kJA, rc = kJRC;
    double J = 0e0;
    if (r < rc) J = A * std::pow(1.0 - r / rc, 3);
    return J;
}

static double deriv7(double (*fn)(double), double x) {
    double dx = x / 1000e0;
    double p1 = fn(x + dx), m1 = fn(x - dx);
    double p2 = fn(x + 2 * dx), m2 = fn(x - 2 * dx);
    double p3 = fn(x + 3 * dx), m3 = fn(x - 3 * dx);
    return (45e0 * (p1 - m1) - 9e0 * (p2 - m2) + (p3 - m3)) / (60e0 * dx);
}

const double kLandau[4] = {-0.744824, 0.345295, -0.00790205, 0e0};

void build_tables(Tables& T, double rmax) {
    double rhomax = 2e0 * dens_f(1e0);
    if (rhomax < 1000e0) rhomax = 1000e0;
    const double finput = (double)kNInput;
    T.rmax = rmax;
    T.rhomax = rhomax;
    T.inv_r = finput / rmax;
    T.inv_rho = finput / rhomax;
    for (int k = 0; k < kTabCount; ++k) T.t[k].assign(kNInput, 0.0);
    unsigned nth = std::thread::hardware_concurrency();
    if (nth == 0) nth = 4;
    if (nth > 16) nth = 16;
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nth; ++w) {
        pool.emplace_back([&T, rmax, rhomax, w, nth]() {
            for (int n = (int)w; n < kNInput; n += (int)nth) {
                double r = rmax / (double)kNInput * (double)(n + 1);
                double rho = rhomax / (double)kNInput * (double)(n + 1);
                T.t[kF][n] = emb_F(rho);
                T.t[kdF][n] = deriv7(emb_F, rho);
                T.t[kf][n] = dens_f(r);
                T.t[kdf][n] = deriv7(dens_f, r);
                T.t[kPhi][n] = pair_phi(r);
                T.t[kdPhi][n] = deriv7(pair_phi, r);
                T.t[kJ][n] = exch_J(r);
                T.t[kdJ][n] = deriv7(exch_J, r);
            }
        });
    }
    for (auto& t : pool) t.join();
    for (int k = 0; k < 4; ++k) T.landau[k] = kLandau[k];
}

// analytic forms for callers that evaluate the potential directly
double pot_F(double rho) { return emb_F(rho); }
double pot_f(double r) { return dens_f(r); }
double pot_phi(double r) { return pair_phi(r); }
double pot_J(double r) { return exch_J(r); }

void pot_theta(double o[36]) {
    o[0] = kEmbA;
    o[1] = kEmbB;
    for (int i = 0; i < 6; ++i) { o[2 + i] = kDensA[i]; o[8 + i] = kDensK[i]; }
    for (int i = 0; i < 8; ++i) { o[14 + i] = kPV[i]; o[22 + i] = kPK[i]; }
    o[30] = kJA;
    o[31] = kJRC;
    for (int i = 0; i < 4; ++i) o[32 + i] = kLandau[i];
}

void pot_join_data(double o[7]) {
    const double x1 = 1.8, x2 = 2.0, h = 1e-7;
    o[0] = zbl(x1);
    o[1] = (zbl(x1 + h) - zbl(x1 - h)) / 2e-7;
    o[2] = (zbl(x1 + h) + zbl(x1 - h) - 2e0 * zbl(x1)) / std::pow(h, 2);
    o[3] = pair_knots(x2, 0);
    o[4] = pair_knots(x2, 1);
    o[5] = pair_knots(x2, 2);
    o[6] = 0.88535e0 * 0.52917720859e0 / (2e0 * std::pow(26e0, 0.23));
}

// the cubics of sum_i a_i (k_i - r)^3 for r < k_i (knots given descending)
static void cubic_pieces(const double* a, const double* k, int n, float* K, float* blocks,
                         double* K64, double* C64) {
    std::vector<int> ord(n);   // ascending
    for (int i = 0; i < n; ++i) ord[i] = n - 1 - i;
    for (int i = 0; i < n; ++i) {
        K[i] = (float)k[ord[i]];
        K64[i] = (double)K[i];
    }
    for (int m = 0; m <= n; ++m) {
        double c[4] = {0, 0, 0, 0};
        const double base = (double)(m == 0 ? K[0] : K[m - 1]);
        if (m < n) {
            for (int q = m; q < n; ++q) {   // knots above the interval are active
                const int i = ord[q];
                const double dl = k[i] - base;
                c[0] += a[i] * dl * dl * dl;
                c[1] += -3e0 * a[i] * dl * dl;
                c[2] += 3e0 * a[i] * dl;
                c[3] += -a[i];
            }
        }
        float* b = blocks + 8 * m;
        for (int q = 0; q < 4; ++q) {
            b[q] = (float)c[q];
            C64[4 * m + q] = c[q];
        }
        b[4] = (float)base;
        b[5] = m < n ? K[m] : 1e30f;
        b[6] = m > 0 ? (float)a[ord[m - 1]] : 0.f;
        b[7] = m < n ? (float)a[ord[m]] : 0.f;
    }
}

void pot_cubic_tables(float out[kCubicFloats], double o64[kCubicDoubles]) {
    static const double da[6] = {0.9332056681088162, -1.162558782567700, -0.3502026949249225,
                                 0.4287820835430028, 4.907925057809273, -5.307049068415304};
    static const double dk[6] = {3.0, 2.8666666666666666, 2.7333333333333333, 2.6, 2.4, 2.3};
    for (int k = 0; k < kCubicFloats; ++k) out[k] = 0.f;
    for (int k = 0; k < kCubicDoubles; ++k) o64[k] = 0.0;
    cubic_pieces(kPV, kPK, 8, out, out + kPairIv, o64, o64 + 8);
    cubic_pieces(da, dk, 6, out + kDensKnots, out + kDensIv, o64 + 44, o64 + 50);
}

}  // namespace sld
