/*
 * Test infrastructure only: the potential of the reference's "param" build
 * (oracle/ref/build.sh), used to finite-difference the reference's own CPU
 * code in the 36 parameters of its potential.  It replaces DD05.cpp and
 * JijFe.cpp at link time with the same functional forms, written here, whose
 * constants are read from theta.in in the working directory (36 numbers, the
 * order of sld_adjoint_theta_default):
 *   F(rho) = -a sqrt(rho) - [rho < 1] b/ln2 (1 - sqrt(rho)) ln(2 - rho)
 *   f(r)   = sum_k a_k (r_k - r)^3 for r < r_k                  (6 terms)
 *   phi(r) = sum_k V_k (r_k - r)^3 for r < r_k, r > 2 A         (8 terms);
 *            the ZBL screened Coulomb term below 1.8 A and the quintic with
 *            matched value, slope and curvature between 1.8 and 2.0 A
 *            (the ZBL end's slope and curvature by central differences of
 *            step 1e-7, as the reference forms them)
 *   J(r)   = A (1 - r/rc)^3 for r < rc
 *   Landau A, B, C, D constant in rho
 * (DD05: Dudarev and Derlet, J. Phys.: Condens. Matter 17, 7097 (2005).)
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>

static double g_th[36];
static bool g_loaded = false;

static const double* theta() {
    if (!g_loaded) {
        FILE* f = std::fopen("theta.in", "r");
        if (!f) {
            std::fprintf(stderr, "param_pot: theta.in missing\n");
            std::exit(2);
        }
        for (int k = 0; k < 36; ++k)
            if (std::fscanf(f, "%lf", &g_th[k]) != 1) {
                std::fprintf(stderr, "param_pot: theta.in short\n");
                std::exit(2);
            }
        std::fclose(f);
        g_loaded = true;
    }
    return g_th;
}

double bigf_gen(double rho) {
    const double* t = theta();
    double v = -t[0] * std::sqrt(rho);
    if (rho < 1e0) v -= t[1] / std::log(2e0) * (1e0 - std::sqrt(rho)) * std::log(2e0 - rho);
    return v;
}

double smallf_gen(double r) {
    const double* t = theta();
    double v = 0e0;
    for (int k = 0; k < 6; ++k)
        if (r < t[8 + k]) v += t[2 + k] * std::pow(t[8 + k] - r, 3);
    return v;
}

static double zbl(double r) {
    const double z = 26e0, abohr = 0.52917720859e0;
    const double as = 0.88535e0 * abohr / (2e0 * std::pow(z, 0.23));
    const double x = r / as;
    double s = 0.1818e0 * std::exp(-3.2 * x) + 0.5099e0 * std::exp(-0.9423 * x) +
               0.2802e0 * std::exp(-0.4029 * x) + 0.02817e0 * std::exp(-0.2016 * x);
    return z * z * 14.3992 * s / r;
}

// the knot cubics and their first two derivatives at r
static void knots(double r, double& v, double& d1, double& d2) {
    const double* t = theta();
    v = d1 = d2 = 0e0;
    for (int k = 0; k < 8; ++k)
        if (r < t[22 + k]) {
            double u = t[22 + k] - r;
            v += t[14 + k] * std::pow(u, 3);
            d1 -= 3e0 * t[14 + k] * u * u;
            d2 += 6e0 * t[14 + k] * u;
        }
}

double pair_gen(double r) {
    const double x1 = 1.8, x2 = 2.0;
    if (r <= x1) return zbl(r);
    double v, d1, d2;
    if (r > x2) {
        knots(r, v, d1, d2);
        return v;
    }
    const double e = 1e-7;
    double y1 = zbl(x1), p1 = (zbl(x1 + e) - zbl(x1 - e)) / 2e-7;
    double c1 = (zbl(x1 + e) + zbl(x1 - e) - 2e0 * zbl(x1)) / (e * e);
    knots(x2, v, d1, d2);
    // quintic with these end values, slopes and curvatures, in Hermite form
    const double h = x2 - x1, s = (r - x1) / h;
    const double s2 = s * s, s3 = s2 * s, s4 = s3 * s, s5 = s4 * s;
    return y1 * (1 - 10 * s3 + 15 * s4 - 6 * s5) + h * p1 * (s - 6 * s3 + 8 * s4 - 3 * s5) +
           h * h * c1 * (0.5 * s2 - 1.5 * s3 + 1.5 * s4 - 0.5 * s5) +
           v * (10 * s3 - 15 * s4 + 6 * s5) + h * d1 * (-4 * s3 + 7 * s4 - 3 * s5) +
           h * h * d2 * (0.5 * s3 - s4 + 0.5 * s5);
}

double Jij_gen(double r) {
    const double* t = theta();
    if (r < t[31]) return t[30] * std::pow(1.0 - r / t[31], 3);
    return 0e0;
}

double LandauA_gen(double) { return theta()[32]; }
double LandauB_gen(double) { return theta()[33]; }
double LandauC_gen(double) { return theta()[34]; }
double LandauD_gen(double) { return theta()[35]; }
