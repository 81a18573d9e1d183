// Host-built potential tables (see potential.cpp).
#pragma once
#include <vector>

namespace sld {

constexpr int kNInput = 1000000;
enum { kF = 0, kdF, kf, kdf, kPhi, kdPhi, kJ, kdJ, kTabCount };

struct Tables {
    std::vector<double> t[kTabCount];
    double rmax = 0, rhomax = 0, inv_r = 0, inv_rho = 0;
    double landau[4] = {0, 0, 0, 0};
};

void build_tables(Tables& T, double rmax);
double pot_F(double rho);
double pot_f(double r);
double pot_phi(double r);
double pot_J(double r);
// The 36 parameters of the forms above, in the order of the adjoint's
// parameter vector: F's a, b; f's 6 coefficients, 6 knots; phi's 8
// coefficients, 8 knots; J's amplitude and range; Landau A, B, C, D
void pot_theta(double out[36]);
// Hermite data of the pair term's 1.8-2.0 A join: y, y', y'' of the ZBL core
// at 1.8 A and of the cubic knots at 2.0 A, then the ZBL screening length
void pot_join_data(double out[7]);

// Piecewise-cubic form of the DD05 pair term (r > 2 A) and density: between
// consecutive knots each is one cubic, written here in t = r - base with the
// base stored as FP32.  Layout (floats): pair knots [0,8), pair coefficients
// [8,44) (9 intervals x c0..c3), density knots [44,50), density coefficients
// [50,78) (7 intervals).  Interval m holds r with m knots <= r; its base is
// knot m-1 (knot 0 for m = 0); the last interval is zero.  Then the amplitude
// a_i of each knot's term a_i (k_i - r)^3, in the same ascending knot order:
// pair [78,86), density [86,92) (the seven-point derivative near a knot needs
// the one term that changes form there).
constexpr int kCubicFloats = 92;
void pot_cubic_tables(float out[kCubicFloats], double out64[kCubicFloats]);

}  // namespace sld
