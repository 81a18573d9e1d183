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
// consecutive knots each is one cubic, written in t = r - base with the base
// stored as FP32.  Interval m holds r with m knots <= r (knots ascending); its
// base is knot m-1 (knot 0 for m = 0); the last interval is zero.
//
// FP32 table (the split form), kCubicFloats floats: pair knots [0,8), then
// the pair's 9 intervals as 8-float blocks from kPairIv, density knots at
// kDensKnots (6 and two unused), then the density's 7 intervals from
// kDensIv.  A block is {c0, c1, c2, c3, base, upper knot (1e30 for the last
// interval), amplitude a of the knot below and of the knot above (0 where
// there is none)} for the terms a (k - r)^3 whose seven-point derivative
// differs from the exact one near their knot.  Every block starts on 32
// bytes.
//
// FP64 table (the analytic FP64 form), kCubicDoubles doubles: pair knots
// [0,8), pair coefficients [8,44) (c0..c3 per interval), density knots
// [44,50), density coefficients [50,78).
constexpr int kCubicFloats = 144;
constexpr int kPairIv = 8, kDensKnots = 80, kDensIv = 88;
constexpr int kCubicDoubles = 78;
void pot_cubic_tables(float out[kCubicFloats], double out64[kCubicDoubles]);

}  // namespace sld
