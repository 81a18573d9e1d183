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

}  // namespace sld
