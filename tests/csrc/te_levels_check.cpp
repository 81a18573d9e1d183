// Host check of te_levels (spilady_b200/csrc/sld_host.cpp): the colour sweep
// of core_dTe's C step run in sequence over cells (core_dTe_CPU.cpp:140-175's
// order: groups 0..G-1, then G-1..0) against the same sweep run by levels
// over colour positions, with an update that reads the cell, its energy and
// its six face neighbours as the diffusion update does.  Every level reads
// all its inputs before any task of it writes (a barrier between levels).
// The two must agree bit for bit on every mesh.  Exit status 1 on a
// difference.
#include "sld_host.h"
#include <cstdio>
#include <cmath>
using namespace sld;
// sequential colour sweep in cell space against the level schedule in position space
static double upd(double self, double x, const double* a) {
    double s = 0; for (int j = 0; j < 6; ++j) s += a[j] * (j + 1.5);
    return std::sin(self * 1.3 + 0.1 * s) + 0.01 * x;
}
int main() {
    int sizes[][3] = {{4, 4, 4}, {5, 5, 5}, {6, 6, 6}, {7, 5, 6}, {16, 16, 16}, {3, 4, 5}, {11, 6, 7}};
    int bad = 0;
    for (auto& sz : sizes) {
        int nx = sz[0], ny = sz[1], nz = sz[2], n = nx * ny * nz;
        std::vector<int> gs, gc, ls; std::vector<unsigned short> tk, nbp;
        int G = colour_grid(nx, ny, nz, gs, gc);
        int L = te_levels(nx, ny, nz, gs, gc, ls, tk, nbp);
        std::vector<double> T(n), X(n);
        for (int c = 0; c < n; ++c) { T[c] = std::cos(c * 0.7); X[c] = c * 0.01; }
        std::vector<double> T2(n), X2(n);   // position space
        for (int m = 0; m < n; ++m) { T2[m] = T[gc[m]]; X2[m] = X[gc[m]]; }
        // sequential
        for (int pass = 0; pass < 2; ++pass)
            for (int gg = 0; gg < G; ++gg) {
                int g = pass == 0 ? gg : G - 1 - gg;
                for (int m = gs[g]; m < gs[g + 1]; ++m) {
                    int c = gc[m], x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
                    int nb[6] = {(x + 1) % nx + (y + z * ny) * nx, (x + nx - 1) % nx + (y + z * ny) * nx,
                                 x + ((y + 1) % ny + z * ny) * nx, x + ((y + ny - 1) % ny + z * ny) * nx,
                                 x + (y + ((z + 1) % nz) * ny) * nx, x + (y + ((z + nz - 1) % nz) * ny) * nx};
                    double a[6]; for (int j = 0; j < 6; ++j) a[j] = T[nb[j]];
                    X[c] = X[c] + a[0]; T[c] = upd(T[c], X[c], a);
                }
            }
        // levels: all tasks of a level read first, then write (a barrier between levels)
        for (int l = 0; l < L; ++l) {
            std::vector<std::pair<int, std::pair<double,double>>> out;
            for (int e = ls[l]; e < ls[l + 1]; ++e) {
                int t = tk[e], m = t & 0x7fff;
                double a[6]; for (int j = 0; j < 6; ++j) a[j] = T2[nbp[8 * m + j]];
                double x = X2[m] + a[0], tt = upd(T2[m], x, a);
                if (t & 0x8000) { x = x + a[0]; tt = upd(tt, x, a); }
                out.push_back({m, {tt, x}});
            }
            for (auto& o : out) { T2[o.first] = o.second.first; X2[o.first] = o.second.second; }
        }
        int diff = 0;
        for (int m = 0; m < n; ++m) diff += (T2[m] != T[gc[m]]) || (X2[m] != X[gc[m]]);
        printf("%dx%dx%d G=%d L=%d tasks=%zu diff=%d\n", nx, ny, nz, G, L, tk.size(), diff);
        bad += diff;
    }
    return bad != 0;
}
