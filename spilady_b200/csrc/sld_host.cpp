// Host-side geometry and set-up (see sld_host.h).
#include "sld_host.h"

#include <algorithm>
#include <cmath>

namespace sld {

void host_periodic(const HostGeom& G, double& x, double& y, double& z) {
    const double* I = G.inv;
    const double* d = G.d;
    double qx = I[0] * x + I[1] * y + I[3] * z;
    double qy = I[2] * y + I[4] * z;
    double qz = I[5] * z;
    int idx = 0;
    if (qx < 0e0 || qx >= 1e0) { qx -= (int)qx; ++idx; }
    if (qy < 0e0 || qy >= 1e0) { qy -= (int)qy; ++idx; }
    if (qz < 0e0 || qz >= 1e0) { qz -= (int)qz; ++idx; }
    if (idx > 0) {
        x = d[0] * qx + d[1] * qy + d[3] * qz;
        y = d[2] * qy + d[4] * qz;
        z = d[5] * qz;
    }
}

// the 26 neighbour offsets in the order of map_cells.cpp:96-121
static const int kNbrOff[26][3] = {
    {1, 0, 0},   {1, 1, 0},  {0, 1, 0},   {-1, 1, 0},  {1, 0, -1},  {1, 1, -1}, {0, 1, -1},
    {-1, 1, -1}, {1, 0, 1},  {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {0, 0, 1},  {-1, 0, 0},
    {0, -1, 0},  {0, 0, -1}, {1, -1, 0},  {-1, -1, 0}, {-1, 0, 1},  {-1, 0, -1}, {0, -1, 1},
    {0, -1, -1}, {1, -1, 1}, {1, -1, -1}, {-1, -1, 1}, {-1, -1, -1}};

// neighbour k of cell (ix, iy, iz) in the order of map_cells.cpp:96-121
static int nbr(int nx, int ny, int nz, int ix, int iy, int iz, int k) {
    const int (&O)[26][3] = kNbrOff;
    int x = (ix + O[k][0] + nx) % nx, y = (iy + O[k][1] + ny) % ny, z = (iz + O[k][2] + nz) % nz;
    return x + y * nx + z * nx * ny;
}

int colour_grid(int nx, int ny, int nz, std::vector<int>& gstart, std::vector<int>& gcells) {
    int nc = nx * ny * nz;
    std::vector<int> type(nc, 0);
    gcells.clear();
    gstart.assign(1, 0);
    int left = nc;
    while (left > 0) {
        for (int i = 0; i < nc; ++i) {
            if (type[i] != 0) continue;
            gcells.push_back(i);
            type[i] = 1;
            --left;
            int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
            for (int k = 0; k < 26; ++k) {
                int j = nbr(nx, ny, nz, ix, iy, iz, k);
                if (type[j] != 1) type[j] = -1;
            }
        }
        gstart.push_back((int)gcells.size());
        for (int i = 0; i < nc; ++i)
            if (type[i] == -1) type[i] = 0;
    }
    return (int)gstart.size() - 1;
}

int te_levels(int nx, int ny, int nz, const std::vector<int>& gstart,
              const std::vector<int>& gcells, std::vector<int>& lstart,
              std::vector<unsigned short>& tasks, std::vector<unsigned short>& nbp) {
    lstart.clear();
    tasks.clear();
    nbp.clear();
    const int nc = nx * ny * nz;
    if (nc >= 0x8000) return 0;
    const int G = (int)gstart.size() - 1;
    std::vector<int> pos(nc);
    for (int m = 0; m < nc; ++m) pos[gcells[m]] = m;
    auto nb6 = [&](int c, int* nb) {
        const int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        nb[0] = (x + 1) % nx + (y + z * ny) * nx;
        nb[1] = (x + nx - 1) % nx + (y + z * ny) * nx;
        nb[2] = x + ((y + 1) % ny + z * ny) * nx;
        nb[3] = x + ((y + ny - 1) % ny + z * ny) * nx;
        nb[4] = x + (y + ((z + 1) % nz) * ny) * nx;
        nb[5] = x + (y + ((z + nz - 1) % nz) * ny) * nx;
    };
    nbp.assign(8 * (size_t)nc, 0);
    for (int m = 0; m < nc; ++m) {
        int nb[6];
        nb6(gcells[m], nb);
        for (int j = 0; j < 6; ++j) nbp[8 * (size_t)m + j] = (unsigned short)pos[nb[j]];
    }
    std::vector<int> last(nc, 0);      // level of the cell's latest update (0: none yet)
    std::vector<int> at(nc, -1);       // that update's index in its level's list
    std::vector<std::vector<unsigned short>> lv;
    for (int pass = 0; pass < 2; ++pass)
        for (int gg = 0; gg < G; ++gg) {
            const int g = pass == 0 ? gg : G - 1 - gg;
            for (int m = gstart[g]; m < gstart[g + 1]; ++m) {
                const int c = gcells[m];
                int nb[6];
                nb6(c, nb);
                int l = last[c];
                for (int j : nb)
                    if (j != c) l = std::max(l, last[j]);
                if (last[c] > 0 && l == last[c]) {   // nothing read changed since: same task
                    lv[l - 1][at[c]] |= 0x8000;
                    continue;
                }
                ++l;
                if ((int)lv.size() < l) lv.resize(l);
                at[c] = (int)lv[l - 1].size();
                lv[l - 1].push_back((unsigned short)m);
                last[c] = l;
            }
        }
    lstart.push_back(0);
    for (const auto& v : lv) {
        tasks.insert(tasks.end(), v.begin(), v.end());
        lstart.push_back((int)tasks.size());
    }
    return (int)lv.size();
}

void box_derived(HostGeom& G) {
    const double* d = G.d;
    // vec_utils_CPU.cpp:135-148
    G.inv[0] = 1e0 / d[0];
    G.inv[1] = -d[1] / (d[0] * d[2]);
    G.inv[2] = 1e0 / d[2];
    G.inv[3] = (d[1] * d[4] - d[2] * d[3]) / (d[0] * d[2] * d[5]);
    G.inv[4] = -d[4] / (d[2] * d[5]);
    G.inv[5] = 1e0 / d[5];
    G.box_len[0] = std::fabs(d[0]);
    G.box_len[1] = std::sqrt(d[1] * d[1] + d[2] * d[2]);
    G.box_len[2] = std::sqrt(d[3] * d[3] + d[4] * d[4] + d[5] * d[5]);
    G.box_volume = d[0] * d[2] * d[5];
}

int setup_geometry(const sld_params& P, int natom, const std::vector<double>& r, HostGeom& G,
                   std::vector<int>& id_of_slot, std::vector<int>& slot_of_id) {
    const double* d = P.box;
    for (int k = 0; k < 6; ++k) G.d[k] = d[k];
    box_derived(G);
    G.rcut_max = P.rcut_max;
    G.min_len = P.min_length_link_cell;
    if (G.rcut_max > G.min_len) G.min_len = G.rcut_max + 0.001;   // read_variables.cpp:262
    // map_cells.cpp:41-61
    double a1 = std::sin(std::atan2(d[2], d[1]));
    double a2 = std::sin(std::atan2(d[5], d[3]));
    double a3 = std::sin(std::atan2(d[5], d[4]));
    double ex = std::max(G.min_len / a1, G.min_len / a2);
    double ey = std::max(G.min_len, G.min_len / a3);
    double ez = G.min_len;
    G.nx = (int)(d[0] / ex);
    G.ny = (int)(d[2] / ey);
    G.nz = (int)(d[5] / ez);
    if (G.nx < 3 || G.ny < 3 || G.nz < 3) return SLD_ERR_GEOMETRY;
    G.ncells = G.nx * G.ny * G.nz;
    if (P.te_mesh > 0) {
        G.tx = G.ty = G.tz = P.te_mesh;
    } else {
        G.tx = G.nx; G.ty = G.ny; G.tz = G.nz;
    }
    G.nte = G.tx * G.ty * G.tz;
    G.ngroups = colour_grid(G.nx, G.ny, G.nz, G.gstart, G.gcells);
    if (P.te_mesh > 0) {
        G.te_ngroups = colour_grid(G.tx, G.ty, G.tz, G.te_gstart, G.te_gcells);
    } else {
        G.te_ngroups = G.ngroups;
        G.te_gstart = G.gstart;
        G.te_gcells = G.gcells;
    }
    G.te_nlevels = te_levels(G.tx, G.ty, G.tz, G.te_gstart, G.te_gcells, G.te_lstart, G.te_ltasks,
                             G.te_lnb);
    // initial_links_CPU (links_CPU.cpp:33-83): wrap, bin; each cell's list
    // holds its atoms in descending index order
    std::vector<int> cell(natom);
    std::vector<int> count(G.ncells + 1, 0);
    for (int i = 0; i < natom; ++i) {
        double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
        host_periodic(G, x, y, z);
        double qx = G.inv[0] * x + G.inv[1] * y + G.inv[3] * z;
        double qy = G.inv[2] * y + G.inv[4] * z;
        double qz = G.inv[5] * z;
        int lx = std::min(std::max((int)(qx * G.nx), 0), G.nx - 1);
        int ly = std::min(std::max((int)(qy * G.ny), 0), G.ny - 1);
        int lz = std::min(std::max((int)(qz * G.nz), 0), G.nz - 1);
        cell[i] = lx + ly * G.nx + lz * G.nx * G.ny;
        ++count[cell[i] + 1];
    }
    for (int c = 0; c < G.ncells; ++c) count[c + 1] += count[c];
    id_of_slot.assign(natom, 0);
    slot_of_id.assign(natom, 0);
    std::vector<int> fill(G.ncells, 0);
    for (int i = natom - 1; i >= 0; --i) {
        int c = cell[i];
        int s = count[c] + fill[c]++;
        id_of_slot[s] = i;
        slot_of_id[i] = s;
    }
    return SLD_OK;
}

}  // namespace sld
