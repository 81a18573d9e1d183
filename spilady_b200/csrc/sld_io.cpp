// File formats kept from the reference for drop-in use:
//   variables.in   read_variables.cpp:40-253 (key value pairs, unknown keys
//                  ignored), plus this engine's runtime switches
//   con- files     read_config.cpp:39-116 (atoms configuration)
//   readTe files   map_cells.cpp:33-39,136-150 (electron temperature per cell)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/sld.h"

extern "C" int sld_read_variables(const char* path, sld_params* P) {
    if (!path || !P) return SLD_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SLD_ERR_IO;
    std::string key, val;
    while (in >> key >> val) {
        double v = std::atof(val.c_str());
        int iv = std::atoi(val.c_str());
        if (key == "step") P->step = v;
        else if (key == "temperature") P->temperature = v;
        else if (key == "atmass") P->atmass = v;
        else if (key == "gamma_L_over_mass") P->gamma_L_over_mass = v;
        else if (key == "gamma_S_HL") P->gamma_S_HL = v;
        else if (key == "random_seed") P->random_seed = iv;
        else if (key == "rcut_pot") P->rcut_pot = v;
        else if (key == "rcut_mag") P->rcut_mag = v;
        else if (key == "rcut_max") P->rcut_max = v;
        else if (key == "min_length_link_cell") P->min_length_link_cell = v;
        else if (key == "kappa_e") P->kappa_e = v;
        else if (key == "interval_of_print_out") P->interval_of_print_out = iv;
        // control.h switches, which the reference fixes at compile time
        else if (key == "spinlang") P->spinlang = iv;
        else if (key == "lattlang") P->lattlang = iv;
        else if (key == "eltemp") P->eltemp = iv;
        else if (key == "localcolmot") P->localcolmot = iv;
        else if (key == "renormalizeEnergy") P->renormalize_energy = iv;
        else if (key == "te_mesh") P->te_mesh = iv;
        else if (key == "te_nloop") P->te_nloop = iv;
        else if (key == "precision") P->precision = (val == "split" || iv == 1) ? SLD_SPLIT : SLD_FP64;
        else if (key == "current_device") P->device = iv;
        else if (key == "replica") P->replica = iv;
    }
    return SLD_OK;
}

namespace {

// number of link cells per axis as map_cells.cpp:41-51 computes it
void link_grid(const sld_params& P, int& nx, int& ny, int& nz) {
    const double* d = P.box;
    double ml = P.min_length_link_cell;
    if (P.rcut_max > ml) ml = P.rcut_max + 0.001;
    double a1 = std::sin(std::atan2(d[2], d[1]));
    double a2 = std::sin(std::atan2(d[5], d[3]));
    double a3 = std::sin(std::atan2(d[5], d[4]));
    double ex = std::fmax(ml / a1, ml / a2);
    double ey = std::fmax(ml, ml / a3);
    nx = (int)(d[0] / ex);
    ny = (int)(d[2] / ey);
    nz = (int)(d[5] / ml);
}

}  // namespace

extern "C" int sld_create_from_config(sld_ctx** out, const sld_params* prm, const char* con_path,
                                      const char* te_path) {
    if (!out || !prm || !con_path) return SLD_ERR_ARG;
    std::ifstream in(con_path);
    if (!in) return SLD_ERR_IO;
    long natom = 0;
    double total_time = 0;
    std::string type;
    sld_params P = *prm;
    if (!(in >> natom >> total_time >> type)) return SLD_ERR_IO;
    if (type != "SLDHL") return SLD_ERR_IO;   // read_config.cpp:60-65
    if (!(in >> P.box[0] >> P.box[1] >> P.box[2] >> P.box[3] >> P.box[4] >> P.box[5]))
        return SLD_ERR_IO;
    if (natom <= 0) return SLD_ERR_IO;
    std::vector<double> r(3 * natom), p(3 * natom), s(3 * natom);
    std::string line;
    std::getline(in, line);
    for (long i = 0; i < natom; ++i) {
        if (!std::getline(in, line)) return SLD_ERR_IO;
        std::istringstream ls(line);
        long idx;
        std::string el;
        double v[30];
        if (!(ls >> idx >> el)) return SLD_ERR_IO;
        // r(3) p(3) f(3) stress(6) rho ke pe s(3) s0 Heff_H(3) Heff_L(3) me me0 local_volume
        for (int k = 0; k < 27; ++k)
            if (!(ls >> v[k])) return SLD_ERR_IO;
        for (int k = 0; k < 3; ++k) {
            r[3 * i + k] = v[k];
            p[3 * i + k] = v[3 + k];
            s[3 * i + k] = v[18 + k];
        }
    }
    std::vector<double> te;
    if (te_path && te_path[0]) {
        std::ifstream tin(te_path);
        if (!tin) return SLD_ERR_IO;
        long ncells;
        double tt, dd[6];
        if (!(tin >> ncells >> tt >> dd[0] >> dd[1] >> dd[2] >> dd[3] >> dd[4] >> dd[5]))
            return SLD_ERR_IO;
        int nx, ny, nz;
        if (P.te_mesh > 0) nx = ny = nz = P.te_mesh;
        else link_grid(P, nx, ny, nz);
        if (ncells != (long)nx * ny * nz) return SLD_ERR_IO;
        te.assign(ncells, 0.0);
        for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy)
                for (int iz = 0; iz < nz; ++iz) {
                    double a, b, c, T, Tl, TsR, TsL;
                    if (!(tin >> a >> b >> c >> T >> Tl >> TsR >> TsL)) return SLD_ERR_IO;
                    te[ix + iy * nx + iz * nx * ny] = T;
                }
    }
    return sld_create(out, &P, (int)natom, r.data(), p.data(), s.data(),
                      te.empty() ? nullptr : te.data());
}
