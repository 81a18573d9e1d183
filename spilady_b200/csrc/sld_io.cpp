// File formats kept from the reference for drop-in use:
//   variables.in   read_variables.cpp:40-253 (key value pairs, unknown keys
//                  ignored), plus this engine's runtime switches
//   con- files     read_config.cpp:39-116 (atoms configuration)
//   readTe files   map_cells.cpp:33-39,136-150 (electron temperature per cell)
// and the output files (written by sld_check / sld_write_config):
//   enr- tmp- str- prs- spn- lines   check.cpp:31-47 and check_*_CPU.cpp
//   con- cel- files                  write_config.cpp:31-169
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sld.h"
#include "sld_host.h"

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
        else if (key == "gamma_S_H") P->gamma_S_H = v;
        else if (key == "hamiltonian") {
            // the name of control.h's switch, or its number
            if (val == "SLDHL") P->hamiltonian = SLD_HAM_SLDHL;
            else if (val == "SLDH") P->hamiltonian = SLD_HAM_SLDH;
            else if (val == "MD") P->hamiltonian = SLD_HAM_MD;
            else if (val == "SDH") P->hamiltonian = SLD_HAM_SDH;
            else if (val == "SDHL") P->hamiltonian = SLD_HAM_SDHL;
            else P->hamiltonian = iv;
        }
        else if (key == "random_seed") P->random_seed = iv;
        else if (key == "rcut_pot") P->rcut_pot = v;
        else if (key == "rcut_mag") P->rcut_mag = v;
        else if (key == "rcut_max") P->rcut_max = v;
        else if (key == "min_length_link_cell") P->min_length_link_cell = v;
        else if (key == "kappa_e") P->kappa_e = v;
        else if (key == "interval_of_print_out") P->interval_of_print_out = iv;
        else if (key == "interval_of_config_out") P->interval_of_config_out = iv;
        else if (key == "interval_of_scale_pressure") P->interval_of_scale_pressure = iv;
        else if (key == "interval_of_scale_stress") P->interval_of_scale_stress = iv;
        else if (key == "pressure") P->pressure = v;
        else if (key == "stress_xx") P->stress[0] = v;
        else if (key == "stress_yx") P->stress[1] = v;
        else if (key == "stress_yy") P->stress[2] = v;
        else if (key == "stress_zx") P->stress[3] = v;
        else if (key == "stress_zy") P->stress[4] = v;
        else if (key == "stress_zz") P->stress[5] = v;
        else if (key == "baro_damping_time") P->baro_damping_time = v;
        else if (key == "displace_limit") P->displace_limit = v;
        else if (key == "phi_limit") P->phi_limit = v;
        // control.h switches, which the reference fixes at compile time
        else if (key == "spinlang") P->spinlang = iv;
        else if (key == "lattlang") P->lattlang = iv;
        else if (key == "eltemp") P->eltemp = iv;
        else if (key == "localcolmot") P->localcolmot = iv;
        else if (key == "renormalizeEnergy") P->renormalize_energy = iv;
        else if (key == "PRESSURE") P->pressure_control = iv;
        else if (key == "STRESS") P->stress_control = iv;
        else if (key == "changestep") P->change_step = iv;
        else if (key == "quantumnoise") P->quantum_noise = iv;
        else if (key == "Msteps_quantum") P->msteps_quantum = iv;
        else if (key == "Nfrequency_quantum") P->nfrequency_quantum = iv;
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
    // the file's Hamiltonian (read_config.cpp:60-65) selects the context's
    if (type == "SLDHL") P.hamiltonian = SLD_HAM_SLDHL;
    else if (type == "SLDH") P.hamiltonian = SLD_HAM_SLDH;
    else if (type == "MD") P.hamiltonian = SLD_HAM_MD;
    else if (type == "SDH") P.hamiltonian = SLD_HAM_SDH;
    else if (type == "SDHL") P.hamiltonian = SLD_HAM_SDHL;
    else return SLD_ERR_IO;
    const bool latt = P.hamiltonian <= SLD_HAM_MD, spin = P.hamiltonian != SLD_HAM_MD;
    const bool hl = P.hamiltonian == SLD_HAM_SLDHL || P.hamiltonian == SLD_HAM_SDHL;
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
        double v[32];
        if (!(ls >> idx >> el)) return SLD_ERR_IO;
        // r(3) [p(3) f(3) stress(6) rho ke pe] [s(3) s0 Heff_H(3) [Heff_L(3)] me me0]
        // local_volume (write_config.cpp:100-127)
        const int nv = 3 + (latt ? 15 : 0) + (spin ? 9 + (hl ? 3 : 0) : 0) + 1;
        for (int k = 0; k < nv; ++k)
            if (!(ls >> v[k])) return SLD_ERR_IO;
        const int sat = latt ? 18 : 3;
        for (int k = 0; k < 3; ++k) {
            r[3 * i + k] = v[k];
            p[3 * i + k] = latt ? v[3 + k] : 0.0;
            s[3 * i + k] = spin ? v[sat + k] : 0.0;
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
                    // centre, Te, then [Tl] [Ts_R] [Ts_L] (write_config.cpp:154-166)
                    double a, b, c, T, x;
                    if (!(tin >> a >> b >> c >> T)) return SLD_ERR_IO;
                    const int extra = (latt ? 1 : 0) + (spin ? 1 : 0) + (hl ? 1 : 0);
                    for (int q = 0; q < extra; ++q)
                        if (!(tin >> x)) return SLD_ERR_IO;
                    te[ix + iy * nx + iz * nx * ny] = T;
                }
    }
    return sld_create(out, &P, (int)natom, r.data(), p.data(), s.data(),
                      te.empty() ? nullptr : te.data());
}

// ---------------------------------------------------------------------
// Output files (check.cpp, write_config.cpp).  Numbers are written as the
// reference's streams write them, setiosflags(ios::scientific) with
// setprecision(15): printf's "%.15e".

namespace sld {

std::string out_path(const char* dir, const char* prefix, const char* body, int n_output) {
    std::string p;
    if (dir && *dir) {
        p = dir;
        if (p.back() != '/') p += '/';
    }
    p += prefix;
    p += body;
    if (n_output >= 0) {
        // write_config.cpp:48-58 forms the four digits by character
        // arithmetic (n_output 9999 is the final write, write(-2))
        char s[6] = {'_', (char)(n_output / 1000 + '0'), (char)((n_output % 1000) / 100 + '0'),
                     (char)((n_output % 100) / 10 + '0'), (char)(n_output % 10 + '0'), '\0'};
        p += s;
    }
    p += ".dat";
    return p;
}

int append_line(const std::string& path, int step, const double* v, int n) {
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return SLD_ERR_IO;
    std::fprintf(f, "%d", step);
    for (int k = 0; k < n; ++k) std::fprintf(f, " %.15e", v[k]);
    std::fputc('\n', f);
    return std::fclose(f) == 0 ? SLD_OK : SLD_ERR_IO;
}

namespace {

// rows [r0, r1) of a table, formatted by up to T threads into one buffer per
// thread, written in order; a row is "<i> <element> v0 ... v(n-1)\n" (con-)
// or "v0 ... v(n-1) \n" (cel-, every value followed by a space)
int write_rows(FILE* f, long nrows, int ncols, const double* table, const char* element) {
    const long kBatch = 1L << 14;
    unsigned T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::string> buf(T);
    for (long b0 = 0; b0 < nrows; b0 += kBatch * (long)T) {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < T; ++t) {
            th.emplace_back([&, t] {
                std::string& o = buf[t];
                o.clear();
                long r0 = b0 + (long)t * kBatch, r1 = std::min(nrows, r0 + kBatch);
                char num[40];
                for (long r = r0; r < r1; ++r) {
                    const double* v = table + (size_t)r * ncols;
                    if (element) {
                        int m = std::snprintf(num, sizeof num, "%ld ", r);
                        o.append(num, m);
                        o += element;
                        for (int k = 0; k < ncols; ++k) {
                            m = std::snprintf(num, sizeof num, " %.15e", v[k]);
                            o.append(num, m);
                        }
                    } else {
                        for (int k = 0; k < ncols; ++k) {
                            int m = std::snprintf(num, sizeof num, "%.15e ", v[k]);
                            o.append(num, m);
                        }
                    }
                    o += '\n';
                }
            });
        }
        for (auto& x : th) x.join();
        for (unsigned t = 0; t < T; ++t)
            if (!buf[t].empty() && std::fwrite(buf[t].data(), 1, buf[t].size(), f) != buf[t].size())
                return SLD_ERR_IO;
    }
    return SLD_OK;
}

void box_lines(FILE* f, const double* d) {
    std::fprintf(f, "%.15e %.15e %.15e\n", d[0], d[1], d[2]);
    std::fprintf(f, "%.15e %.15e %.15e\n", d[3], d[4], d[5]);
}

}  // namespace

int write_con_file(const std::string& path, long natom, double total_time, const double* box,
                   const char* type, const char* element, int ncols, const double* table) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return SLD_ERR_IO;
    std::fprintf(f, "%ld %.15e %s\n", natom, total_time, type);
    box_lines(f, box);
    int rc = write_rows(f, natom, ncols, table, element);
    if (std::fclose(f) != 0 && rc == SLD_OK) rc = SLD_ERR_IO;
    return rc;
}

int write_cel_file(const std::string& path, long ncells, double total_time, const double* box,
                   int ncols, const double* table) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return SLD_ERR_IO;
    std::fprintf(f, "%ld %.15e\n", ncells, total_time);
    box_lines(f, box);
    int rc = write_rows(f, ncells, ncols, table, nullptr);
    if (std::fclose(f) != 0 && rc == SLD_OK) rc = SLD_ERR_IO;
    return rc;
}

}  // namespace sld
