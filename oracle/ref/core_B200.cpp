/* core_B200.cpp: the reference's step functions backed by the B200 engine.
 *
 * SPILADY plugs its backends in at link time: core() (core.cpp:31-76) calls
 * free functions declared in prototype_CPU.h:123-237, implemented once in
 * *_CPU.cpp and once in *_GPU.cu.  This file is a third implementation of
 * them, on one engine context (include/sld.h).  oracle/ref/build.sh (mode
 * b200) links it in front of the reference's own objects, including its
 * spilady.cpp main loop, so that its definitions are the ones used; the
 * reference's initialize(), check_* and write_config code run unchanged on
 * the host copies this file keeps current.
 *
 *   links, calculate_rho, calculate_force_energy, core_ds, core_dp, core_dr
 *                                       one engine call each (sld_links ...);
 *                                       links also relinks the host lists
 *                                       (links_CPU), which check_temperature
 *                                       walks
 *   check(step)                         at print-out steps: the engine's state
 *                                       copied into the reference's atoms and
 *                                       cells, then the reference's own
 *                                       check_energy / check_temperature /
 *                                       check_stress / check_pressure /
 *                                       check_spin (check.cpp:31-47)
 *
 * The context is made at the first step function's call, from the state
 * initialize() read (read_config / build_lattice).  The host copies are
 * current at every print-out step, so interval_of_print_out 1 keeps the host
 * cell lists (relinked from the positions of the last print-out) in step
 * with the engine's.  Noise: the engine draws Philox numbers, the reference
 * MWC ones, so Langevin runs agree statistically, NVE runs number for number.
 * Electron-temperature builds are refused (below).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "spilady.h"   // declares struct vector (with using namespace std: no <vector> here)
#include "sld.h"

// a host buffer of n doubles
struct Buf {
    double* v;
    explicit Buf(size_t n) : v(new double[n]) {}
    ~Buf() { delete[] v; }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
};

void links_CPU();   // links_CPU.cpp:85-177, the host lists

static sld_ctx* g_ctx = nullptr;

static void ok(int rc, const char* where) {
    if (rc != SLD_OK) {
        std::fprintf(stderr, "B200 backend: %s: %s\n", where, sld_error_string(rc));
        std::exit(1);
    }
}

static sld_ctx* ctx() {
    if (g_ctx) return g_ctx;
    sld_params P;
    ok(sld_params_default(&P), "sld_params_default");
    P.box[0] = d.xx; P.box[1] = d.yx; P.box[2] = d.yy;
    P.box[3] = d.zx; P.box[4] = d.zy; P.box[5] = d.zz;
    P.step = step;
    P.temperature = temperature / boltz;
    P.atmass = atmass / (utoeV * length_scale * length_scale);
    P.rcut_pot = rcut_pot;
    P.rcut_mag = rcut_mag;
    P.rcut_max = rcut_max;
    P.min_length_link_cell = min_length_link_cell;
    P.random_seed = random_seed;
    P.interval_of_print_out = interval_of_print_out;
#ifdef lattlang
    P.lattlang = 1;
    P.gamma_L_over_mass = gamma_L_over_mass;
#endif
#ifdef spinlang
    P.spinlang = 1;
    P.gamma_S_HL = gamma_S_HL;
#endif
#ifdef eltemp
    P.eltemp = 1;
    P.kappa_e = kappa_e;
#endif
#ifdef localcolmot
    P.localcolmot = 1;
#endif
#ifdef renormalizeEnergy
    P.renormalize_energy = 1;
#endif
    Buf rb(3 * (size_t)natom), pb(3 * (size_t)natom), sb(3 * (size_t)natom);
    double *r = rb.v, *p = pb.v, *s = sb.v;
    for (int i = 0; i < natom; ++i) {
        const atom_struct* a = first_atom_ptr + i;
        r[3 * i] = a->r.x; r[3 * i + 1] = a->r.y; r[3 * i + 2] = a->r.z;
        p[3 * i] = a->p.x; p[3 * i + 1] = a->p.y; p[3 * i + 2] = a->p.z;
        s[3 * i] = a->s.x; s[3 * i + 1] = a->s.y; s[3 * i + 2] = a->s.z;
    }
    ok(sld_create(&g_ctx, &P, natom, r, p, s, nullptr), "sld_create");
    return g_ctx;
}

void links() {
    ok(sld_links(ctx()), "links");
    links_CPU();
}
void calculate_rho() { ok(sld_calculate_rho(ctx()), "calculate_rho"); }
void calculate_force_energy() {
    ok(sld_calculate_force_energy(ctx()), "calculate_force_energy");
    // the total virial calculate_force_energy_CPU.cpp:296-299 leaves for check_pressure
    ok(sld_virial(ctx(), &virial), "sld_virial");
}
void core_ds(double dt) { ok(sld_core_ds(ctx(), dt), "core_ds"); }
void core_dp(double dt) { ok(sld_core_dp(ctx(), dt), "core_dp"); }
void core_dr(double dt) { ok(sld_core_dr(ctx(), dt), "core_dr"); }
#ifdef eltemp
// The electron cells' arrays (Te, Ee and calculate_temperature's sums) and the
// energy renormalisation check_energy applies to them would have to travel
// both ways at every print-out; this backend keeps the engine's own step
// (sld_run) for the electron runs.
#error "core_B200.cpp: eltemp runs use sld_run, which keeps the electrons on the device"
#endif

// the engine's per-atom arrays into the reference's atoms
static void pull_atoms() {
    sld_ctx* c = ctx();
    const long cap = 6 * (long)natom;
    Buf vb((size_t)cap);
    double* v = vb.v;
    auto vec = [&](const char* name, vector atom_struct::*field) {
        if (sld_get(c, name, v, cap) < 0) ok(SLD_ERR_ARG, name);
        for (int i = 0; i < natom; ++i) {
            vector& x = first_atom_ptr[i].*field;
            x.x = v[3 * i]; x.y = v[3 * i + 1]; x.z = v[3 * i + 2];
        }
    };
    auto scal = [&](const char* name, double atom_struct::*field) {
        if (sld_get(c, name, v, cap) < 0) ok(SLD_ERR_ARG, name);
        for (int i = 0; i < natom; ++i) first_atom_ptr[i].*field = v[i];
    };
    vec("r", &atom_struct::r);
    vec("p", &atom_struct::p);
    vec("f", &atom_struct::f);
    vec("s", &atom_struct::s);
    vec("H", &atom_struct::Heff_H);
    vec("HL", &atom_struct::Heff_L);
    scal("rho", &atom_struct::rho);
    scal("pe", &atom_struct::pe);
    scal("ke", &atom_struct::ke);
    scal("me", &atom_struct::me);
    scal("me0", &atom_struct::me0);
    scal("vir", &atom_struct::vir);
    scal("sumJ", &atom_struct::sum_Jij_sj);
    scal("s0", &atom_struct::s0);
    if (sld_get(c, "stress", v, cap) < 0) ok(SLD_ERR_ARG, "stress");
    for (int i = 0; i < natom; ++i) {
        atom_struct* a = first_atom_ptr + i;
        a->stress11 = v[6 * i];     a->stress22 = v[6 * i + 1]; a->stress33 = v[6 * i + 2];
        a->stress12 = v[6 * i + 3]; a->stress23 = v[6 * i + 4]; a->stress31 = v[6 * i + 5];
    }
}

void check(int current_step) {
    if ((current_step + 1) % interval_of_print_out != 0) return;
    pull_atoms();
    check_energy(current_step);
    check_temperature(current_step);
    check_stress(current_step);
    check_pressure(current_step);
    check_spin(current_step);
}
