/*
 * Test infrastructure only: a driver that links the reference's own CPU
 * objects (SPILADY 1.0, built by oracle/ref/build.sh from its unmodified
 * sources) in place of its spilady.cpp main(), so that the tests can feed it
 * a synthetic state and read back full-precision per-atom and per-cell
 * arrays at any point of the step.  Nothing in the product links this.
 *
 * The set-up follows the reference's initialize() (initial.cpp:31-106) with
 * the file readers replaced by the job file below:
 *   potential_table()                     potential_CPU.cpp:61
 *   box and atoms as read_config() does    read_config.cpp:39-141
 *   map_cells(), initial_links(),          map_cells.cpp:31, links_CPU.cpp:33
 *   allocate_cells()                       allocate_cells_CPU.cpp:33
 *   calculate_rho(); calculate_force_energy()   (initial.cpp:78-83, run
 *                                          unconditionally, as a fresh start)
 *   calculate_temperature() with eltemp    initial.cpp:85-87
 *   initialize_random_number()             initial.cpp:99
 *   check_energy(-1) with renormalizeEnergy   spilady.cpp:38 -> check.cpp:33
 * and one "core" op is the body of the reference main loop
 * (spilady.cpp:50-57): core(step); total_time += step; and, because it
 * changes Te, the check_energy() call of check() when renormalizeEnergy is on.
 * The "step" op is the whole body with the reference's output: core(step);
 * total_time += step; check(step); scale(step); write_config(step) (scale()
 * does nothing without the PRESSURE, STRESS or changestep switches of the
 * baro and dtstep builds).  check() appends to
 * enr-/tmp-/str-/prs-/spn-ref.dat and write_config() writes
 * con-ref_NNNN.dat (and cel-ref_NNNN.dat with eltemp) in the working
 * directory, with interval_of_print_out 1 and interval_of_config_out as set
 * by the config-interval op (default 1).
 *
 * Job file (little endian):
 *   int32  magic 0x534c4431, natom, omp_threads, n_te, n_ops
 *   double box[6] (xx yx yy zx zy zz), step, temperature_K, atmass_u,
 *          gamma_L_over_mass, gamma_S_HL, rcut_pot, rcut_mag, rcut_max,
 *          min_length_link_cell, kappa_e
 *   int32  random_seed
 *   double r[3N], p[3N], s[3N]
 *   double te_K[n_te]           (n_te == 0: Te = temperature everywhere)
 *   n_ops x { int32 code, double arg }
 * Output: one record per DUMP op (see dump()).
 */
#define MAIN
#include "spilady.h"

/* what the compiled Hamiltonian has (struct.h:44-118 declares the fields) */
#if defined MD || defined SLDH || defined SLDHL
#define H_LATT 1
#endif
#if defined SDH || defined SDHL || defined SLDH || defined SLDHL
#define H_SPIN 1
#endif
#if defined SDHL || defined SLDHL
#define H_HL 1
#endif

#include <stdio.h>
#include <stdint.h>
#include <vector>

enum {
    OP_DUMP = 0, OP_LINKS = 1, OP_RHO = 2, OP_FORCE = 3, OP_DS = 4,
    OP_DP = 5, OP_DR = 6, OP_DTE = 7, OP_TEMP = 8, OP_CORE = 9,
    OP_CHECK_ENERGY = 10, OP_STEP = 11, OP_CONFIG_INTERVAL = 12, OP_WRITE_CONFIG = 13,
    OP_CHECK = 14,
    /* quantum build: initial_quantum_noise() after the OP_SET ops of its
       variables (initial.cpp:102-104), and its filter written to qfilter.dat */
    OP_QINIT = 15, OP_QFILTER = 16,
    /* a dump record without the arrays (natom = ncells = 0): the time and
       the wall time of the last OP_CORE, for timing runs of large systems */
    OP_STATS = 17,
    /* OP_SET + k sets input variable k (read_variables.cpp:197-241):
       0 pressure, 1 baro_damping_time, 2-7 stress_xx yx yy zx zy zz,
       8 interval_of_scale_pressure, 9 interval_of_scale_stress,
       10 displace_limit, 11 phi_limit, 12 Msteps_quantum, 13 Nfrequency_quantum */
    OP_SET = 100
};

static double g_last_wall = 0.0;
static long g_steps_done = 0;

static void die(const char* m) { fprintf(stderr, "harness: %s\n", m); exit(2); }

template <class T> static void rd(FILE* f, T* p, size_t n) {
    if (n && fread(p, sizeof(T), n, f) != n) die("short job file");
}
template <class T> static void wr(FILE* f, const T* p, size_t n) {
    if (n && fwrite(p, sizeof(T), n, f) != n) die("short write");
}

/* Per-atom record fields, in this order. */
static const int ATOM_FIELDS = 34;
static void dump(FILE* out) {
    int32_t hdr[4] = {0x44554d50, natom, ncells, ngroups};
    wr(out, hdr, 4);
    double sc[2] = {total_time, g_last_wall};
    wr(out, sc, 2);
    std::vector<double> a((size_t)natom * ATOM_FIELDS);
    for (int i = 0; i < natom; ++i) {
        atom_struct* p = first_atom_ptr + i;
        double* o = &a[(size_t)i * ATOM_FIELDS];
        int k = 0;
        /* fields the compiled Hamiltonian lacks are written as 0 */
        for (int q = 0; q < ATOM_FIELDS; ++q) o[q] = 0.0;
        o[k++] = p->r.x; o[k++] = p->r.y; o[k++] = p->r.z;
#ifdef H_LATT
        o[k++] = p->p.x; o[k++] = p->p.y; o[k++] = p->p.z;
        o[k++] = p->f.x; o[k++] = p->f.y; o[k++] = p->f.z;
#else
        k += 6;
#endif
#ifdef H_SPIN
        o[k++] = p->s.x; o[k++] = p->s.y; o[k++] = p->s.z;
        o[k++] = p->s0;
        o[k++] = p->Heff_H.x; o[k++] = p->Heff_H.y; o[k++] = p->Heff_H.z;
#else
        k += 7;
#endif
#ifdef H_HL
        o[k++] = p->Heff_L.x; o[k++] = p->Heff_L.y; o[k++] = p->Heff_L.z;
#else
        k += 3;
#endif
#ifdef H_LATT
        o[k++] = p->rho; o[k++] = p->pe; o[k++] = p->ke;
#else
        k += 3;
#endif
#ifdef H_SPIN
        o[k++] = p->me; o[k++] = p->me0;
#else
        k += 2;
#endif
#ifdef H_LATT
        o[k++] = p->vir;
        o[k++] = p->stress11; o[k++] = p->stress22; o[k++] = p->stress33;
        o[k++] = p->stress12; o[k++] = p->stress23; o[k++] = p->stress31;
#else
        k += 7;
#endif
#ifdef SLDHL
        o[k++] = p->sum_Jij_sj;
#else
        k += 1;
#endif
        o[k++] = p->local_volume;
        o[k++] = (double)p->new_cell_index;
        if (k != ATOM_FIELDS) die("field count");
    }
    wr(out, a.data(), a.size());
    /* per-cell: count, Te, Ee, Tl, Ts_R, Ts_L, Gel, Ges (K for temperatures
       as the reference prints them: Te / boltz, the others as stored) */
    std::vector<double> c((size_t)ncells * 8, 0.0);
    for (int i = 0; i < ncells; ++i) {
        cell_struct* q = first_cell_ptr + i;
        double* o = &c[(size_t)i * 8];
        o[0] = q->no_of_atoms_in_cell;
#ifdef eltemp
        o[1] = q->Te / boltz; o[2] = q->Ee;
#ifdef H_LATT
        o[3] = q->Tl; o[6] = q->Gel;
#endif
#ifdef H_SPIN
        o[4] = q->Ts_R; o[7] = q->Ges;
#endif
#ifdef H_HL
        o[5] = q->Ts_L;
#endif
#endif
    }
    wr(out, c.data(), c.size());
    /* cell member lists head -> tail */
    std::vector<int32_t> lists;
    lists.reserve(natom);
    for (int i = 0; i < ncells; ++i) {
        for (atom_struct* p = first_cell_ptr[i].head_ptr; p; p = p->next_atom_ptr)
            lists.push_back((int32_t)(p - first_atom_ptr));
    }
    int32_t nl = (int32_t)lists.size();
    wr(out, &nl, 1);
    wr(out, lists.data(), lists.size());
    /* colour groups: member count, then cell indices in sweep order */
    std::vector<int32_t> grp;
    for (int g = 0; g < ngroups; ++g) {
        int n = allocate_threads_ptr[g];
        grp.push_back(n);
        for (int j = 0; j < n; ++j)
            grp.push_back((int32_t)(allocate_cell_ptr_ptr[g * max_no_of_members + j] - first_cell_ptr));
    }
    int32_t ng = (int32_t)grp.size();
    wr(out, &ng, 1);
    wr(out, grp.data(), grp.size());
}

int main(int argc, char** argv) {
    if (argc != 3) die("usage: harness job.bin out.bin");
    FILE* f = fopen(argv[1], "rb");
    if (!f) die("cannot open job");
    int32_t h[5];
    rd(f, h, 5);
    if (h[0] != 0x534c4431) die("bad magic");
    int n = h[1], nthr = h[2], n_te = h[3], n_ops = h[4];
    double pr[17];
    rd(f, pr, 17);
    int32_t seed;
    rd(f, &seed, 1);

    OMP_threads = nthr > 0 ? nthr : 1;
    omp_set_num_threads(OMP_threads);
    out_body = (char*)malloc(8);
    strcpy(out_body, "ref");
    interval_of_print_out = 1;
    interval_of_config_out = 1;

    d.xx = pr[0]; d.yx = pr[1]; d.yy = pr[2]; d.zx = pr[3]; d.zy = pr[4]; d.zz = pr[5];
    step = pr[6];
    temperature = pr[7] * boltz;
    atmass = pr[8] * utoeV * pow(length_scale, 2);
#ifdef lattlang
    gamma_L_over_mass = pr[9];
    gamma_L = gamma_L_over_mass * atmass;
#endif
#ifdef spinlang
#if defined SDH || defined SLDH
    gamma_S_H = pr[10];
#else
    gamma_S_HL = pr[10];
#endif
#endif
#ifdef H_LATT
    rcut_pot = pr[11];
#endif
#ifdef H_SPIN
    rcut_mag = pr[12];
#endif
    rcut_max = pr[13];
    min_length_link_cell = pr[14];
#ifdef eltemp
    kappa_e = pr[15];
#endif
    random_seed = seed;
    /* read_variables.cpp:256-276 */
    if (rcut_max > min_length_link_cell) min_length_link_cell = rcut_max + 0.001;
#ifdef H_LATT
    rcut_pot_sq = pow(rcut_pot, 2);
#endif
#ifdef H_SPIN
    rcut_mag_sq = pow(rcut_mag, 2);
#endif
    rcut_max_sq = pow(rcut_max, 2);

    potential_table();

    natom = n;
    Inv_d = inverse_box_vector(d);
    first_atom_ptr = (atom_struct*)calloc((size_t)natom, sizeof(atom_struct));
    std::vector<double> r(3 * (size_t)n), p(3 * (size_t)n), s(3 * (size_t)n);
    rd(f, r.data(), r.size());
    rd(f, p.data(), p.size());
    rd(f, s.data(), s.size());
    for (int i = 0; i < n; ++i) {
        atom_struct* a = first_atom_ptr + i;
        a->r = vec_init(r[3 * i], r[3 * i + 1], r[3 * i + 2]);
#ifdef H_LATT
        a->p = vec_init(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
        a->ke = vec_sq(a->p) / 2e0 / atmass;
#endif
#ifdef H_SPIN
        a->s = vec_init(s[3 * i], s[3 * i + 1], s[3 * i + 2]);
        a->s0 = vec_length(a->s);
        a->m = vec_times(-el_g, a->s);
        a->m0 = vec_length(a->m);
#endif
        a->element[0] = 'F'; a->element[1] = 'e';
    }
#ifdef extfield
    external_field(-1);   /* initial.cpp:58-60: extfield.in in the working directory */
#endif
#ifdef extforce
    external_force(-1);   /* initial.cpp:61-63: extforce.in */
#endif
    box_length.x = fabs(d.xx);
    box_length.y = sqrt(d.yx * d.yx + d.yy * d.yy);
    box_length.z = sqrt(d.zx * d.zx + d.zy * d.zy + d.zz * d.zz);
    box_length_half = vec_times(0.5, box_length);
    box_volume = d.xx * d.yy * d.zz;
    density = double(natom) / box_volume;

    map_cells();
    std::vector<double> te(n_te > 0 ? n_te : 0);
    rd(f, te.data(), te.size());
#ifdef eltemp
    if (n_te > 0) {
        if (n_te != ncells) die("n_te != ncells");
        for (int i = 0; i < ncells; ++i) {
            first_cell_ptr[i].Te = te[i] * boltz;
            first_cell_ptr[i].Ee = Te_to_Ee(first_cell_ptr[i].Te);
        }
    }
#endif
    initial_links();
    allocate_cells();
#ifdef H_LATT
    calculate_rho();
#endif
    calculate_force_energy();
#ifdef eltemp
    calculate_temperature();
#endif
    total_time = 0e0;
#ifdef PRESSURE
    last_total_time_pressure = total_time;   /* initial.cpp:92-97 */
#endif
#ifdef STRESS
    last_total_time_stress = total_time;
#endif
    initialize_random_number();
#if defined eltemp && defined renormalizeEnergy
    check_energy(-1);
#endif

    FILE* out = fopen(argv[2], "wb");
    if (!out) die("cannot open output");
    for (int k = 0; k < n_ops; ++k) {
        int32_t code;
        double arg;
        rd(f, &code, 1);
        rd(f, &arg, 1);
        switch (code) {
        case OP_DUMP: dump(out); break;
        case OP_STATS: {
            int32_t hdr[4] = {0x44554d50, 0, 0, ngroups};
            wr(out, hdr, 4);
            double sc[2] = {total_time, g_last_wall};
            wr(out, sc, 2);
            int32_t none[2] = {0, 0};   /* no list entries, no groups */
            wr(out, none, 2);
            break;
        }
        case OP_LINKS: links(); break;
        case OP_FORCE: calculate_force_energy(); break;
#ifdef H_LATT
        case OP_RHO: calculate_rho(); break;
        case OP_DP: core_dp(arg); break;
        case OP_DR: core_dr(arg); break;
#endif
#ifdef H_SPIN
        case OP_DS: core_ds(arg); break;
#endif
#ifdef eltemp
        case OP_DTE: core_dTe(arg); break;
        case OP_TEMP: calculate_temperature(); break;
#endif
        case OP_CORE: {
            long nsteps = (long)arg;
            double t_core = 0.0;
            for (long j = 0; j < nsteps; ++j) {
                int cur = (int)g_steps_done;
                double t0 = omp_get_wtime();
                core(cur);
                t_core += omp_get_wtime() - t0;
                total_time += step;
#if defined eltemp && defined renormalizeEnergy
                if ((cur + 1) % interval_of_print_out == 0) check_energy(cur);
#endif
                ++g_steps_done;
            }
            g_last_wall = t_core;
            break;
        }
        case OP_CHECK_ENERGY: check_energy((int)arg); break;
        case OP_STEP: {
            long nsteps = (long)arg;
            for (long j = 0; j < nsteps; ++j) {
                int cur = (int)g_steps_done;
                core(cur);
                total_time += step;
                check(cur);
                scale(cur);
                write_config(cur);
                ++g_steps_done;
            }
            break;
        }
        case OP_CONFIG_INTERVAL: interval_of_config_out = (int)arg; break;
        case OP_WRITE_CONFIG: write_config((int)arg); break;
        case OP_CHECK: check((int)arg); break;
#ifdef PRESSURE
        case OP_SET + 0: pressure = arg; break;
        case OP_SET + 8: interval_of_scale_pressure = (int)arg; break;
#endif
#if defined STRESS || defined PRESSURE
        case OP_SET + 1: baro_damping_time = arg; break;
#endif
#ifdef STRESS
        case OP_SET + 2: stress_xx = arg; break;
        case OP_SET + 3: stress_yx = arg; break;
        case OP_SET + 4: stress_yy = arg; break;
        case OP_SET + 5: stress_zx = arg; break;
        case OP_SET + 6: stress_zy = arg; break;
        case OP_SET + 7: stress_zz = arg; break;
        case OP_SET + 9: interval_of_scale_stress = (int)arg; break;
#endif
#ifdef changestep
        case OP_SET + 10: displace_limit = arg; break;
        case OP_SET + 11: phi_limit = arg; break;
#endif
#ifdef quantumnoise
        case OP_SET + 12: Msteps_quantum = (int)arg; break;
        case OP_SET + 13:
            Nfrequency_quantum = (int)arg;
            Nfrequency_quantum_2 = 2 * Nfrequency_quantum;   /* read_variables.cpp:247-250 */
            break;
        case OP_QINIT: initial_quantum_noise(); break;
        case OP_QFILTER: {
            FILE* q = fopen("qfilter.dat", "w");
            for (int k = 0; k < Nfrequency_quantum_2; ++k) fprintf(q, "%.17g\n", H_ptr[k]);
            fclose(q);
            break;
        }
#endif
        default: die("unknown op");
        }
    }
    fclose(out);
    fclose(f);
    return 0;
}
