/*
 * Test infrastructure only (the checker, never the product): a plain C
 * restatement of the reference's CPU step (SPILADY 1.0, -DSLDHL) for one
 * system, single-threaded.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.
 *
 * Pinning: with rng = ORC_RNG_MWC and one thread it follows the reference's
 * operation order, and tests/test_oracle_pin.py checks it against the
 * reference's own build (oracle/_ref) and the committed tests/golden fixtures.
 * With rng = ORC_RNG_PHILOX it draws the engine's counter-based noise, so the
 * CUDA path can be compared with it number for number.
 */
#ifndef SLD_ORACLE_H
#define SLD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_RNG_MWC = 0, ORC_RNG_PHILOX = 1 };

typedef struct {
    double box[6];            /* d.xx d.yx d.yy d.zx d.zy d.zz (Angstrom) */
    double step;              /* s */
    double temperature;       /* K */
    double atmass;            /* u */
    double gamma_L_over_mass; /* s^-1 */
    double gamma_S_HL;
    double rcut_pot, rcut_mag, rcut_max, min_length_link_cell;
    double kappa_e;
    int random_seed;
    int spinlang, lattlang, eltemp, localcolmot, renormalize;
    int rng;                  /* ORC_RNG_* */
    int te_mesh;              /* 0: Te on link cells; n > 0: n^3 Te mesh */
    int te_nloop;             /* Te substeps per core_dTe call (reference: 50) */
    int interval_of_print_out;
    /* quantum thermostat (control.h's quantumnoise, quantum_noise_CPU.cpp):
       the lattice noise coloured by an FIR filter; Msteps_quantum,
       Nfrequency_quantum (default.h:222-225) */
    int quantum, msteps_quantum, nfrequency_quantum;
} orc_params;

typedef struct orc_sys orc_sys;

/* Set-up as the reference's initialize(); te_K is per Te cell (NULL: all at
   the lattice temperature).  Returns NULL on invalid input. */
orc_sys* orc_create(const orc_params* prm, int natom, const double* r,
                    const double* p, const double* s, const double* te_K);
void orc_destroy(orc_sys*);

void orc_links(orc_sys*);
void orc_rho(orc_sys*);
void orc_force(orc_sys*);
void orc_core_ds(orc_sys*, double dt);
void orc_core_dp(orc_sys*, double dt);
void orc_core_dr(orc_sys*, double dt);
void orc_core_dte(orc_sys*, double dt);
void orc_temperature(orc_sys*);
/* nsteps of the reference main loop body: core(); time; check_energy
   renormalisation when enabled */
void orc_run(orc_sys*, int nsteps);
/* averages: pe, ke, me, me0, Ee, Tl, Te(K), <sx>, <sy>, <sz> */
void orc_averages(orc_sys*, double* out10);
/* the quantum thermostat's filter (2 Nfrequency_quantum coefficients) */
int orc_quantum_filter(orc_sys*, double* out, int n);

int orc_natom(const orc_sys*);
int orc_ncells(const orc_sys*);
int orc_nte(const orc_sys*);
int orc_ngroups(const orc_sys*);
/* field names: r p f s s0 H HL rho pe ke me me0 vir sumJ cell
   per-Te-cell: Te Ee Tl Ts_R Ts_L Gel Ges count */
int orc_get(const orc_sys*, const char* name, double* out);
/* cell member lists head->tail concatenated (natom ints) */
void orc_lists(const orc_sys*, int* out);
double orc_total_time(const orc_sys*);
/* Philox4x32-10 normals as the engine draws them (exposed for tests) */
void orc_philox_normals(unsigned seed, unsigned replica, unsigned atom,
                        unsigned long long epoch, double* out3);

/* raw Philox4x32-10 block (for known-answer tests) */
void orc_philox4x32(const unsigned* ctr4, const unsigned* key2, unsigned* out4);

#ifdef __cplusplus
}
#endif
#endif
