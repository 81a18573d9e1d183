/*
 * sld.h - C ABI of the B200 spin-lattice dynamics step engine.
 *
 * The engine runs the per-step hot path of SPILADY 1.0 (-DSLDHL) on one
 * NVIDIA B200: link-cell relinking, EAM density, forces and energies,
 * Heisenberg + Landau effective fields with the Suzuki-Trotter colour sweeps,
 * the lattice updates, Langevin noise, and the electron-temperature
 * subsystem.  In the reference these are free functions that share global
 * state (prototype_CPU.h:123-237, called from core(), core.cpp:31-76) and are
 * swapped for their GPU twins at link time; here each becomes an entry point
 * on a context that owns the device state.  Plain C types only.
 *
 * Conventions
 *   - every entry point returns SLD_OK (0) or a negative SLD_ERR_* code;
 *   - one host thread drives one context at a time; several contexts may
 *     live in one process (each owns its own device memory and stream);
 *   - units are the reference's (spilady.h:53-62): Angstrom, eV, seconds;
 *     sld_params holds the variables.in values in their input units
 *     (temperature in K, atmass in u), converted as read_variables.cpp:256
 *     does;
 *   - arrays are row-major, one row per atom in the caller's atom order
 *     (x, y, z for vectors); the engine reorders internally and always
 *     returns data in the caller's order;
 *   - control.h's compile-time switches are the runtime fields spinlang,
 *     lattlang, eltemp, localcolmot and renormalize_energy.
 */
#ifndef SLD_H
#define SLD_H

#ifdef __cplusplus
extern "C" {
#endif

#define SLD_OK 0
#define SLD_ERR_ARG (-1)        /* invalid argument or parameter */
#define SLD_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define SLD_ERR_GEOMETRY (-3)   /* fewer than 3 link cells per axis (the
                                   reference then double counts neighbours,
                                   map_cells.cpp:89-121) */
#define SLD_ERR_CAPACITY (-4)   /* a link cell holds more atoms than the
                                   kernels support (SLD_MAX_CELL_ATOMS) */
#define SLD_ERR_TABLE (-5)      /* r or rho outside the potential table
                                   (the reference reads out of bounds,
                                   potential_CPU.cpp:172-179) */
#define SLD_ERR_NAN (-6)        /* a non-finite value was produced */
#define SLD_ERR_IO (-7)         /* a file could not be read or parsed */
#define SLD_ERR_STATE (-8)      /* call out of order (e.g. no state loaded) */
#define SLD_ERR_NOMEM (-9)      /* device allocation failed */
#define SLD_ERR_TIMEOUT (-10)   /* a bounded device-side wait ran out (the
                                   spin sweeps' cell-by-cell schedule); the
                                   state is no longer valid */

#define SLD_MAX_CELL_ATOMS 64

/* SLD_FP64: the reference's arithmetic (FP64, interpolated 10^6-point
   tables); SLD_SPLIT: FP32 pair terms with compensated sums, the same
   functions as the reference's tables (the functional forms with the
   tables' seven-point derivatives; F(rho) from the tables), FP64 integration
   and reductions; SLD_FP64_ANALYTIC: the functional forms in FP64 with their
   exact derivatives (the model the adjoint differentiates; near the knots of
   the cubics it differs from the tables' derivatives by about 1e-4). */
typedef enum { SLD_FP64 = 0, SLD_SPLIT = 1, SLD_FP64_ANALYTIC = 2 } sld_precision;

/* The Hamiltonian, control.h's mode switch (control.h:8-12; core.cpp:31-76):
   SLDHL spin-lattice, Heisenberg-Landau (the default); SLDH spin-lattice,
   Heisenberg; MD lattice only; SDH and SDHL spins only, on a fixed lattice. */
typedef enum {
    SLD_HAM_SLDHL = 0, SLD_HAM_SLDH = 1, SLD_HAM_MD = 2, SLD_HAM_SDH = 3, SLD_HAM_SDHL = 4
} sld_hamiltonian;

typedef struct {
    double box[6];               /* d.xx d.yx d.yy d.zx d.zy d.zz (Angstrom);
                                    struct.h box_vector, upper-triangular */
    double step;                 /* time step (s)                 default.h:62 */
    double temperature;          /* K                             default.h:159 */
    double atmass;               /* u                             default.h:158 */
    double gamma_L_over_mass;    /* s^-1 (lattice Langevin)       default.h:166 */
    double gamma_S_HL;           /* spin Langevin, Heisenberg-Landau  default.h:174 */
    double rcut_pot;             /* Angstrom                      default.h:200 */
    double rcut_mag;             /* Angstrom                      default.h:205 */
    double rcut_max;             /* Angstrom                      default.h:209 */
    double min_length_link_cell; /* Angstrom                      default.h:217 */
    double kappa_e;              /* electron thermal conductivity, W/(m K) default.h:96 */
    int random_seed;             /*                               default.h:161 */
    int spinlang;                /* control.h:22 */
    int lattlang;                /* control.h:23 */
    int eltemp;                  /* control.h:25 */
    int localcolmot;             /* control.h:28 */
    int renormalize_energy;      /* control.h:27 */
    int te_mesh;                 /* 0: Te per link cell as the reference
                                    (map_cells.cpp:128); n > 0: an n^3 Te
                                    mesh decoupled from the link cells */
    int te_nloop;                /* Te substeps per core_dTe call; the
                                    reference CPU path uses 50
                                    (core_dTe_CPU.cpp:49) */
    int interval_of_print_out;   /* energy renormalisation interval
                                    (check.cpp:33)                default.h:64 */
    int precision;               /* sld_precision */
    int device;                  /* CUDA device ordinal */
    int replica;                 /* key of this system's noise stream: the
                                    Philox key is (random_seed, replica), so
                                    replicas of one seed draw independent
                                    noise (0 for a single system) */
    int interval_of_config_out;  /* con-/cel- file interval (write_config.cpp:33)
                                                                  default.h:65 */
    /* sld_scale (scale.cpp:31-44): control.h's PRESSURE, STRESS and
       changestep switches and their variables */
    int pressure_control;        /* Berendsen barostat on the pressure
                                    (scale_pressure_CPU.cpp:35-60) */
    int stress_control;          /* Berendsen barostat on the stress tensor
                                    (scale_stress_CPU.cpp:35-85) */
    int change_step;             /* adaptive time step (scale_step_CPU.cpp:35-100) */
    int interval_of_scale_pressure;  /*                           default.h:188 */
    int interval_of_scale_stress;    /*                           default.h:179 */
    double pressure;             /* target pressure, GPa          default.h:189 */
    double stress[6];            /* target stresses, GPa: stress_xx yx yy zx zy zz
                                                                  default.h:180-185 */
    double baro_damping_time;    /* s                             default.h:192 */
    double displace_limit;       /* Angstrom per step             default.h:218 */
    double phi_limit;            /* rad per step                  default.h:219 */
    int quantum_noise;           /* control.h's quantumnoise: the lattice
                                    thermostat's noise coloured to the quantum
                                    spectrum (quantum_noise_CPU.cpp) */
    int msteps_quantum;          /* the coloured noise changes every M kicks
                                                                  default.h:223 */
    int nfrequency_quantum;      /* frequency intervals of its filter
                                                                  default.h:224 */
    int hamiltonian;             /* sld_hamiltonian */
    double gamma_S_H;            /* spin Langevin, Heisenberg (SDH, SLDH), unitless
                                                                  default.h:172 */
} sld_params;

typedef struct sld_ctx sld_ctx;

/* Reference defaults (default.h:44-226 with variables.in's cutoffs). */
int sld_params_default(sld_params* out);

/* Parse a variables.in file (read_variables.cpp:40-253: whitespace
   separated key/value pairs, unknown keys ignored) into *inout. */
int sld_read_variables(const char* path, sld_params* inout);

/* Create a context and load a state: natom atoms, positions r, momenta p
   (eV s / Angstrom) and spins s, each natom x 3; te_K holds the initial
   electron temperature per Te cell (NULL: the lattice temperature), the
   readTe input of map_cells.cpp:33-39,136-150.  Then, as initialize()
   (initial.cpp:31-106) does: potential tables, link cells and colour groups,
   rho, forces and energies, cell temperatures, and with renormalize_energy
   the reference energy of check_energy(-1).  The split form takes at most
   2^27 - 1 atoms (SLD_ERR_CAPACITY beyond: its neighbour lists pack a
   27-bit slot with a neighbour-cell code). */
int sld_create(sld_ctx** out, const sld_params* prm, int natom,
               const double* r, const double* p, const double* s,
               const double* te_K);

/* Read an atoms configuration file in the reference's con- format
   (read_config.cpp:39-116) and create a context from it; params->box is
   taken from the file. */
int sld_create_from_config(sld_ctx** out, const sld_params* prm,
                           const char* con_path, const char* te_path);

void sld_destroy(sld_ctx* ctx);

/* Replace r, p, s (host arrays, caller order) and recompute rho, forces and
   energies as after a fresh start. */
int sld_set_state(sld_ctx* ctx, const double* r, const double* p,
                  const double* s);

/* The reference's step functions, one for one. */
int sld_links(sld_ctx* ctx);                       /* links_CPU.cpp:85 */
int sld_calculate_rho(sld_ctx* ctx);               /* calculate_rho_CPU.cpp:71 */
int sld_calculate_force_energy(sld_ctx* ctx);      /* calculate_force_energy_CPU.cpp:220 */
int sld_core_ds(sld_ctx* ctx, double dt);          /* core_ds_CPU.cpp:35 */
int sld_core_dp(sld_ctx* ctx, double dt);          /* core_dp_CPU.cpp:51 */
int sld_core_dr(sld_ctx* ctx, double dt);          /* core_dr_CPU.cpp:33 */
int sld_core_dTe(sld_ctx* ctx, double dt);         /* core_dTe_CPU.cpp:47 */
int sld_calculate_temperature(sld_ctx* ctx);       /* calculate_temperature_CPU.cpp:35 */

/* nsteps passes of the reference main-loop body (spilady.cpp:50-57):
   core(); total_time += step; and, when eltemp and renormalize_energy are
   set, check_energy's renormalisation every interval_of_print_out steps.
   The step is captured once as a CUDA graph and replayed. */
int sld_run(sld_ctx* ctx, int nsteps);

/* Copy a field to a host array in caller atom order.  Per-atom fields:
   "r" "p" "f" "s" (natom x 3), "H" "HL" (Heff_H, Heff_L, natom x 3), "s0"
   "rho" "pe" "ke" "me" "me0" "vir" "sum_Jij_sj" "local_volume" (natom),
   "stress" (natom x 6: 11 22 33 12 23 31), "cell" (link cell index).
   Per-Te-cell fields: "Te" (K) "Ee" "Tl" "Ts_R" "Ts_L" "Gel" "Ges"
   "count".  Returns the number of doubles written, or a negative code.
   `capacity` is the size of `out` in doubles. */
long sld_get(sld_ctx* ctx, const char* field, double* out, long capacity);

/* Cell member lists (atom indices, caller order) head -> tail, cells in
   index order: natom ints. */
int sld_get_cell_lists(sld_ctx* ctx, int* out);

/* Averages as check_energy/check_temperature/check_spin compute them:
   out[0..9] = <pe>, <ke>, <me>, <me0>, <Ee>, Tl (K), <Te> (K), <sx>,
   <sy>, <sz>. */
int sld_averages(sld_ctx* ctx, double* out10);

/* Print-out of check(int current_step) (check.cpp:31-47): when
   (current_step + 1) % interval_of_print_out == 0, appends one line each to
   enr-<out_body>.dat (step, time, <pe>, <ke>, <me>, <me0>[, <Ee>]),
   tmp- (step, time, Tl, Ts_R, Ts_L[, <Te>]), str- (step, time, box, density,
   mean and six components of the stress in GPa), prs- (step, time, box,
   density, pressure in GPa) and spn- (step, time, <s>, |<s>|, <m>, |<m>|),
   in the directory dir (NULL or "": the working directory), as
   check_energy/temperature/stress/pressure/spin_CPU.cpp:35-79 do.  Call it
   after sld_run with the index of the last step run (-1 before the first).
   The energy renormalisation that check_energy performs runs inside the step
   (sld_run); with it, enr- holds the averages formed before that step's
   renormalisation, as the reference prints.  Without eltemp, Ts_R and Ts_L
   come from freshly computed fields, which, as in the reference, overwrite
   Heff_H, Heff_L and sum_Jij_sj (check_temperature_CPU.cpp:58-116). */
int sld_check(sld_ctx* ctx, const char* dir, const char* out_body, int current_step);

/* write_config(int current_step) (write_config.cpp:31-169): when
   current_step is -1 (file 0000), -2 (file 9999) or
   (current_step + 1) % interval_of_config_out == 0 (file
   current_step / interval_of_config_out + 1), writes
   con-<out_body>_NNNN.dat (natom, time, "SLDHL"; box; per atom: index,
   element, r, p, f, stress (6), rho, ke, pe, s, |s|, Heff_H, Heff_L, me,
   me0, local volume) and, with eltemp, cel-<out_body>_NNNN.dat (per cell,
   x-major: centre, Te, Tl, Ts_R, Ts_L; the Te mesh's nodes when te_mesh >
   0).  The reference prints the x component of Heff_H and Heff_L in their y
   columns (write_config.cpp:120,123); this writes the y component unless
   flags holds SLD_WRITE_HEFF_AS_REFERENCE. */
#define SLD_WRITE_HEFF_AS_REFERENCE 1
int sld_write_config(sld_ctx* ctx, const char* dir, const char* out_body, int current_step,
                     int flags);

/* scale(int current_step) (scale.cpp:31-44), called after sld_check:
   - stress_control, when (current_step + 1) % interval_of_scale_stress == 0:
     the box and positions follow the stresses of the last sld_check
     (scale_stress_CPU.cpp:35-85);
   - pressure_control, when (current_step + 1) % interval_of_scale_pressure
     == 0: the box and positions are scaled by the cube root of
     1 + dt_since_last/baro_damping_time (P_last_check - pressure)/100 GPa
     (scale_pressure_CPU.cpp:35-60);
   - change_step: the time step becomes 0.8 of itself when an atom moved
     more than displace_limit or a spin turned more than phi_limit in one
     step, else 1.05 of itself (scale_step_CPU.cpp:35-100).
   After a box change the next step uses exchange couplings of the new
   positions and the densities of the old ones, as the reference does.
   out3 (may be NULL) receives displace_max (Angstrom), phi_max (rad) and
   the new time step (s), which the reference prints; without change_step
   they are 0, 0 and the unchanged step.  With any of the three switches
   set, sld_run launches each step's kernels directly instead of replaying
   a graph, because the box and step change between steps; such contexts
   cannot join a batch. */
int sld_scale(sld_ctx* ctx, int current_step, double* out3);

/* Gradients with respect to the potential's parameters.  No reference
   counterpart: the reference's potential is fixed code (DD05.cpp,
   JijFe.cpp).  theta holds the 36 constants of its forms, in this order:
     [0, 2)   F(rho): a, b                       DD05.cpp:6-20
     [2, 8)   f(r): coefficients a_k, [8, 14) knots r_k    DD05.cpp:22-44
     [14, 22) phi(r): coefficients V_k, [22, 30) knots     DD05.cpp:64-84
     [30, 32) J(r) = A (1 - r/rc)^3: A, rc        JijFe.cpp:5-12
     [32, 36) Landau A, B, C, D                   JijFe.cpp:15-43
   The ZBL core and the 1.8-2.0 A join keep their form; the join's end at
   2.0 A follows the parameters.  The energy is E = sum_i (pe + me + me0)
   (calculate_force_energy_CPU.cpp:33-216); the loss is L = sum_i |f_i|^2 +
   |Heff_H,i|^2, forces and exchange fields of the configuration.  The
   context must be NVE (no thermostats, no electron temperature, no sld_scale
   switches) in an FP64 form; its state is unchanged afterwards. */
#define SLD_ADJ_NTHETA 36
int sld_adjoint_theta_default(double* theta36);

/* One configuration (the context's current state): out4 = E, L, sum |f|^2,
   sum |H|^2; dE and dL (36 each, may be NULL) = their gradients in theta,
   evaluated in FP64 by reverse-mode differentiation. */
int sld_adjoint_config(sld_ctx* ctx, const double* theta36, double* out4, double* dE36,
                       double* dL36);

/* Jacobians of one configuration's forces and exchange fields in theta,
   forward mode in FP64: dF and dH (natom x 3 x 36, caller order, the
   parameter index fastest; dH may be NULL) with d f_i / d theta_k and
   d Heff_H,i / d theta_k; f and H (natom x 3, may be NULL) the forces and
   fields themselves. */
int sld_adjoint_jacobians(sld_ctx* ctx, const double* theta36, double* f, double* H,
                          double* dF, double* dH);

/* Through a trajectory: nsteps NVE main-loop steps (core.cpp:55-63) from
   the context's current state with the parameters theta; *L = the loss of
   the final configuration and dL36 (may be NULL: forward only) its gradient
   in theta, by reverse-mode differentiation through every step with the
   state kept every checkpoint_every steps and each segment recomputed once
   in the reverse pass. */
int sld_adjoint_trajectory(sld_ctx* ctx, const double* theta36, int nsteps,
                           int checkpoint_every, double* L, double* dL36);

/* External field and force (control.h's extfield and extforce;
   external_field_CPU.cpp, external_force_CPU.cpp).  H: natom x 3 in eV, caller
   order: the exchange field of every atom starts at it and the magnetic
   energy gains -s.H (calculate_spin_CPU.cpp:35-40,
   calculate_force_energy_CPU.cpp:200-202).  f: natom x 3 in eV/A, added into
   each atom's force at every kick, which keeps it (core_dp_CPU.cpp:68-71,
   129-132).  NULL removes either.  A field set before the first step is
   part of the start state (its force pass, cell temperatures and reference
   energy are formed again, as initialize() does); later ones act from the
   next step.  The readers take the reference's
   extfield.in (Tesla, converted by -g muB) and extforce.in files.  Set them
   before sld_batch_create: a batch keeps the kernel arguments it captured. */
int sld_set_external_field(sld_ctx* ctx, const double* H_eV);
int sld_set_external_force(sld_ctx* ctx, const double* f);
int sld_read_external_field(sld_ctx* ctx, const char* path);
int sld_read_external_force(sld_ctx* ctx, const char* path);

/* The quantum thermostat's filter (initial_quantum_noise,
   quantum_noise_CPU.cpp:75-104): 2 nfrequency_quantum coefficients into out
   (capacity n).  Returns the count, or a negative code without quantum_noise. */
int sld_quantum_filter(sld_ctx* ctx, double* out, int n);

/* Autotuner of the launch shapes (no reference counterpart): times `steps`
   captured steps twice for each candidate and keeps one that is faster by
   more than 1% than the best so far, by coordinate
   descent over the cells per block of the spin sweeps and their CTAs per
   SM, the atoms per block of the pair/list and force passes, and, with
   eltemp, the core_dTe kernel (one CTA, a cluster, or the hub cluster by
   colour phases or by levels), the hub's threads per CTA and the Te-mesh
   temperature pass.  The state is copied first and put back, so the context
   continues exactly as if it had not run.  out8 (may be NULL): the chosen
   sweep, pair, force and temperature block sizes (0: default), core_dTe
   kernel (-1: default), hub threads (0: default), sweep CTAs per SM (0: no
   cap) and 0.  Not with sld_scale's switches (their steps are not
   captured). */
int sld_autotune(sld_ctx* ctx, int steps, int* out8);

/* out[0..5] = natom, ncells, ngroups, n_te_cells, nx, ny (link cells). */
int sld_info(sld_ctx* ctx, int* out6);

/* Total virial (sum of the per-atom virials, calculate_force_energy_CPU.cpp:298). */
int sld_virial(sld_ctx* ctx, double* out);

/* Simulated time (s). */
int sld_total_time(sld_ctx* ctx, double* out);

/* Block until the device work of this context is done and report any
   device-side error flag as an SLD_ERR_* code. */
int sld_sync(sld_ctx* ctx);

/* Milliseconds of device time of the last sld_run call (CUDA events on the
   context's stream). */
int sld_last_run_ms(sld_ctx* ctx, double* out);

/* Run one main-loop step phase by phase (no graph), timing each phase with
   CUDA events on the context's stream.  ms_out[SLD_PHASES] receives the
   device milliseconds of: links, core_dTe (both calls), core_dp (both),
   core_ds (both), core_dr, calculate_rho, calculate_force_energy,
   calculate_temperature, energy check, bookkeeping.  The step advances the
   state exactly as sld_run(ctx, 1) does.  Spin-lattice Hamiltonians (SLDHL,
   SLDH) only. */
#define SLD_PHASES 10
int sld_profile_step(sld_ctx* ctx, double* ms_out);

/* Number of kernel launches in one captured main-loop step. */
int sld_step_kernel_count(sld_ctx* ctx, int* out);

const char* sld_error_string(int code);

/* Batched replicas: several independent systems (contexts created on one
   device, each with its own size, parameters and noise stream, see
   sld_params.replica) advanced together.  Each step is one CUDA graph with
   every context's main-loop step (sld_run's sequence) as an independent
   branch, so the launches of small systems overlap on the GPU.  Every
   context ends in the state that sld_run on it alone would give.  A context
   may still be used on its own between batch runs; destroy the batch before
   its contexts.  No reference counterpart: the reference runs one system per
   process. */
typedef struct sld_batch sld_batch;
int sld_batch_create(sld_batch** out, sld_ctx* const* ctxs, int n);
int sld_batch_run(sld_batch* batch, int nsteps);
/* Milliseconds of device time of the last sld_batch_run (CUDA events). */
int sld_batch_last_run_ms(sld_batch* batch, double* out);
void sld_batch_destroy(sld_batch* batch);

/* Allocation-free averages.  This entry point has no counterpart in the
   reference; it exists for callers that cannot let a library allocate
   device memory (a code that gives all device memory to its own pool, or
   cannot afford cudaFree, which waits for all device work, during its
   stream-ordered work).  It computes out[0..7] = <pe>, <ke>, <me>, <me0>,
   Tl (K), <sx>, <sy>, <sz>, the same values as out[0,1,2,3,5,7,8,9] of
   the context-based averages entry point, from caller-owned device arrays
   pe, ke, me, me0 (natom each) and s (3 * natom, xyz per atom), and writes
   them to the device array out8, all on `stream` (a cudaStream_t; NULL is
   the default stream).  It calls no cudaMalloc or cudaFree: its scratch
   is a fixed device array compiled into the library, large enough for
   SLD_AVERAGES_STATIC_MAX_ATOMS atoms (2 MiB); larger natom is refused
   with SLD_ERR_CAPACITY before any launch.
   - The first call on each device (the device current at the call) looks
     up that array's device address (cudaGetSymbolAddress) and keeps it;
     make that first call before capturing any stream.
   - There is one scratch array per device, so calls that overlap on one
     device (on different streams, or from different host threads without
     ordering) race on it and can return wrong averages.  Order them on one
     stream or with events. */
#define SLD_AVERAGES_STATIC_MAX_ATOMS 8388608
int sld_averages_static(const double* pe, const double* ke, const double* me,
                        const double* me0, const double* s, int natom, double* out8,
                        void* stream);

#ifdef __cplusplus
}
#endif
#endif
