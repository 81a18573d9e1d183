// C ABI of the step engine (include/sld.h): context set-up, the reference's
// step functions as entry points, the CUDA-graph main loop and read-outs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/sld.h"
#include "potential.h"
#include "sld_pot32.cuh"
static_assert(SLD_DENS_KNOTS == sld::kDensKnots && SLD_PAIR_IV == sld::kPairIv &&
                  SLD_DENS_IV == sld::kDensIv,
              "split-form potential table offsets");
#include "sld_common.cuh"
#include "sld_ctx.cuh"
#include "sld_host.h"

namespace {

const double kBoltz = 8.617343e-5;
const double kLight = 299792458e0;
const double kUtoeV = 931.494028e6 / kLight / kLight;

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            std::fprintf(stderr, "sld: %s failed: %s\n", #call,    \
                         cudaGetErrorString(e_));                  \
            return SLD_ERR_CUDA;                                   \
        }                                                          \
    } while (0)

}  // namespace


namespace {

void use_set(sld_ctx* c, int k) {
    c->cur = k;
    c->D = dev_set(c, k);
}

int check_flags(sld_ctx* c) {
    unsigned err = 0;
    CK(cudaStreamSynchronize(c->st));
    CK(cudaMemcpy(&err, &c->D.ctl->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err & SLD_FLAG_CAPACITY) return SLD_ERR_CAPACITY;
    if (err & SLD_FLAG_TABLE) return SLD_ERR_TABLE;
    if (err & SLD_FLAG_NAN) return SLD_ERR_NAN;
    if (err & SLD_FLAG_WAIT) return SLD_ERR_TIMEOUT;
    return SLD_OK;
}

int launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "sld: launch failed: %s\n", cudaGetErrorString(e));
        return SLD_ERR_CUDA;
    }
    return SLD_OK;
}

// One core_ds call: forward sweep, backward sweep.
// core_ds (core_ds_CPU.cpp:35-83).  fields: store H, HL and sum J at each
// atom's last visit, as the reference's calculate_spin does; the step graph
// passes false where the same step overwrites them before anything reads
// them (the first core_ds of a step; with eltemp, calculate_temperature
// recomputes all three).
// noise_drawn: the caller launched this call's visit records already
void enqueue_ds(sld_ctx* c, const Dev& D, double dt, int& eoff, bool fields = true,
                bool noise_drawn = false) {
    const auto& G = c->G;
    double dt_half = dt / 2e0;
    if (c->P.spinlang && !noise_drawn) launch_spin_noise(D, c->st, eoff, dt_half);
    if (sweep_uses_flow() && !D.hint) {
        launch_sweep_flow(D, c->st, c->flow, dt_half, fields);
        if (c->P.spinlang) eoff += 2;
        return;
    }
    for (int g = 0; g < G.ngroups; ++g)
        launch_sweep(D, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g],
                     dt_half, false, fields);
    if (c->P.spinlang) ++eoff;
    for (int g = G.ngroups - 1; g >= 0; --g)
        launch_sweep(D, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g],
                     dt_half, true, fields);
    if (c->P.spinlang) ++eoff;
}
void enqueue_ds(sld_ctx* c, double dt, int& eoff) { enqueue_ds(c, c->D, dt, eoff); }

void enqueue_dp(sld_ctx* c, const Dev& D, double dt, int& eoff, bool temp = false,
                bool defer_scale = false) {
    launch_dp(D, c->st, dt, eoff, temp, defer_scale);
    if (c->P.lattlang) ++eoff;
}
void enqueue_dp(sld_ctx* c, double dt, int& eoff) { enqueue_dp(c, c->D, dt, eoff); }

// core.cpp:31-76 (spin-lattice branch) plus the main-loop bookkeeping, as
// two branches of one graph.  The second branch runs what does not read the
// spins beside the sweeps:
//   main:   links | dp(dt/2) | ds(dt/2) ........ | ds(dt/2) | force(magnetic) | dp(dt/2) | Te ...
//   second:  core_dTe(dt/2), visit records of the first ds | dr | rho + lists | force(EAM)
//            ... fold of the magnetic part (beside Te)
// The lists and rho of this step go to the other buffer set, so the first
// sweep still reads the previous ones; the step ends with that set current.
// MD (core.cpp:38-56 without spins): links | dp | dr | rho | forces | dp
void enqueue_step_md(sld_ctx* c) {
    double dt = c->P.step;
    int eoff = 0;
    const Dev Dc = dev_set(c, c->cur), Dn = dev_set(c, 1 - c->cur);
    cudaStream_t M = c->st;
    launch_links(Dc, M, false, c->scan_blocks);
    if (c->P.eltemp) launch_dte(Dc, M, dt / 2e0);
    enqueue_dp(c, Dc, dt / 2e0, eoff);
    launch_dr(Dc, M, dt);
    launch_pairs(Dn, M, true);
    launch_force(Dn, M);
    c->force_volume = Dn.box_volume;
    enqueue_dp(c, Dn, dt / 2e0, eoff);
    if (c->P.eltemp) {
        launch_temperature(Dn, M);
        launch_dte(Dn, M, dt / 2e0);
        if (c->P.renormalize_energy) launch_energy_check(Dn, M, 1);
    }
    launch_advance(Dn, M, eoff, 1);
}

// SDH, SDHL (core.cpp:41-48): the spins on a fixed lattice, core_ds(step);
// the energies of the force pass every step (the reference forms them at
// print-out steps only; nothing else reads them).  Both buffer sets hold the
// same lists and rho (sld_set_state), so the alternation of the step graphs
// changes nothing.
void enqueue_step_spin(sld_ctx* c) {
    double dt = c->P.step;
    int eoff = 0;
    const Dev Dc = dev_set(c, c->cur);
    cudaStream_t M = c->st;
    if (c->P.eltemp) launch_dte(Dc, M, dt / 2e0);
    enqueue_ds(c, Dc, dt, eoff, !c->P.eltemp);
    launch_force(Dc, M);
    if (c->P.eltemp) {
        launch_temperature(Dc, M);
        launch_dte(Dc, M, dt / 2e0);
        if (c->P.renormalize_energy) launch_energy_check(Dc, M, 1);
    }
    launch_advance(Dc, M, eoff, 1);
}

void enqueue_step(sld_ctx* c) {
    if (!c->D.spin) return enqueue_step_md(c);
    if (!c->D.latt) return enqueue_step_spin(c);
    double dt = c->P.step;
    int eoff = 0;
    const Dev Dc = dev_set(c, c->cur), Dn = dev_set(c, 1 - c->cur);
    static const bool one_stream = getenv("SLD_ONE_STREAM") && getenv("SLD_ONE_STREAM")[0] == '1';
    cudaStream_t M = c->st, A = one_stream ? c->st : c->st2;
    cudaEvent_t* ev = c->fork_ev;
    // The first core_ds's visit records read Te, rho and the noise counters,
    // not the momenta: the side branch writes them while the main branch
    // runs the first kick (the second core_ds's must wait for the first
    // sweep, which reads the same records, and stay in place)
    const bool early_noise = c->P.spinlang != 0;
    const int eoff_ds1 = eoff + (c->P.lattlang ? 1 : 0);   // after the first kick's draw
    if (c->P.eltemp) {
        cudaEventRecord(ev[0], M);
        cudaStreamWaitEvent(A, ev[0], 0);
        launch_dte(Dc, A, dt / 2e0);
        cudaEventRecord(ev[1], A);
        launch_links(Dc, M, false, c->scan_blocks);
        if (early_noise) {
            // the records read each atom's Te node, which the links rewrite
            cudaEventRecord(ev[5], M);
            cudaStreamWaitEvent(A, ev[5], 0);
            launch_spin_noise(Dc, A, eoff_ds1, dt / 2e0 / 2e0);
            cudaEventRecord(ev[4], A);
        }
        cudaStreamWaitEvent(M, ev[1], 0);
    } else {
        if (early_noise) {
            cudaEventRecord(ev[0], M);
            cudaStreamWaitEvent(A, ev[0], 0);
            launch_spin_noise(Dc, A, eoff_ds1, dt / 2e0 / 2e0);
            cudaEventRecord(ev[4], A);
        }
        launch_links(Dc, M, false, c->scan_blocks);
    }
    // The first kick's rescale_momentum scales the momenta in the drift, on
    // the side branch: the main branch reads no momenta before the second
    // kick, which runs after the side branch's EAM forces
    enqueue_dp(c, Dc, dt / 2e0, eoff, false, true);
    cudaEventRecord(ev[0], M);
    cudaStreamWaitEvent(A, ev[0], 0);
    launch_dr(Dc, A, dt, true);
    launch_pairs(Dn, A, true);
    cudaEventRecord(ev[2], A);
    launch_force_eam(Dn, A);
    cudaEventRecord(ev[3], A);
    if (early_noise) cudaStreamWaitEvent(M, ev[4], 0);
    enqueue_ds(c, Dc, dt / 2e0, eoff, false, early_noise);
    cudaStreamWaitEvent(M, ev[2], 0);
    enqueue_ds(c, Dn, dt / 2e0, eoff, !c->P.eltemp);
    // The magnetic force pass reads the spins and the exchange rows, not what
    // the EAM pass writes: it runs beside it, into buffers of its own (Dm).
    // The last kick adds the two forces; the fold into f, vir and stress runs
    // on the side branch beside the rest of the step.
    // On a Te mesh, calculate_temperature's per-atom terms are summed where
    // their inputs are final: the spin terms by the magnetic force pass
    // (after the last sweep; the exchange field from the spins it gathers
    // anyway) and the kinetic ones by the last kick's rescale.
    Dev Dm = Dn;
    Dm.fm = c->fm;
    Dm.virm = c->virm;
    Dm.stressm = c->stressm;
    const bool temp_fused = c->P.eltemp && Dn.te_mesh > 0;
    if (temp_fused) launch_temperature_begin(Dn, M);
    launch_force_mag(Dm, M, temp_fused);
    cudaStreamWaitEvent(M, ev[3], 0);
    c->force_volume = Dn.box_volume;
    enqueue_dp(c, Dm, dt / 2e0, eoff, temp_fused);
    cudaEventRecord(ev[0], M);
    cudaStreamWaitEvent(A, ev[0], 0);
    launch_fold_mag(Dm, A);
    cudaEventRecord(ev[1], A);
    if (c->P.eltemp) {
        if (temp_fused) launch_temperature_end(Dn, M);
        else launch_temperature(Dn, M);
        launch_dte(Dn, M, dt / 2e0);
        if (c->P.renormalize_energy) launch_energy_check(Dn, M, 1);
    }
    cudaStreamWaitEvent(M, ev[1], 0);
    launch_advance(Dn, M, eoff, 1);
}

// The cells of a colour group are independent, so their order within the
// group is free.  A thread walks one cell, and a warp takes as long as its
// fullest cell: ordering each group by atom count (taken after the links of
// the context's first set_state) gives the 32 cells of a warp about the same
// walk.  Counts change little over a run, and the order affects only speed.
int order_groups_by_count(sld_ctx* c) {
    auto& G = c->G;
    std::vector<int> cnt(G.ncells);
    if (cudaMemcpy(cnt.data(), c->D.cell_count, sizeof(int) * G.ncells, cudaMemcpyDeviceToHost))
        return SLD_ERR_CUDA;
    for (int g = 0; g < G.ngroups; ++g)
        std::stable_sort(G.gcells.begin() + G.gstart[g], G.gcells.begin() + G.gstart[g + 1],
                         [&](int a, int b) { return cnt[a] > cnt[b]; });
    if (cudaMemcpy(c->d_gcells, G.gcells.data(), sizeof(int) * G.ncells, cudaMemcpyHostToDevice))
        return SLD_ERR_CUDA;
    return SLD_OK;
}

// FP32 pair pre-test margin (k_pair.cu) for the cells of G.  A pair-vector
// component is at most three products M_ab d_b of the cell matrix and
// fixed-point differences (each below 3 cells), each rounded: with B the
// largest row sum of |M| over three cells, a component moves by at most
// e = 4 B 2^-24, and r^2 near the cutoff by 2 r_max sqrt(3) e + 3 e^2 plus the
// FP32 rounding of the sum.  The margin is twice that.
float pair_margin(const sld::HostGeom& G) {
    const double rx = std::fabs(G.d[0]) / G.nx + std::fabs(G.d[1]) / G.ny + std::fabs(G.d[3]) / G.nz;
    const double ry = std::fabs(G.d[2]) / G.ny + std::fabs(G.d[4]) / G.nz;
    const double rz = std::fabs(G.d[5]) / G.nz;
    const double B = 3.0 * std::max(rx, std::max(ry, rz));
    const double e = 4.0 * B * std::ldexp(1.0, -24);
    const double rm = G.rcut_max;
    const double bound = 2.0 * rm * std::sqrt(3.0) * e + 3.0 * e * e + 4.0 * std::ldexp(rm * rm, -23);
    return (float)(2.0 * bound);
}

// initial_quantum_noise (quantum_noise_CPU.cpp:75-104): the quantum
// thermostat's filter from the spectrum hbar w (1/2 + n(w)) at 2 Nf
// frequencies up to pi/h, h = Msteps_quantum step/2 (Dammak et al., Phys.
// Rev. Lett. 103, 190601 (2009); Barrat and Rodney, J. Stat. Phys. 144, 679
// (2011))
std::vector<double> quantum_filter(const sld_params& P) {
    const double hbar = 6.58211899e-16, pi = 3.141592653589793238462e0;
    const int Nf = P.nfrequency_quantum, Nf2 = 2 * Nf;
    const double h = P.msteps_quantum * P.step / 2e0;
    const double dw = pi / h / (double)Nf, T = P.temperature * kBoltz;
    std::vector<double> Ht(Nf2), H(Nf2, 0.0);
    for (int i = 0; i < Nf2; ++i) {
        int k = i - Nf;
        double w = dw * (double)k;
        Ht[i] = std::sqrt(hbar * std::fabs(w) * (0.5e0 + 1e0 / std::expm1(hbar * std::fabs(w) / T)));
        Ht[i] *= (w * h / 2e0) / std::sin(w * h / 2e0);
        if (k == 0) Ht[i] = std::sqrt(T);
    }
    for (int i = 0; i < Nf2; ++i) {
        for (int j = 0; j < Nf2; ++j) {
            int k = j - Nf;
            H[i] += Ht[j] * std::cos(pi / (double)Nf * (double)k * (double)(i - Nf));
        }
        H[i] /= (double)Nf2;
    }
    return H;
}

// the box or the time step changes between steps (sld_scale)
bool dynamic_step(const sld_ctx* c) {
    return c->P.change_step || c->P.pressure_control || c->P.stress_control;
}

int validate(const sld_params* p) {
    if (!p) return SLD_ERR_ARG;
    if (!(p->box[0] > 0 && p->box[2] > 0 && p->box[5] > 0)) return SLD_ERR_ARG;
    if (!(p->step > 0) || !(p->atmass > 0) || !(p->temperature >= 0)) return SLD_ERR_ARG;
    if (!(p->rcut_pot > 0 && p->rcut_mag > 0 && p->rcut_max > 0)) return SLD_ERR_ARG;
    if (p->rcut_pot > p->rcut_max || p->rcut_mag > p->rcut_max) return SLD_ERR_ARG;
    if (p->hamiltonian < SLD_HAM_SLDHL || p->hamiltonian > SLD_HAM_SDHL) return SLD_ERR_ARG;
    const bool latt = p->hamiltonian <= SLD_HAM_MD, spin = p->hamiltonian != SLD_HAM_MD;
    // thermostats of degrees of freedom the Hamiltonian has; with eltemp the
    // thermostats of all of them (the reference would not compile the rest)
    if ((p->spinlang && !spin) || (p->lattlang && !latt)) return SLD_ERR_ARG;
    if (p->eltemp && !((p->spinlang || !spin) && (p->lattlang || !latt))) return SLD_ERR_ARG;
    if (p->localcolmot && !p->lattlang) return SLD_ERR_ARG;
    if ((p->pressure_control || p->stress_control) && !latt) return SLD_ERR_ARG;
    // the quantum thermostat colours the lattice noise; its filter is made for
    // one time step (quantum_noise_CPU.cpp:79-81)
    if (p->quantum_noise &&
        (!p->lattlang || p->change_step || p->msteps_quantum < 1 || p->nfrequency_quantum < 1))
        return SLD_ERR_ARG;
    if (p->precision != SLD_FP64 && p->precision != SLD_SPLIT &&
        p->precision != SLD_FP64_ANALYTIC)
        return SLD_ERR_ARG;
    if (p->te_mesh != 0 && p->te_mesh < 3) return SLD_ERR_ARG;
    return SLD_OK;
}

}  // namespace

extern "C" {

const char* sld_error_string(int code) {
    switch (code) {
    case SLD_OK: return "ok";
    case SLD_ERR_ARG: return "invalid argument";
    case SLD_ERR_CUDA: return "CUDA runtime error";
    case SLD_ERR_GEOMETRY: return "fewer than 3 link cells along an axis";
    case SLD_ERR_CAPACITY: return "a link cell holds more atoms than supported";
    case SLD_ERR_TABLE: return "r or rho outside the potential table";
    case SLD_ERR_NAN: return "non-finite value produced";
    case SLD_ERR_IO: return "file could not be read";
    case SLD_ERR_STATE: return "call out of order";
    case SLD_ERR_NOMEM: return "device allocation failed";
    case SLD_ERR_TIMEOUT: return "a bounded device-side wait ran out (spin-sweep schedule)";
    default: return "unknown error";
    }
}

// Potential tables on the device, shared by every context on that device
// with the same table range (they depend only on rcut_max): 8 tables of 10^6
// doubles, built once (about a second on the host) and kept until the
// process exits.  Replicas of one system then share one copy.
struct DevTables {
    double* t[sld::kTabCount];
    double inv_r, inv_rho;
    double landau[4];
};
static std::mutex g_tab_mu;
static std::map<std::pair<int, uint64_t>, DevTables> g_tabs;

static int device_tables(int dev, double rmax, DevTables* out) {
    std::lock_guard<std::mutex> lock(g_tab_mu);
    uint64_t bits;
    std::memcpy(&bits, &rmax, sizeof(bits));
    auto it = g_tabs.find({dev, bits});
    if (it != g_tabs.end()) {
        *out = it->second;
        return SLD_OK;
    }
    sld::Tables T;
    sld::build_tables(T, rmax);
    DevTables d{};
    d.inv_r = T.inv_r;
    d.inv_rho = T.inv_rho;
    for (int k = 0; k < 4; ++k) d.landau[k] = T.landau[k];
    for (int k = 0; k < sld::kTabCount; ++k) {
        if (cudaMalloc(&d.t[k], sizeof(double) * sld::kNInput) != cudaSuccess) {
            for (int q = 0; q < k; ++q) cudaFree(d.t[q]);
            return SLD_ERR_NOMEM;
        }
        if (cudaMemcpy(d.t[k], T.t[k].data(), sizeof(double) * sld::kNInput,
                       cudaMemcpyHostToDevice) != cudaSuccess) {
            for (int q = 0; q <= k; ++q) cudaFree(d.t[q]);
            return SLD_ERR_CUDA;
        }
    }
    g_tabs[{dev, bits}] = d;
    *out = d;
    return SLD_OK;
}

int sld_params_default(sld_params* o) {
    if (!o) return SLD_ERR_ARG;
    std::memset(o, 0, sizeof(*o));
    o->step = 1e-15;
    o->temperature = 300e0;
    o->atmass = 55.847e0;
    o->gamma_L_over_mass = 6e11;
    o->gamma_S_HL = 5.88e13;
    o->gamma_S_H = 8e-3;
    o->hamiltonian = SLD_HAM_SLDHL;
    o->msteps_quantum = 50;
    o->nfrequency_quantum = 150;
    o->rcut_pot = 4.1001;
    o->rcut_mag = 3.7501;
    o->rcut_max = 4.1001;
    o->min_length_link_cell = 4.11;
    o->kappa_e = 80e0;
    o->random_seed = 1234;
    o->te_nloop = 50;
    o->interval_of_print_out = 1;
    o->interval_of_config_out = 1000;
    o->interval_of_scale_pressure = 1;
    o->interval_of_scale_stress = 1;
    o->baro_damping_time = 1e-13;
    o->displace_limit = 0.01;
    o->phi_limit = 2e0 * 3.141592653589793238462e0 / 10e0;
    o->precision = SLD_FP64;
    return SLD_OK;
}

int sld_create(sld_ctx** out, const sld_params* prm, int natom, const double* r,
               const double* p, const double* s, const double* te_K) {
    if (!out || !r || !p || !s || natom <= 0) return SLD_ERR_ARG;
    *out = nullptr;
    int rc = validate(prm);
    if (rc) return rc;
    // the split form's neighbour lists pack a slot (27 bits) with a cell code
    if (prm->precision == SLD_SPLIT && natom >= (1 << 27)) return SLD_ERR_CAPACITY;
    sld_ctx* c = new (std::nothrow) sld_ctx();
    if (!c) return SLD_ERR_NOMEM;
    c->P = *prm;
    if (c->P.te_nloop <= 0) c->P.te_nloop = 50;
    if (c->P.interval_of_print_out <= 0) c->P.interval_of_print_out = 1;
    if (c->P.interval_of_config_out <= 0) c->P.interval_of_config_out = 1000;
    if (c->P.interval_of_scale_pressure <= 0) c->P.interval_of_scale_pressure = 1;
    if (c->P.interval_of_scale_stress <= 0) c->P.interval_of_scale_stress = 1;

    // geometry, link cells, colour groups, initial order (host)
    std::vector<double> r0(r, r + 3 * (size_t)natom);
    rc = sld::setup_geometry(c->P, natom, r0, c->G, c->id_of_slot, c->slot_of_id);
    if (rc) { delete c; return rc; }
    const auto& G = c->G;

    DevGuard dev_guard(prm->device);   // the caller's device is current again on return
    if (!dev_guard.ok) { delete c; return SLD_ERR_CUDA; }
    sweep_init();
    dte_init(prm->device);
    // the main branch (spin sweeps: few, latency-bound blocks) gets the
    // highest priority so that the side branch's wide grids fill in around it
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
        delete c;
        return SLD_ERR_CUDA;
    }
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    if (cudaStreamCreateWithPriority(&c->st2, cudaStreamNonBlocking, prio_lo) != cudaSuccess) {
        sld_destroy(c);
        return SLD_ERR_CUDA;
    }
    for (int k = 0; k < 6; ++k) cudaEventCreateWithFlags(&c->fork_ev[k], cudaEventDisableTiming);

    DevTables T;
    rc = device_tables(prm->device, G.rcut_max, &T);
    if (rc) { sld_destroy(c); return rc; }

    Dev& D = c->D;
    for (int k = 0; k < 6; ++k) { D.d[k] = G.d[k]; D.inv[k] = G.inv[k]; }
    for (int k = 0; k < 3; ++k) D.box_len[k] = G.box_len[k];
    D.box_volume = G.box_volume;
    D.rcut_pot = prm->rcut_pot;
    D.rcut_mag = prm->rcut_mag;
    D.rcut_max = G.rcut_max;
    D.rcut_pot_sq = prm->rcut_pot * prm->rcut_pot;
    D.rcut_mag_sq = prm->rcut_mag * prm->rcut_mag;
    D.rcut_max_sq = G.rcut_max * G.rcut_max;
    D.pair_loose = pair_margin(G);
    D.atmass = prm->atmass * kUtoeV * (1e-10 * 1e-10);
    D.temperature = prm->temperature * kBoltz;
    D.gamma_L = prm->gamma_L_over_mass * D.atmass;
    D.gamma_S_HL = prm->gamma_S_HL;
    D.gamma_S_H = prm->gamma_S_H;
    D.ham = prm->hamiltonian;
    D.latt = (D.ham == SLD_HAM_SLDHL || D.ham == SLD_HAM_SLDH || D.ham == SLD_HAM_MD) ? 1 : 0;
    D.spin = D.ham != SLD_HAM_MD ? 1 : 0;
    D.landau_on = (D.ham == SLD_HAM_SLDHL || D.ham == SLD_HAM_SDHL) ? 1 : 0;
    D.hc = D.ham == SLD_HAM_SLDHL ? 1 : 0;
    D.hint = (D.ham == SLD_HAM_SDH || D.ham == SLD_HAM_SLDH) ? 1 : 0;
    D.tune = Tune{0, 0, 0, 0, -1, 0, 0, 0, 0, 1};
    {
        // starting launch shapes: caps on the CTAs per SM of the sweeps and
        // of the side branch's pair and EAM passes, the hub core_dTe kernel's
        // threads (tests compare shapes; the autotuner chooses its own)
        auto cap = [](const char* name) {
            const char* v = getenv(name);
            const int k = v ? atoi(v) : 0;
            return k > 0 && k <= 32 ? k : 0;
        };
        D.tune.sweep_cap = cap("SLD_SWEEP_CAP");
        D.tune.pair_cap = cap("SLD_PAIR_CAP");
        D.tune.force_cap = cap("SLD_FORCE_CAP");
        const char* gp = getenv("SLD_GRAPH_PRIO");
        if (gp && gp[0] == '0') D.tune.graph_prio = 0;
        const char* t = getenv("SLD_DTE_THREADS");
        if (t) {
            const int k = atoi(t);
            if (k == 256 || k == 512 || k == 1024) D.tune.dte_threads = k;
        }
    }
    D.quantum = prm->quantum_noise ? 1 : 0;
    D.qM = prm->msteps_quantum;
    D.step = prm->step;
    D.inv_r = T.inv_r;
    D.inv_rho = T.inv_rho;
    for (int k = 0; k < 4; ++k) D.landau[k] = T.landau[k];
    D.kappa_e = prm->kappa_e;
    D.natom = natom;
    D.nx = G.nx; D.ny = G.ny; D.nz = G.nz; D.ncells = G.ncells;
    D.tx = G.tx; D.ty = G.ty; D.tz = G.tz; D.nte = G.nte; D.te_mesh = prm->te_mesh;
    D.seed = (unsigned)prm->random_seed;
    D.replica = (unsigned)prm->replica;
    D.spinlang = prm->spinlang; D.lattlang = prm->lattlang; D.eltemp = prm->eltemp;
    D.localcolmot = prm->localcolmot; D.renormalize = prm->renormalize_energy;
    D.print_every = c->P.interval_of_print_out;
    D.te_nloop = c->P.te_nloop;
    D.small_grid = (G.nx < 4 || G.ny < 4 || G.nz < 4) ? 1 : 0;
    D.split = prm->precision == SLD_SPLIT ? 1 : 0;
    D.analytic = prm->precision == SLD_FP64_ANALYTIC ? 1 : 0;
    {
        double jd[7];
        sld::pot_join_data(jd);
        D.pot32 = Pot32{(float)jd[0], (float)jd[1], (float)jd[2], (float)jd[3],
                        (float)jd[4], (float)jd[5], (float)jd[6]};
    }
    float cubic_h[sld::kCubicFloats];
    double cubic64_h[sld::kCubicDoubles];
    sld::pot_cubic_tables(cubic_h, cubic64_h);

    size_t n = (size_t)natom;
    bool ok = true;
    double* const* tabs = T.t;
    D.tF = tabs[sld::kF]; D.tdF = tabs[sld::kdF]; D.tf = tabs[sld::kf]; D.tdf = tabs[sld::kdf];
    D.tphi = tabs[sld::kPhi]; D.tdphi = tabs[sld::kdPhi]; D.tJ = tabs[sld::kJ]; D.tdJ = tabs[sld::kdJ];

    ok = c->alloc(&D.r, n) == 0 && c->alloc(&D.p, n) == 0 && c->alloc(&D.f, n) == 0 &&
         c->alloc(&D.s, n) == 0 && c->alloc(&D.H, n) == 0 && c->alloc(&D.HL, n) == 0 &&
         c->alloc(&c->rho_set[0], n) == 0 && c->alloc(&c->rho_set[1], n) == 0 &&
         c->alloc(&D.pe, n) == 0 && c->alloc(&D.ke, n) == 0 &&
         c->alloc(&D.me, n) == 0 && c->alloc(&D.me0, n) == 0 && c->alloc(&D.vir, n) == 0 &&
         c->alloc(&D.sumJ, n) == 0 && c->alloc(&D.stress, 6 * n) == 0 &&
         c->alloc(&D.cell_of, n) == 0 && c->alloc(&D.id, n) == 0 && c->alloc(&D.stamp, n) == 0 &&
         c->alloc(&D.cell_start, (size_t)G.ncells) == 0 &&
         c->alloc(&D.cell_count, (size_t)G.ncells) == 0 &&
         c->alloc(&D.cell_atoms, n) == 0 && c->alloc(&D.cell_fill, (size_t)G.ncells) == 0 &&
         c->alloc(&D.nbr, (size_t)SLD_MAXNB * n) == 0 && c->alloc(&D.nbr_n, n) == 0 &&
         c->alloc(&c->jl_set[0], (size_t)SLD_MAXJ * n) == 0 &&
         c->alloc(&c->jl_set[1], (size_t)SLD_MAXJ * n) == 0 &&
         c->alloc(&c->jln_set[0], n) == 0 && c->alloc(&c->jln_set[1], n) == 0 &&
         c->alloc(&D.dF, n) == 0;
    if (prm->spinlang) ok = ok && c->alloc(&D.vrec, 2 * n) == 0;
    if (D.spin && D.latt)
        ok = ok && c->alloc(&c->fm, n) == 0 && c->alloc(&c->virm, n) == 0 &&
             c->alloc(&c->stressm, 6 * n) == 0;
    if (prm->precision == SLD_SPLIT) ok = ok && c->alloc(&D.s32, n) == 0;
    ok = ok && c->alloc(&D.fxs, n) == 0 && c->alloc(&D.cell_slot, n) == 0;
    if (prm->precision == SLD_SPLIT)
        ok = ok && c->alloc(&D.fxa, n) == 0 && c->alloc(&D.nbk, (size_t)SLD_MAXNB * n) == 0;
    {
        float* cub = nullptr;
        double* cub64 = nullptr;
        ok = ok && c->alloc(&cub, sld::kCubicFloats) == 0 && c->alloc(&cub64, sld::kCubicDoubles) == 0;
        if (ok) {
            cudaMemcpy(cub, cubic_h, sizeof(cubic_h), cudaMemcpyHostToDevice);
            cudaMemcpy(cub64, cubic64_h, sizeof(cubic64_h), cudaMemcpyHostToDevice);
        }
        D.cubic = cub;
        D.cubic64 = cub64;
    }
    for (int k = 0; k < 2 && ok; ++k) {
        if (prm->precision == SLD_SPLIT)
            ok = c->alloc(&c->jvf_set[k], (size_t)SLD_MAXJ * n) == 0 &&
                 c->alloc(&c->jlk_set[k], (size_t)SLD_MAXJ * n) == 0;
        else ok = c->alloc(&c->jv_set[k], (size_t)SLD_MAXJ * n) == 0;
    }
    if (ok) use_set(c, 0);
    c->scan_blocks = div_up(G.ncells, 1024);
    ok = ok && c->alloc(&D.scan_tmp, (size_t)c->scan_blocks) == 0;
    if (prm->te_mesh > 0) {
        ok = ok && c->alloc(&D.node, n) == 0 && c->alloc(&D.te_count, (size_t)G.nte) == 0;
    } else {
        D.node = D.cell_of;
        D.te_count = D.cell_count;
    }
    int nte = G.nte;
    ok = ok && c->alloc(&D.Te, nte) == 0 && c->alloc(&D.Ee, nte) == 0 && c->alloc(&D.Tl, nte) == 0 &&
         c->alloc(&D.TsR, nte) == 0 && c->alloc(&D.TsL, nte) == 0 && c->alloc(&D.Gel, nte) == 0 &&
         c->alloc(&D.Ges, nte) == 0 && c->alloc(&D.acc, 9 * (size_t)nte) == 0 &&
         c->alloc(&D.trl, 4 * (size_t)nte) == 0;
    c->red_cap = std::max(div_up(natom, 128), div_up(G.ncells, 128)) + 8;
    ok = ok && c->alloc(&D.red, 8 * (size_t)c->red_cap) == 0;
    ok = ok && c->alloc(&D.ctl, 1) == 0 && c->alloc(&c->d_avg, 16) == 0;
    ok = ok && c->alloc(&c->d_chk, SLD_CHK_ATOM * (size_t)div_up(natom, 256) + SLD_CHK_N) == 0;
    if (ok && prm->quantum_noise) {
        std::vector<double> h = quantum_filter(*prm);
        double* qH = nullptr;
        ok = c->alloc(&qH, h.size()) == 0 && c->alloc(&D.qnoise, n) == 0 &&
             cudaMemcpy(qH, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
        D.qH = qH;
        D.qNf2 = (int)h.size();
    }
    ok = ok && c->alloc(&c->d_gcells, (size_t)G.ncells) == 0;
    ok = ok && c->alloc(&c->d_te_gcells, (size_t)nte) == 0 &&
         c->alloc(&c->d_te_gstart, G.te_gstart.size()) == 0 &&
         c->alloc(&c->d_te_color, (size_t)nte) == 0 &&
         c->alloc(&c->d_te_ltasks, G.te_ltasks.size()) == 0 &&
         c->alloc(&c->d_te_lstart, G.te_lstart.size()) == 0 &&
         c->alloc(&c->d_te_lnb, G.te_lnb.size() / 8) == 0;
    if (!ok) { sld_destroy(c); return SLD_ERR_NOMEM; }
    if (G.te_nlevels > 0) {
        cudaMemcpy(c->d_te_lnb, G.te_lnb.data(), sizeof(unsigned short) * G.te_lnb.size(),
                   cudaMemcpyHostToDevice);
        cudaMemcpy(c->d_te_ltasks, G.te_ltasks.data(), sizeof(unsigned short) * G.te_ltasks.size(),
                   cudaMemcpyHostToDevice);
        cudaMemcpy(c->d_te_lstart, G.te_lstart.data(), sizeof(int) * G.te_lstart.size(),
                   cudaMemcpyHostToDevice);
    }
    cudaMemcpy(c->d_gcells, G.gcells.data(), sizeof(int) * G.ncells, cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_te_gcells, G.te_gcells.data(), sizeof(int) * nte, cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_te_gstart, G.te_gstart.data(), sizeof(int) * G.te_gstart.size(),
               cudaMemcpyHostToDevice);
    {
        std::vector<unsigned char> col(nte, 0);
        for (int g = 0; g < G.te_ngroups; ++g)
            for (int m = G.te_gstart[g]; m < G.te_gstart[g + 1]; ++m)
                col[G.te_gcells[m]] = (unsigned char)g;
        cudaMemcpy(c->d_te_color, col.data(), nte, cudaMemcpyHostToDevice);
        D.te_color = c->d_te_color;
    }
    {
        // spin-sweep tasks: at most 32 cells of one colour group each, forward
        // groups 0..G-1 then backward G-1..0 (core_ds_CPU.cpp:35-83)
        std::vector<int4> tasks;
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 0; k < G.ngroups; ++k) {
                const int g = pass == 0 ? k : G.ngroups - 1 - k;
                for (int m = G.gstart[g]; m < G.gstart[g + 1]; m += 32)
                    tasks.push_back(make_int4(pass, m, std::min(32, G.gstart[g + 1] - m), g));
            }
        std::vector<unsigned char> grp(G.ncells, 0);
        for (int g = 0; g < G.ngroups; ++g)
            for (int m = G.gstart[g]; m < G.gstart[g + 1]; ++m) grp[G.gcells[m]] = (unsigned char)g;
        int4* d_tasks = nullptr;
        unsigned char* d_grp = nullptr;
        ok = c->alloc(&d_tasks, tasks.size()) == 0 && c->alloc(&d_grp, (size_t)G.ncells) == 0 &&
             c->alloc(&c->flow.cell_flag, (size_t)G.ncells) == 0 && c->alloc(&c->flow.sync, 2) == 0;
        if (!ok) { sld_destroy(c); return SLD_ERR_NOMEM; }
        cudaMemcpy(d_tasks, tasks.data(), sizeof(int4) * tasks.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(d_grp, grp.data(), (size_t)G.ncells, cudaMemcpyHostToDevice);
        c->flow.tasks = d_tasks;
        c->flow.ntasks = (int)tasks.size();
        c->flow.gcells = c->d_gcells;
        c->flow.cell_group = d_grp;
    }
    D.te_gcells = c->d_te_gcells;
    D.te_gstart = c->d_te_gstart;
    D.te_ngroups = G.te_ngroups;
    D.te_ltasks = c->d_te_ltasks;
    D.te_lstart = c->d_te_lstart;
    D.te_lnb = c->d_te_lnb;
    D.te_nlevels = G.te_nlevels;

    // Te per Te cell (map_cells.cpp:128-158), stored in eV as the reference does
    std::vector<double> te(nte);
    for (int k = 0; k < nte; ++k) te[k] = te_K ? te_K[k] * kBoltz : D.temperature;
    cudaMemcpy(D.Te, te.data(), sizeof(double) * nte, cudaMemcpyHostToDevice);
    std::vector<int> idv(c->id_of_slot);
    cudaMemcpy(D.id, idv.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    // the set-up copies and memsets above ran on the default stream; the
    // engine's own stream does not order against it
    if (cudaDeviceSynchronize() != cudaSuccess) { sld_destroy(c); return SLD_ERR_CUDA; }

    rc = sld_set_state(c, r0.data(), p, s);
    if (rc) { sld_destroy(c); return rc; }
    *out = c;
    return SLD_OK;
}

int sld_set_state(sld_ctx* c, const double* r, const double* p, const double* s) {
    if (!c || !r || !p || !s) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    Dev& D = c->D;
    const size_t n = (size_t)D.natom;
    // The caller's arrays go to the device as they are, into the neighbour
    // list's memory (192 bytes per atom; the pair pass below rebuilds the
    // list), and one kernel puts them in slot order with the periodic wrap,
    // |s| and the kinetic energy.
    double* raw = reinterpret_cast<double*>(D.nbr);
    CK(cudaMemcpyAsync(raw, r, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(raw + 3 * n, p, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(raw + 6 * n, s, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    launch_load_state(D, c->st, raw, raw + 3 * n, raw + 6 * n);
    Ctl z{};
    CK(cudaMemcpyAsync(D.ctl, &z, sizeof(Ctl), cudaMemcpyHostToDevice, c->st));
    // a fresh start: the barostats' clocks at total_time 0 (initial.cpp:92-97)
    c->last_t_pressure = c->last_t_stress = 0.0;
    c->pressure0 = 0.0;
    for (int q = 0; q < 6; ++q) c->ave_stress[q] = 0.0;
    // initialize(): links, rho, forces, cell temperatures, reference energy
    launch_links(D, c->st, true, c->scan_blocks);
    launch_pairs(D, c->st, true);
    // a fixed lattice: both buffer sets get the (only) lists and densities
    if (!D.latt) launch_pairs(dev_set(c, 1 - c->cur), c->st, true);
    c->lists_stale = false;
    launch_force(D, c->st);
    c->force_volume = D.box_volume;
    if (c->P.eltemp) {
        launch_temperature(D, c->st);
        if (c->P.renormalize_energy) launch_energy_check(D, c->st, 0);
    }
    int rc = launch_status();
    if (rc) return rc;
    rc = check_flags(c);
    if (rc) return rc;
    if (c->groups_ordered) return SLD_OK;
    c->groups_ordered = true;
    return order_groups_by_count(c);
}

void sld_destroy(sld_ctx* c) {
    if (!c) return;
    DevGuard sld_dev_guard_(c->P.device);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    for (int k = 0; k < 2; ++k)
        if (c->step_graphs[k]) cudaGraphExecDestroy(c->step_graphs[k]);
    for (int k = 0; k < 6; ++k)
        if (c->fork_ev[k]) cudaEventDestroy(c->fork_ev[k]);
    if (c->st2) cudaStreamDestroy(c->st2);
    for (void* q : c->allocs) cudaFree(q);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

int sld_links(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    launch_links(c->D, c->st, false, c->scan_blocks);
    return launch_status();
}

int sld_calculate_rho(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    launch_pairs(c->D, c->st, true);
    c->lists_stale = false;
    return launch_status();
}

// refresh the neighbour lists (not rho) when positions moved since
static void fresh_lists(sld_ctx* c) {
    if (c->lists_stale) {
        launch_pairs(c->D, c->st, false);
        c->lists_stale = false;
    }
}

int sld_calculate_force_energy(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    fresh_lists(c);
    launch_force(c->D, c->st);
    c->force_volume = c->D.box_volume;
    return launch_status();
}

int sld_core_ds(sld_ctx* c, double dt) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    fresh_lists(c);
    int eoff = 0;
    enqueue_ds(c, dt, eoff);
    launch_advance(c->D, c->st, eoff, 0);
    return launch_status();
}

int sld_core_dp(sld_ctx* c, double dt) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    int eoff = 0;
    enqueue_dp(c, dt, eoff);
    launch_advance(c->D, c->st, eoff, 0);
    return launch_status();
}

int sld_core_dr(sld_ctx* c, double dt) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    launch_dr(c->D, c->st, dt);
    c->lists_stale = true;
    return launch_status();
}

int sld_core_dTe(sld_ctx* c, double dt) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (!c->P.eltemp) return SLD_OK;
    launch_dte(c->D, c->st, dt);
    return launch_status();
}

int sld_calculate_temperature(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (!c->P.eltemp) return SLD_OK;
    fresh_lists(c);
    launch_temperature(c->D, c->st);
    return launch_status();
}

int sld_run(sld_ctx* c, int nsteps) {
    if (!c || nsteps < 0) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    fresh_lists(c);
    if (dynamic_step(c)) {
        // box or time step set by sld_scale between steps: launch directly
        CK(cudaEventRecord(c->ev0, c->st));
        for (int k = 0; k < nsteps; ++k) {
            enqueue_step(c);
            use_set(c, 1 - c->cur);
        }
        CK(cudaEventRecord(c->ev1, c->st));
        return launch_status();
    }
    for (int k = 0; k < 2; ++k) {
        if (c->step_graphs[k]) continue;
        int saved = c->cur;
        use_set(c, k);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue_step(c);
            // always end the capture, so that the stream leaves capture mode
            // even when a launch inside it failed
            e = cudaStreamEndCapture(c->st, &g);
        }
        // with node priorities the sweeps' branch (the high-priority stream)
        // gets its CTAs dispatched before the side branch's waiting ones
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&c->step_graphs[k], g,
                                     c->D.tune.graph_prio ? cudaGraphInstantiateFlagUseNodePriority : 0);
        if (g) cudaGraphDestroy(g);
        use_set(c, saved);
        if (e != cudaSuccess) {
            c->step_graphs[k] = nullptr;
            cudaGetLastError();
            return SLD_ERR_CUDA;
        }
    }
    CK(cudaEventRecord(c->ev0, c->st));
    for (int k = 0; k < nsteps; ++k) {
        CK(cudaGraphLaunch(c->step_graphs[c->cur], c->st));
        use_set(c, 1 - c->cur);
    }
    CK(cudaEventRecord(c->ev1, c->st));
    return SLD_OK;
}

// ---------------------------------------------------------------------
// batched replicas

struct sld_batch {
    std::vector<sld_ctx*> ctx;
    std::vector<int> base;             // each context's buffer set when graph 0 was made
    cudaStream_t st = nullptr;
    cudaEvent_t root = nullptr, done = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> join;     // one per context
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    int device = 0;
};

static void batch_drop_graphs(sld_batch* b) {
    for (int k = 0; k < 2; ++k)
        if (b->graphs[k]) {
            cudaGraphExecDestroy(b->graphs[k]);
            b->graphs[k] = nullptr;
        }
}

// graph k: every context at buffer set base ^ k
static int batch_capture(sld_batch* b, int k) {
    std::vector<int> saved(b->ctx.size());
    for (size_t q = 0; q < b->ctx.size(); ++q) {
        saved[q] = b->ctx[q]->cur;
        use_set(b->ctx[q], b->base[q] ^ k);
    }
    cudaGraph_t g = nullptr;
    int rc = SLD_OK;
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = SLD_ERR_CUDA;
    if (rc == SLD_OK) {
        cudaEventRecord(b->root, b->st);
        for (size_t q = 0; q < b->ctx.size(); ++q) {
            sld_ctx* c = b->ctx[q];
            cudaStreamWaitEvent(c->st, b->root, 0);
            enqueue_step(c);
            cudaEventRecord(b->join[q], c->st);
            cudaStreamWaitEvent(b->st, b->join[q], 0);
        }
        if (cudaStreamEndCapture(b->st, &g) != cudaSuccess) rc = SLD_ERR_CUDA;
    }
    if (rc == SLD_OK &&
        cudaGraphInstantiate(&b->graphs[k], g,
                             b->ctx[0]->D.tune.graph_prio ? cudaGraphInstantiateFlagUseNodePriority
                                                          : 0) != cudaSuccess)
        rc = SLD_ERR_CUDA;
    if (g) cudaGraphDestroy(g);
    for (size_t q = 0; q < b->ctx.size(); ++q) use_set(b->ctx[q], saved[q]);
    return rc;
}

int sld_batch_create(sld_batch** out, sld_ctx* const* ctxs, int n) {
    if (!out || !ctxs || n <= 0) return SLD_ERR_ARG;
    *out = nullptr;
    std::vector<sld_ctx*> v(ctxs, ctxs + n);
    for (int q = 0; q < n; ++q) {
        if (!v[q] || v[q]->P.device != v[0]->P.device || dynamic_step(v[q])) return SLD_ERR_ARG;
        for (int r = 0; r < q; ++r)
            if (v[r] == v[q]) return SLD_ERR_ARG;
    }
    sld_batch* b = new (std::nothrow) sld_batch;
    if (!b) return SLD_ERR_NOMEM;
    b->ctx = v;
    b->device = v[0]->P.device;
    b->join.assign(n, nullptr);
    DevGuard dev_guard(b->device);
    bool ok = dev_guard.ok &&
              cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->root, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess;
    for (int q = 0; q < n && ok; ++q)
        ok = cudaEventCreateWithFlags(&b->join[q], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        sld_batch_destroy(b);
        return SLD_ERR_CUDA;
    }
    *out = b;
    return SLD_OK;
}

int sld_batch_run(sld_batch* b, int nsteps) {
    if (!b || nsteps < 0) return SLD_ERR_ARG;
    DevGuard dev_guard(b->device);
    if (!dev_guard.ok) return SLD_ERR_CUDA;
    // the batch stream follows whatever is queued on each context's stream
    for (size_t q = 0; q < b->ctx.size(); ++q) {
        sld_ctx* c = b->ctx[q];
        fresh_lists(c);
        CK(cudaEventRecord(b->join[q], c->st));
        CK(cudaStreamWaitEvent(b->st, b->join[q], 0));
    }
    // graphs are made for the contexts' buffer sets relative to each other;
    // a context stepped on its own since then has shifted, so remake them
    bool same = b->base.size() == b->ctx.size();
    for (size_t q = 0; same && q < b->ctx.size(); ++q)
        same = (b->ctx[q]->cur ^ b->base[q]) == (b->ctx[0]->cur ^ b->base[0]);
    if (!same) {
        batch_drop_graphs(b);
        b->base.resize(b->ctx.size());
        for (size_t q = 0; q < b->ctx.size(); ++q) b->base[q] = b->ctx[q]->cur;
    }
    for (int k = 0; k < 2; ++k)
        if (!b->graphs[k]) {
            int rc = batch_capture(b, k);
            if (rc) return rc;
        }
    int k = b->ctx[0]->cur ^ b->base[0];
    CK(cudaEventRecord(b->ev0, b->st));
    for (int s = 0; s < nsteps; ++s) {
        CK(cudaGraphLaunch(b->graphs[k], b->st));
        for (sld_ctx* c : b->ctx) use_set(c, 1 - c->cur);
        k ^= 1;
    }
    CK(cudaEventRecord(b->ev1, b->st));
    // later work on each context follows the batch
    CK(cudaEventRecord(b->done, b->st));
    for (sld_ctx* c : b->ctx) CK(cudaStreamWaitEvent(c->st, b->done, 0));
    return launch_status();
}

int sld_batch_last_run_ms(sld_batch* b, double* out) {
    if (!b || !out) return SLD_ERR_ARG;
    CK(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    *out = ms;
    return SLD_OK;
}

void sld_batch_destroy(sld_batch* b) {
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    batch_drop_graphs(b);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {b->root, b->done, b->ev0, b->ev1})
        if (e) cudaEventDestroy(e);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

int sld_profile_step(sld_ctx* c, double* ms) {
    if (!c || !ms) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (!c->D.latt || !c->D.spin) return SLD_ERR_ARG;   // the spin-lattice step's phases
    fresh_lists(c);
    cudaEvent_t ev[2];
    CK(cudaEventCreate(&ev[0]));
    CK(cudaEventCreate(&ev[1]));
    for (int k = 0; k < SLD_PHASES; ++k) ms[k] = 0.0;
    auto timed = [&](int slot, auto&& fn) {
        cudaEventRecord(ev[0], c->st);
        fn();
        cudaEventRecord(ev[1], c->st);
        cudaEventSynchronize(ev[1]);
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        ms[slot] += t;
    };
    double dt = c->P.step;
    int eoff = 0;
    const Dev Dc = dev_set(c, c->cur), Dn = dev_set(c, 1 - c->cur);
    timed(0, [&] { launch_links(Dc, c->st, false, c->scan_blocks); });
    if (c->P.eltemp) timed(1, [&] { launch_dte(Dc, c->st, dt / 2e0); });
    timed(2, [&] { enqueue_dp(c, Dc, dt / 2e0, eoff); });
    timed(3, [&] { enqueue_ds(c, Dc, dt / 2e0, eoff, false); });
    timed(4, [&] { launch_dr(Dc, c->st, dt); });
    timed(5, [&] { launch_pairs(Dn, c->st, true); });
    timed(3, [&] { enqueue_ds(c, Dn, dt / 2e0, eoff, !c->P.eltemp); });
    timed(6, [&] { launch_force(Dn, c->st); });
    c->force_volume = Dn.box_volume;
    timed(2, [&] { enqueue_dp(c, Dn, dt / 2e0, eoff); });
    if (c->P.eltemp) {
        timed(7, [&] { launch_temperature(Dn, c->st); });
        timed(1, [&] { launch_dte(Dn, c->st, dt / 2e0); });
        if (c->P.renormalize_energy) timed(8, [&] { launch_energy_check(Dn, c->st, 1); });
    }
    timed(9, [&] { launch_advance(Dn, c->st, eoff, 1); });
    use_set(c, 1 - c->cur);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return launch_status();
}

int sld_step_kernel_count(sld_ctx* c, int* out) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    cudaGraph_t g = nullptr;
    fresh_lists(c);
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c);
    CK(cudaStreamEndCapture(c->st, &g));
    size_t n = 0;
    CK(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    CK(cudaGraphGetNodes(g, nodes.data(), &n));
    int k = 0;
    for (size_t i = 0; i < n; ++i) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(nodes[i], &t);
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    cudaGraphDestroy(g);
    *out = k;
    return SLD_OK;
}

int sld_last_run_ms(sld_ctx* c, double* out) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *out = ms;
    return SLD_OK;
}

int sld_sync(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    int rc = launch_status();
    if (rc) return rc;
    return check_flags(c);
}

// a per-atom field in caller order on the device: out[width id(k) + w] for
// the atom in slot k (x, y, z of a double4 field, or width consecutive doubles)
__global__ void k_pack_caller(const Dev D, const double* __restrict__ src, int src_width,
                              int width, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.natom) return;
    const size_t i = (size_t)D.id[k];
    const double* a = src + (size_t)src_width * k;
    for (int w = 0; w < width; ++w) out[(size_t)width * i + w] = a[w];
}

long sld_get(sld_ctx* c, const char* field, double* out, long cap) {
    if (!c || !field || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    Dev& D = c->D;
    size_t n = (size_t)D.natom;
    std::string f(field);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return SLD_ERR_CUDA;
    // per-atom fields are put in caller order on the device and copied out in
    // one transfer (direct DMA when the caller's buffer is pinned)
    auto packed = [&](const double* src, int src_width, int width) -> long {
        if (cap < (long)(width * n)) return SLD_ERR_ARG;
        if (!c->d_stage && c->alloc(&c->d_stage, 6 * n) != SLD_OK) return SLD_ERR_NOMEM;
        k_pack_caller<<<div_up((long)n, 256), 256, 0, c->st>>>(D, src, src_width, width, c->d_stage);
        if (cudaMemcpyAsync(out, c->d_stage, sizeof(double) * width * n, cudaMemcpyDeviceToHost,
                            c->st) != cudaSuccess ||
            cudaStreamSynchronize(c->st) != cudaSuccess)
            return SLD_ERR_CUDA;
        return (long)(width * n);
    };
    auto vec4 = [&](double4* src) -> long {
        return packed(reinterpret_cast<const double*>(src), 4, 3);
    };
    auto scal = [&](double* src, int width) -> long { return packed(src, width, width); };
    auto percell = [&](double* src, double scale) -> long {
        size_t m = (size_t)D.nte;
        if (cap < (long)m) return SLD_ERR_ARG;
        if (cudaMemcpy(out, src, sizeof(double) * m, cudaMemcpyDeviceToHost)) return SLD_ERR_CUDA;
        for (size_t k = 0; k < m; ++k) out[k] *= scale;
        return (long)m;
    };
    if (f == "r") return vec4(D.r);
    if (f == "p") return vec4(D.p);
    if (f == "f") return vec4(D.f);
    if (f == "s") return vec4(D.s);
    if (f == "H") return vec4(D.H);
    if (f == "HL") return vec4(D.HL);
    if (f == "s0") {
        if (cap < (long)n) return SLD_ERR_ARG;
        std::vector<double4> h(n);
        if (cudaMemcpy(h.data(), D.s, sizeof(double4) * n, cudaMemcpyDeviceToHost)) return SLD_ERR_CUDA;
        for (size_t k = 0; k < n; ++k) out[c->id_of_slot[k]] = h[k].w;
        return (long)n;
    }
    if (f == "rho") return scal(D.rho, 1);
    if (f == "pe") return scal(D.pe, 1);
    if (f == "ke") return scal(D.ke, 1);
    if (f == "me") return scal(D.me, 1);
    if (f == "me0") return scal(D.me0, 1);
    if (f == "vir") return scal(D.vir, 1);
    if (f == "sum_Jij_sj" || f == "sumJ") return scal(D.sumJ, 1);
    if (f == "stress") return scal(D.stress, 6);
    if (f == "local_volume") {
        if (cap < (long)n) return SLD_ERR_ARG;
        for (size_t k = 0; k < n; ++k) out[k] = c->force_volume / D.natom;
        return (long)n;
    }
    if (f == "cell" || f == "node") {
        if (cap < (long)n) return SLD_ERR_ARG;
        std::vector<int> h(n);
        int* src = f == "cell" ? D.cell_of : D.node;
        if (cudaMemcpy(h.data(), src, sizeof(int) * n, cudaMemcpyDeviceToHost)) return SLD_ERR_CUDA;
        for (size_t k = 0; k < n; ++k) out[c->id_of_slot[k]] = h[k];
        return (long)n;
    }
    if (f == "Te") return percell(D.Te, 1.0 / kBoltz);
    if (f == "Ee") return percell(D.Ee, 1.0);
    if (f == "Tl") return percell(D.Tl, 1.0);
    if (f == "Ts_R") return percell(D.TsR, 1.0);
    if (f == "Ts_L") return percell(D.TsL, 1.0);
    if (f == "Gel") return percell(D.Gel, 1.0);
    if (f == "Ges") return percell(D.Ges, 1.0);
    if (f == "count") {
        size_t m = (size_t)D.nte;
        if (cap < (long)m) return SLD_ERR_ARG;
        std::vector<int> h(m);
        if (cudaMemcpy(h.data(), D.te_count, sizeof(int) * m, cudaMemcpyDeviceToHost)) return SLD_ERR_CUDA;
        for (size_t k = 0; k < m; ++k) out[k] = h[k];
        return (long)m;
    }
    return SLD_ERR_ARG;
}

int sld_get_cell_lists(sld_ctx* c, int* out) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    size_t n = (size_t)c->D.natom;
    CK(cudaStreamSynchronize(c->st));
    std::vector<int> h(n);
    CK(cudaMemcpy(h.data(), c->D.cell_atoms, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < n; ++k) out[k] = c->id_of_slot[h[k]];
    return SLD_OK;
}

int sld_averages(sld_ctx* c, double* out10) {
    if (!c || !out10) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    launch_averages(c->D, c->st, c->d_avg);
    CK(cudaMemcpyAsync(out10, c->d_avg, sizeof(double) * 10, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return launch_status();
}

int sld_virial(sld_ctx* c, double* out) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    launch_virial(c->D, c->st);
    CK(cudaMemcpyAsync(out, &c->D.ctl->virial, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return SLD_OK;
}

int sld_total_time(sld_ctx* c, double* out) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    CK(cudaMemcpyAsync(out, &c->D.ctl->total_time, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return SLD_OK;
}

// check() (check.cpp:31-47) without its renormalisation, which the step
// itself runs: one line each appended to enr-, tmp-, str-, prs- and spn-,
// in that order, with the reference's expressions (check_energy_CPU.cpp:35-138,
// check_temperature_CPU.cpp:35-157, check_stress_CPU.cpp:35-79,
// check_pressure_CPU.cpp:35-59, check_spin_CPU.cpp:35-76).
int sld_check(sld_ctx* c, const char* dir, const char* out_body, int current_step) {
    if (!c || !out_body) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if ((current_step + 1) % c->P.interval_of_print_out != 0) return SLD_OK;
    const Dev& D = c->D;
    double* part = c->d_chk;
    double* tot = c->d_chk + SLD_CHK_ATOM * (size_t)div_up(D.natom, 256);
    launch_check_sums(D, c->st, part, tot);
    int rc = launch_status();
    if (rc) return rc;
    double S[SLD_CHK_N];
    Ctl ctl;
    CK(cudaMemcpyAsync(S, tot, sizeof S, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&ctl, D.ctl, sizeof ctl, cudaMemcpyDeviceToHost, c->st));
    rc = check_flags(c);
    if (rc) return rc;

    const double n = (double)D.natom, t = ctl.total_time;
    const double* d = c->G.d;
    const bool el = c->P.eltemp != 0;
    const double density = n / c->G.box_volume;
    double v[16];
    int k = 0;

    // check_energy: with renormalizeEnergy the averages it formed before
    // moving the error into the electrons at this step
    double pe = S[SLD_CHK_PE] / n, ke = S[SLD_CHK_KE] / n;
    double me = S[SLD_CHK_ME] / n, me0 = S[SLD_CHK_ME0] / n, Ee = S[SLD_CHK_EE] / n;
    if (el && c->P.renormalize_energy && ctl.chk_tag == (long long)current_step + 2) {
        pe = ctl.chk[0]; ke = ctl.chk[1]; me = ctl.chk[2]; me0 = ctl.chk[3]; Ee = ctl.chk[4];
    }
    // the columns of the Hamiltonian's degrees of freedom
    v[k++] = t;
    if (D.latt) { v[k++] = pe; v[k++] = ke; }
    if (D.spin) { v[k++] = me; v[k++] = me0; }
    if (el) v[k++] = Ee;
    rc = sld::append_line(sld::out_path(dir, "enr-", out_body, -1), current_step, v, k);
    if (rc) return rc;

    // check_temperature
    k = 0;
    v[k++] = t;
    if (D.latt) v[k++] = S[SLD_CHK_KE] * 2e0 / 3e0 / n / kBoltz;
    if (D.spin) v[k++] = S[SLD_CHK_RUP] / S[SLD_CHK_RDN] / 2e0 / kBoltz;
    if (D.landau_on) v[k++] = S[SLD_CHK_LUP] / S[SLD_CHK_LDN] / kBoltz;
    if (el) v[k++] = S[SLD_CHK_TE] / (double)D.nte / kBoltz;
    rc = sld::append_line(sld::out_path(dir, "tmp-", out_body, -1), current_step, v, k);
    if (rc) return rc;
    if (D.latt) {
        // check_stress: per-atom stresses in eV/A^3, averaged and converted to GPa
        double st[6];
        for (int q = 0; q < 6; ++q) st[q] = S[SLD_CHK_STRESS + q] * (160.217653e0 / n);
        k = 0;
        v[k++] = t;
        for (int q = 0; q < 6; ++q) v[k++] = d[q];
        v[k++] = density;
        v[k++] = (st[0] + st[1] + st[2]) / 3e0;
        for (int q = 0; q < 6; ++q) v[k++] = st[q];
        rc = sld::append_line(sld::out_path(dir, "str-", out_body, -1), current_step, v, k);
        if (rc) return rc;

        // check_pressure
        double tmp = 2e0 / 3e0 * S[SLD_CHK_KE] / n;
        double pressure0 = density * (tmp - S[SLD_CHK_VIR] / (3e0 * n));
        pressure0 *= 160.217653e0;
        c->pressure0 = pressure0;
        for (int q = 0; q < 6; ++q) c->ave_stress[q] = st[q];
        k = 0;
        v[k++] = t;
        for (int q = 0; q < 6; ++q) v[k++] = d[q];
        v[k++] = density;
        v[k++] = pressure0;
        rc = sld::append_line(sld::out_path(dir, "prs-", out_body, -1), current_step, v, k);
        if (rc) return rc;
    }
    if (!D.spin) return SLD_OK;

    // check_spin: magnetisation m = -g s (spilady.h:60)
    const double el_g = 2.0023193043622e0;
    double ax = S[SLD_CHK_SX] / n, ay = S[SLD_CHK_SY] / n, az = S[SLD_CHK_SZ] / n;
    double mx = -el_g * ax, my = -el_g * ay, mz = -el_g * az;
    k = 0;
    v[k++] = t;
    v[k++] = ax; v[k++] = ay; v[k++] = az;
    v[k++] = std::sqrt(ax * ax + ay * ay + az * az);
    v[k++] = mx; v[k++] = my; v[k++] = mz;
    v[k++] = std::sqrt(mx * mx + my * my + mz * mz);
    return sld::append_line(sld::out_path(dir, "spn-", out_body, -1), current_step, v, k);
}

// write_config (write_config.cpp:31-169): con-<out_body>_NNNN.dat and, with
// eltemp, cel-<out_body>_NNNN.dat.
int sld_write_config(sld_ctx* c, const char* dir, const char* out_body, int current_step,
                     int flags) {
    if (!c || !out_body) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    const int every = c->P.interval_of_config_out;
    if (!(current_step == -1 || current_step == -2 || (current_step + 1) % every == 0))
        return SLD_OK;
    int n_output = current_step == -1 ? 0 : current_step == -2 ? 9999 : current_step / every + 1;
    double t = 0;
    int rc = sld_total_time(c, &t);
    if (rc) return rc;
    const long n = c->D.natom;

    // columns (write_config.cpp:100-127), by what the Hamiltonian has:
    // r [p f stress(6) rho ke pe] [s s0 Heff_H [Heff_L] me me0] local_volume
    const Dev& D = c->D;
    struct Col { const char* field; int width; };
    std::vector<Col> cols = {{"r", 3}};
    if (D.latt)
        for (Col k : {Col{"p", 3}, Col{"f", 3}, Col{"stress", 6}, Col{"rho", 1}, Col{"ke", 1},
                      Col{"pe", 1}})
            cols.push_back(k);
    int hcol = -1, lcol = -1, ncol = 0;
    for (const Col& k : cols) ncol += k.width;
    if (D.spin) {
        cols.push_back({"s", 3}); cols.push_back({"s0", 1}); ncol += 4;
        hcol = ncol; cols.push_back({"H", 3}); ncol += 3;
        if (D.landau_on) { lcol = ncol; cols.push_back({"HL", 3}); ncol += 3; }
        cols.push_back({"me", 1}); cols.push_back({"me0", 1}); ncol += 2;
    }
    cols.push_back({"local_volume", 1});
    ncol += 1;
    std::vector<double> table((size_t)n * ncol), tmp((size_t)n * 6);
    int at = 0;
    for (const Col& col : cols) {
        long got = sld_get(c, col.field, tmp.data(), (long)tmp.size());
        if (got < 0) return (int)got;
        for (long i = 0; i < n; ++i)
            for (int w = 0; w < col.width; ++w)
                table[(size_t)i * ncol + at + w] = tmp[(size_t)i * col.width + w];
        at += col.width;
    }
    if (flags & SLD_WRITE_HEFF_AS_REFERENCE) {
        // write_config.cpp:120,123 print the x component in the y column
        for (long i = 0; i < n; ++i) {
            double* row = &table[(size_t)i * ncol];
            if (hcol >= 0) row[hcol + 1] = row[hcol];
            if (lcol >= 0) row[lcol + 1] = row[lcol];
        }
    }
    static const char* kType[] = {"SLDHL", "SLDH", "MD", "SDH", "SDHL"};
    rc = sld::write_con_file(sld::out_path(dir, "con-", out_body, n_output), n, t, c->G.d,
                             kType[D.ham], "Fe", ncol, table.data());
    if (rc || !c->P.eltemp) return rc;

    // cel-: cells x-major (ix outermost), centre, Te (K) [Tl] [Ts_R] [Ts_L]
    const auto& G = c->G;
    const bool mesh = c->P.te_mesh > 0;
    const int ax = mesh ? G.tx : G.nx, ay = mesh ? G.ty : G.ny, az = mesh ? G.tz : G.nz;
    const long m = G.nte;
    std::vector<const char*> names = {"Te"};
    if (D.latt) names.push_back("Tl");
    if (D.spin) names.push_back("Ts_R");
    if (D.landau_on) names.push_back("Ts_L");
    const int nv = (int)names.size(), w = 3 + nv;
    std::vector<double> vals((size_t)m * nv);
    for (int q = 0; q < nv; ++q) {
        long got = sld_get(c, names[q], vals.data() + (size_t)q * m, m);
        if (got < 0) return (int)got;
    }
    const double* d = G.d;
    std::vector<double> cel((size_t)m * w);
    size_t row = 0;
    for (int ix = 0; ix < ax; ++ix)
        for (int iy = 0; iy < ay; ++iy)
            for (int iz = 0; iz < az; ++iz) {
                long i = ix + (long)iy * ax + (long)iz * ax * ay;
                double qx = (ix + 0.5) / ax, qy = (iy + 0.5) / ay, qz = (iz + 0.5) / az;
                double* o = &cel[row++ * w];
                o[0] = d[0] * qx + d[1] * qy + d[3] * qz;
                o[1] = d[2] * qy + d[4] * qz;
                o[2] = d[5] * qz;
                for (int q = 0; q < nv; ++q) o[3 + q] = vals[(size_t)q * m + i];
            }
    return sld::write_cel_file(sld::out_path(dir, "cel-", out_body, n_output), m, t, d, w, cel.data());
}

// A new box (upper-triangular d): the host geometry, the device copy of the
// box and the FP32 pre-test margin follow it; the exchange lists are rebuilt
// from the moved positions before the next step, keeping the densities
// (calculate_spin walks the pairs of the current positions while rho is the
// last calculate_rho's, calculate_spin_CPU.cpp).
static void apply_box(sld_ctx* c, const double* d) {
    auto& G = c->G;
    for (int k = 0; k < 6; ++k) G.d[k] = d[k];
    sld::box_derived(G);
    for (int k = 0; k < 6; ++k) { c->D.d[k] = G.d[k]; c->D.inv[k] = G.inv[k]; }
    for (int k = 0; k < 3; ++k) c->D.box_len[k] = G.box_len[k];
    c->D.box_volume = G.box_volume;
    c->D.pair_loose = pair_margin(G);
    for (int k = 0; k < 6; ++k) c->P.box[k] = d[k];
    c->lists_stale = true;
}

int sld_scale(sld_ctx* c, int current_step, double* out3) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    const sld_params& P = c->P;
    double t = 0.0;
    int rc = sld_total_time(c, &t);
    if (rc) return rc;
    const double ftmass = 100e0;   // the piston's fictitious mass, GPa
    if (P.stress_control && (current_step + 1) % P.interval_of_scale_stress == 0) {
        // scale_stress_CPU.cpp:35-85; the statements run in this order, so
        // later ones read the components updated before them
        double delta_time = t - c->last_t_stress;
        c->last_t_stress = t;
        double pre = delta_time / P.baro_damping_time / ftmass;
        const double* a = c->ave_stress;   // 11 22 33 12 23 31
        const double* w = P.stress;        // xx yx yy zx zy zz
        double fxx = pre * (a[0] - w[0]), fyx = pre * (a[3] - w[1]);
        double fyy = pre * (a[1] - w[2]), fzx = pre * (a[5] - w[3]);
        double fzy = pre * (a[4] - w[4]), fzz = pre * (a[2] - w[5]);
        double xx = c->G.d[0], yx = c->G.d[1], yy = c->G.d[2];
        double zx = c->G.d[3], zy = c->G.d[4], zz = c->G.d[5];
        xx = (1e0 + fxx) * xx;
        yx = (1e0 + fxx) * yx + fyx * (yy + xx) / 2e0;
        yy = (1e0 + fyy) * yy;
        zx = (1e0 + fxx) * zx + fzx * (zz + xx) / 2e0;
        zy = (1e0 + fyy) * zy + fzy * (zz + yy) / 2e0;
        zz = (1e0 + fzz) * zz;
        double old_inv[6], nd[6] = {xx, yx, yy, zx, zy, zz};
        for (int k = 0; k < 6; ++k) old_inv[k] = c->G.inv[k];
        apply_box(c, nd);
        launch_reshape_positions(c->D, c->st, old_inv);
        rc = launch_status();
        if (rc) return rc;
    }
    if (P.pressure_control && (current_step + 1) % P.interval_of_scale_pressure == 0) {
        // scale_pressure_CPU.cpp:35-60
        double delta_time = t - c->last_t_pressure;
        c->last_t_pressure = t;
        double factor = std::pow(
            1e0 + delta_time / P.baro_damping_time * (c->pressure0 - P.pressure) / ftmass, 1e0 / 3e0);
        double nd[6];
        for (int k = 0; k < 6; ++k) nd[k] = c->G.d[k] * factor;
        apply_box(c, nd);
        launch_scale_positions(c->D, c->st, factor);
        rc = launch_status();
        if (rc) return rc;
    }
    double res[3] = {0.0, 0.0, P.step};
    if (P.change_step) {
        // scale_step_CPU.cpp:35-100
        double* part = c->d_chk;
        double* m = c->d_chk + 2 * (size_t)div_up(c->D.natom, 256);
        launch_max_p_h(c->D, c->st, part, m);
        double h[2];
        CK(cudaMemcpyAsync(h, m, sizeof h, cudaMemcpyDeviceToHost, c->st));
        rc = check_flags(c);
        if (rc) return rc;
        const double hbar = 6.58211899e-16;   // eV s (spilady.h:58)
        double step = P.step;
        // the lattice's and the spins' limits, by what the Hamiltonian has
        double displace_max = c->D.latt ? std::sqrt(h[0]) / c->D.atmass * step : 0.0;
        double phi_max = c->D.spin ? std::sqrt(h[1]) / hbar * step : 0.0;
        if ((c->D.latt && displace_max > P.displace_limit) || (c->D.spin && phi_max > P.phi_limit))
            step *= 0.80;
        else
            step *= 1.05;
        c->P.step = step;
        c->D.step = step;
        res[0] = displace_max; res[1] = phi_max; res[2] = step;
    }
    if (out3)
        for (int k = 0; k < 3; ++k) out3[k] = res[k];
    return SLD_OK;
}

// ---------------------------------------------------------------------
// external field and force (control.h's extfield, extforce)

// kernel arguments changed: the step graphs are captured again at the next run
static void drop_step_graphs(sld_ctx* c) {
    cudaStreamSynchronize(c->st);
    for (int k = 0; k < 2; ++k)
        if (c->step_graphs[k]) {
            cudaGraphExecDestroy(c->step_graphs[k]);
            c->step_graphs[k] = nullptr;
        }
}

// caller-order natom x 3 values, times k, into a slot-order device array
static int set_per_atom(sld_ctx* c, double4** buf, double4** dev_ptr, const double* v, double k) {
    if (!v) {
        if (*dev_ptr) {
            *dev_ptr = nullptr;
            drop_step_graphs(c);
        }
        return SLD_OK;
    }
    const size_t n = (size_t)c->D.natom;
    if (!*buf && c->alloc(buf, n) != SLD_OK) return SLD_ERR_NOMEM;
    std::vector<double4> h(n);
    for (size_t q = 0; q < n; ++q) {
        const double* x = v + 3 * (size_t)c->id_of_slot[q];
        h[q] = make_double4(k * x[0], k * x[1], k * x[2], 0.0);
    }
    CK(cudaMemcpyAsync(*buf, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (*dev_ptr != *buf) {
        *dev_ptr = *buf;
        drop_step_graphs(c);
    }
    return SLD_OK;
}

int sld_set_external_field(sld_ctx* c, const double* H) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (H && !c->D.spin) return SLD_ERR_ARG;
    int rc = set_per_atom(c, &c->hext_buf, &c->D.hext, H, 1.0);
    if (rc) return rc;
    // Before the first step this is the reference's initialize(), which sets
    // the field before the first force pass, cell temperatures and reference
    // energy (initial.cpp:58-60,78-87): those are formed again.  Later the
    // field takes effect from the next step.
    long long steps = 0;
    CK(cudaMemcpy(&steps, &c->D.ctl->steps, sizeof steps, cudaMemcpyDeviceToHost));
    if (steps != 0) return SLD_OK;
    fresh_lists(c);
    launch_force(c->D, c->st);
    c->force_volume = c->D.box_volume;
    if (c->P.eltemp) {
        launch_temperature(c->D, c->st);
        if (c->P.renormalize_energy) launch_energy_check(c->D, c->st, 0);
    }
    return launch_status();
}

int sld_set_external_force(sld_ctx* c, const double* f) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (f && !c->D.latt) return SLD_ERR_ARG;
    return set_per_atom(c, &c->fext_buf, &c->D.fext, f, 1.0);
}

// extfield.in / extforce.in (external_field_CPU.cpp:37-49,
// external_force_CPU.cpp:37-48): natom, then one line "i x y z" per atom in
// atom order; fields in Tesla, converted to eV by -g muB
static int read_per_atom(sld_ctx* c, const char* path, std::vector<double>& v) {
    if (!path) return SLD_ERR_ARG;
    FILE* f = std::fopen(path, "r");
    if (!f) return SLD_ERR_IO;
    long n = 0;
    int rc = SLD_OK;
    if (std::fscanf(f, "%ld", &n) != 1 || n != c->D.natom) rc = SLD_ERR_IO;
    v.assign(3 * (size_t)c->D.natom, 0.0);
    for (long i = 0; i < n && rc == SLD_OK; ++i) {
        long idx;
        if (std::fscanf(f, "%ld %lf %lf %lf", &idx, &v[3 * i], &v[3 * i + 1], &v[3 * i + 2]) != 4)
            rc = SLD_ERR_IO;
    }
    std::fclose(f);
    return rc;
}

int sld_read_external_field(sld_ctx* c, const char* path) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    std::vector<double> v;
    int rc = read_per_atom(c, path, v);
    if (rc) return rc;
    const double el_g = 2.0023193043622e0, muB = 5.7883817555e-5;   // spilady.h:59-60
    for (double& x : v) x = (-el_g * muB) * x;
    return sld_set_external_field(c, v.data());
}

int sld_read_external_force(sld_ctx* c, const char* path) {
    if (!c) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    std::vector<double> v;
    int rc = read_per_atom(c, path, v);
    if (rc) return rc;
    return sld_set_external_force(c, v.data());
}

int sld_quantum_filter(sld_ctx* c, double* out, int n) {
    if (!c || !out) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (!c->D.quantum) return SLD_ERR_STATE;
    if (n < c->D.qNf2) return SLD_ERR_ARG;
    CK(cudaMemcpy(out, c->D.qH, sizeof(double) * c->D.qNf2, cudaMemcpyDeviceToHost));
    return c->D.qNf2;
}

// ---------------------------------------------------------------------
// autotuner of the launch shapes

// every device allocation of the context, for a tuning run that leaves the
// state as it found it
struct StateCopy {
    std::vector<void*> buf;
    int cur = 0;
    bool lists_stale = false;
    double force_volume = 0.0;
};

static int state_save(sld_ctx* c, StateCopy& s) {
    s.cur = c->cur;
    s.lists_stale = c->lists_stale;
    s.force_volume = c->force_volume;
    for (size_t k = 0; k < c->allocs.size(); ++k) {
        void* q = nullptr;
        if (cudaMalloc(&q, c->alloc_bytes[k]) != cudaSuccess) return SLD_ERR_NOMEM;
        s.buf.push_back(q);
        CK(cudaMemcpyAsync(q, c->allocs[k], c->alloc_bytes[k], cudaMemcpyDeviceToDevice, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return SLD_OK;
}

static int state_restore(sld_ctx* c, const StateCopy& s) {
    for (size_t k = 0; k < s.buf.size(); ++k)
        CK(cudaMemcpyAsync(c->allocs[k], s.buf[k], c->alloc_bytes[k], cudaMemcpyDeviceToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    use_set(c, s.cur);
    c->lists_stale = s.lists_stale;
    c->force_volume = s.force_volume;
    return SLD_OK;
}

static void state_free(StateCopy& s) {
    for (void* q : s.buf) cudaFree(q);
    s.buf.clear();
}

// device milliseconds of `steps` steps with the current launch shapes, from
// the saved state: one untimed step first (the graph capture), then the
// faster of two timed runs
static int trial(sld_ctx* c, const StateCopy& s, int steps, double* ms) {
    drop_step_graphs(c);
    int rc = state_restore(c, s);
    if (rc) return rc;
    if ((rc = sld_run(c, 1)) || (rc = sld_sync(c))) return rc;
    *ms = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
        double t = 0.0;
        if ((rc = sld_run(c, steps)) || (rc = sld_sync(c)) || (rc = sld_last_run_ms(c, &t)))
            return rc;
        *ms = std::min(*ms, t);
    }
    return SLD_OK;
}

int sld_autotune(sld_ctx* c, int steps, int* out8) {
    if (!c || steps < 1) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    if (dynamic_step(c)) return SLD_ERR_ARG;   // no captured step to time
    StateCopy s;
    int rc = state_save(c, s);
    if (rc) { state_free(s); return rc; }
    Tune& T = c->D.tune;
    double best = 0.0;
    rc = trial(c, s, steps, &best);
    // coordinate descent over the shapes, each from the current best
    struct Axis { int* field; std::vector<int> values; };
    std::vector<Axis> axes = {{&T.sweep_block, {64, 96, 128}},
                              {&T.sweep_cap, {0, 2, 3}},
                              {&T.pair_block, {64, 96, 128}},
                              {&T.force_block, {64, 96, 128}}};
    if (c->P.eltemp) {
        axes.push_back({&T.dte_mode, {0, 1, 2, 3}});
        axes.push_back({&T.dte_threads, {256, 512, 1024}});
        if (c->P.te_mesh > 0) axes.push_back({&T.temp_block, {64, 128}});
    }
    for (auto& ax : axes) {
        if (rc) break;
        int keep = *ax.field;
        for (int v : ax.values) {
            if (v == keep) continue;
            *ax.field = v;
            double ms = 0.0;
            rc = trial(c, s, steps, &ms);
            if (rc) break;
            // a shape must win by 1%: run-to-run noise is about that
            if (ms < 0.99 * best) { best = ms; keep = v; }
        }
        *ax.field = keep;
    }
    drop_step_graphs(c);
    int rc2 = state_restore(c, s);
    state_free(s);
    if (rc) return rc;
    if (rc2) return rc2;
    if (out8) {
        out8[0] = T.sweep_block; out8[1] = T.pair_block; out8[2] = T.force_block;
        out8[3] = T.temp_block; out8[4] = T.dte_mode; out8[5] = T.dte_threads;
        out8[6] = T.sweep_cap; out8[7] = 0;
    }
    return SLD_OK;
}

int sld_info(sld_ctx* c, int* o) {
    if (!c || !o) return SLD_ERR_ARG;
    SLD_DEVICE_OF(c);
    o[0] = c->D.natom; o[1] = c->G.ncells; o[2] = c->G.ngroups; o[3] = c->G.nte;
    o[4] = c->G.nx; o[5] = c->G.ny;
    return SLD_OK;
}

}  // extern "C"
