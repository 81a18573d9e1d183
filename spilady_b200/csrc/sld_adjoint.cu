// Gradients of the energy and of a force/field loss with respect to the
// potential's 36 parameters (include/sld.h: sld_adjoint_*), for one
// configuration and through an NVE spin-lattice trajectory.
//
// The trajectory gradient is reverse mode with checkpoints: the forward run
// keeps the state at every checkpoint; then, segment by segment from the
// last, the segment is run forward again from its checkpoint with every
// intermediate kept (positions, momenta before each rescaling, the spins
// before and after each sweep, link-cell lists, neighbour lists, densities),
// and its steps are reversed one by one (k_adjoint.cu).  The context's own
// state is put back at the end.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/sld.h"
#include "potential.h"
#include "sld_adjoint.cuh"
#include "sld_ctx.cuh"

namespace {

#define ACK(call)                                                       \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) {                                        \
            std::fprintf(stderr, "sld adjoint: %s failed: %s\n", #call, \
                         cudaGetErrorString(e_));                       \
            return SLD_ERR_CUDA;                                        \
        }                                                               \
    } while (0)

// device allocations freed together
struct Pool {
    std::vector<void*> p;
    bool ok = true;
    template <class T>
    T* get(size_t n) {
        void* q = nullptr;
        if (!ok || cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
            ok = false;
            return nullptr;
        }
        // cleared on the default stream, which does not order against the
        // engine's non-blocking stream: finished before any use of it there
        if (cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess) {
            ok = false;
            cudaFree(q);
            return nullptr;
        }
        p.push_back(q);
        return static_cast<T*>(q);
    }
    ~Pool() {
        for (void* q : p) cudaFree(q);
    }
};

// what a forward step reads or a reverse step needs again
struct Snap {
    double4 *r, *p, *s, *f;
    long long* stamp;
    int *cell_of, *cell_start, *cell_count, *cell_atoms, *cell_slot;
    int4* fxs;
    int4* fxa;                        // split form only
    int *nbr, *nbr_n;
    unsigned char* nbk;               // split form only
    Ctl* ctl;
};

// one step's intermediates
struct Tape {
    double4 *r0, *r1, *ppre1, *ppre2, *s0, *sA, *s1, *sB, *s2;
    double *rho1, *dF1;
    int *nbr, *nbr_n;                                         // built after the drift
    int *cell_start, *cell_count, *cell_atoms, *cell_of, *cell_slot;
};

struct Adj {
    sld_ctx* c = nullptr;
    Pool pool;
    AdjDev A{};
    AdjConst K{};
    double* el2 = nullptr;     // [E, L] of the last force pass
    int nb = 0;
    size_t n = 0, nc = 0, nnb = 0;
    double4* scratch_p = nullptr;
};

int alloc_adj(Adj& a, sld_ctx* c, const double* theta) {
    a.c = c;
    a.n = (size_t)c->D.natom;
    a.nc = (size_t)c->G.ncells;
    a.nnb = (size_t)SLD_MAXNB * a.n;
    a.nb = (int)((a.n + 127) / 128);
    size_t n = a.n;
    AdjDev& A = a.A;
    A.rho = a.pool.get<double>(n);
    A.dF = a.pool.get<double>(n);
    A.e = a.pool.get<double>(n);
    A.H = a.pool.get<double4>(n);
    A.part = a.pool.get<double>(2 * (size_t)a.nb);
    A.rb = a.pool.get<double4>(n);
    A.pb = a.pool.get<double4>(n);
    A.sb = a.pool.get<double4>(n);
    A.fb = a.pool.get<double4>(n);
    A.hb = a.pool.get<double4>(n);
    A.rhob = a.pool.get<double>(n);
    // block rows: a thread per atom, or a warp per atom or cell
    size_t nblk = std::max<size_t>((a.n + 3) / 4, (a.nc + 3) / 4) + 1;
    A.thb = a.pool.get<double>(nblk * ADJ_NTHETA);
    A.theta_bar = a.pool.get<double>(ADJ_NTHETA);
    a.el2 = a.pool.get<double>(2);
    a.scratch_p = a.pool.get<double4>(n);
    // colour group of every link cell
    std::vector<int> grp(a.nc, 0);
    const auto& G = c->G;
    for (int g = 0; g < G.ngroups; ++g)
        for (int k = G.gstart[g]; k < G.gstart[g + 1]; ++k) grp[G.gcells[k]] = g;
    int* dg = a.pool.get<int>(a.nc);
    if (!a.pool.ok) return SLD_ERR_NOMEM;
    ACK(cudaMemcpy(dg, grp.data(), sizeof(int) * a.nc, cudaMemcpyHostToDevice));
    A.cell_group = dg;
    // parameters and the ZBL end of the pair term's join
    for (int k = 0; k < ADJ_NTHETA; ++k) a.K.th[k] = theta[k];
    double jd[7];
    sld::pot_join_data(jd);
    a.K.y1 = jd[0];
    a.K.dy1 = jd[1];
    a.K.d2y1 = jd[2];
    a.K.zbl_as = jd[6];
    return SLD_OK;
}

int alloc_snap(Pool& pool, const Adj& a, Snap& s) {
    size_t n = a.n, nc = a.nc;
    s.r = pool.get<double4>(n);
    s.p = pool.get<double4>(n);
    s.s = pool.get<double4>(n);
    s.f = pool.get<double4>(n);
    s.stamp = pool.get<long long>(n);
    s.cell_of = pool.get<int>(n);
    s.cell_start = pool.get<int>(nc);
    s.cell_count = pool.get<int>(nc);
    s.cell_atoms = pool.get<int>(n);
    s.cell_slot = pool.get<int>(n);
    s.fxs = pool.get<int4>(n);
    s.fxa = a.c->D.fxa ? pool.get<int4>(n) : nullptr;
    s.nbk = a.c->D.nbk ? pool.get<unsigned char>(a.nnb) : nullptr;
    s.nbr = pool.get<int>(a.nnb);
    s.nbr_n = pool.get<int>(n);
    s.ctl = pool.get<Ctl>(1);
    return pool.ok ? SLD_OK : SLD_ERR_NOMEM;
}

int alloc_tape(Pool& pool, const Adj& a, Tape& t) {
    size_t n = a.n, nc = a.nc;
    double4** v[] = {&t.r0, &t.r1, &t.ppre1, &t.ppre2, &t.s0, &t.sA, &t.s1, &t.sB, &t.s2};
    for (auto q : v) *q = pool.get<double4>(n);
    t.rho1 = pool.get<double>(n);
    t.dF1 = pool.get<double>(n);
    t.nbr = pool.get<int>(a.nnb);
    t.nbr_n = pool.get<int>(n);
    t.cell_start = pool.get<int>(nc);
    t.cell_count = pool.get<int>(nc);
    t.cell_atoms = pool.get<int>(n);
    t.cell_of = pool.get<int>(n);
    t.cell_slot = pool.get<int>(n);
    return pool.ok ? SLD_OK : SLD_ERR_NOMEM;
}

template <class T>
void dcopy(T* dst, const T* src, size_t n, cudaStream_t st) {
    cudaMemcpyAsync(dst, src, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
}

// the engine state a step reads or the links and list passes rewrite
void save(const Adj& a, Snap& s) {
    const Dev& D = a.c->D;
    cudaStream_t st = a.c->st;
    size_t n = a.n, nc = a.nc;
    dcopy(s.r, D.r, n, st); dcopy(s.p, D.p, n, st); dcopy(s.s, D.s, n, st); dcopy(s.f, D.f, n, st);
    dcopy(s.stamp, D.stamp, n, st); dcopy(s.cell_of, D.cell_of, n, st);
    dcopy(s.cell_start, D.cell_start, nc, st); dcopy(s.cell_count, D.cell_count, nc, st);
    dcopy(s.cell_atoms, D.cell_atoms, n, st); dcopy(s.cell_slot, D.cell_slot, n, st);
    dcopy(s.fxs, D.fxs, n, st);
    if (s.fxa) dcopy(s.fxa, D.fxa, n, st);
    if (s.nbk) dcopy(s.nbk, D.nbk, a.nnb, st);
    dcopy(s.nbr, D.nbr, a.nnb, st); dcopy(s.nbr_n, D.nbr_n, n, st);
    dcopy(s.ctl, D.ctl, 1, st);
}

void restore(const Adj& a, const Snap& s) {
    const Dev& D = a.c->D;
    cudaStream_t st = a.c->st;
    size_t n = a.n, nc = a.nc;
    dcopy(D.r, s.r, n, st); dcopy(D.p, s.p, n, st); dcopy(D.s, s.s, n, st); dcopy(D.f, s.f, n, st);
    dcopy(D.stamp, s.stamp, n, st); dcopy(D.cell_of, s.cell_of, n, st);
    dcopy(D.cell_start, s.cell_start, nc, st); dcopy(D.cell_count, s.cell_count, nc, st);
    dcopy(D.cell_atoms, s.cell_atoms, n, st); dcopy(D.cell_slot, s.cell_slot, n, st);
    dcopy(D.fxs, s.fxs, n, st);
    if (s.fxa) dcopy(D.fxa, s.fxa, n, st);
    if (s.nbk) dcopy(D.nbk, s.nbk, a.nnb, st);
    dcopy(D.nbr, s.nbr, a.nnb, st); dcopy(D.nbr_n, s.nbr_n, n, st);
    dcopy(D.ctl, s.ctl, 1, st);
}

// one core_ds(dt) of the NVE step: the forward sweep over the colour groups,
// then the backward sweep (core_ds_CPU.cpp:35-83); mid receives the spins
// between the two
void sweeps(const Adj& a, double dt, double4* mid) {
    sld_ctx* c = a.c;
    const auto& G = c->G;
    double h = dt / 2e0;
    for (int g = 0; g < G.ngroups; ++g)
        adj_sweep(c->D, a.K, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g], h, false);
    if (mid) dcopy(mid, c->D.s, a.n, c->st);
    for (int g = G.ngroups - 1; g >= 0; --g)
        adj_sweep(c->D, a.K, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g], h, true);
}

// the rho and force passes of the state in the context, after its lists
void fields(const Adj& a) {
    adj_rho(a.c->D, a.A, a.K, a.c->st);
    adj_force(a.c->D, a.A, a.K, a.c->st, a.el2);
}

// One NVE main-loop step with the parameterised potential (core.cpp:55-63);
// with t, its intermediates are kept.
void step_forward(const Adj& a, Tape* t) {
    sld_ctx* c = a.c;
    const Dev& D = c->D;
    cudaStream_t st = c->st;
    double dt = c->P.step;
    size_t n = a.n, nc = a.nc;
    launch_links(D, st, false, c->scan_blocks);
    if (t) {
        dcopy(t->cell_start, D.cell_start, nc, st); dcopy(t->cell_count, D.cell_count, nc, st);
        dcopy(t->cell_atoms, D.cell_atoms, n, st); dcopy(t->cell_of, D.cell_of, n, st);
        dcopy(t->cell_slot, D.cell_slot, n, st);
        dcopy(t->r0, D.r, n, st); dcopy(t->s0, D.s, n, st);
    }
    adj_kick(D, st, dt / 2e0, t ? t->ppre1 : a.scratch_p);
    sweeps(a, dt / 2e0, t ? t->sA : nullptr);
    if (t) dcopy(t->s1, D.s, n, st);
    launch_dr(D, st, dt);
    launch_pairs(D, st, false);
    adj_rho(D, a.A, a.K, st);
    if (t) {
        dcopy(t->r1, D.r, n, st);
        dcopy(t->nbr, D.nbr, a.nnb, st); dcopy(t->nbr_n, D.nbr_n, n, st);
        dcopy(t->rho1, a.A.rho, n, st); dcopy(t->dF1, a.A.dF, n, st);
    }
    sweeps(a, dt / 2e0, t ? t->sB : nullptr);
    if (t) dcopy(t->s2, D.s, n, st);
    adj_force(D, a.A, a.K, st, a.el2);
    adj_kick(D, st, dt / 2e0, t ? t->ppre2 : a.scratch_p);
}

// the engine state with the positions, spins and lists of a tape
Dev tape_dev(const Adj& a, const Tape& t, bool second_half, const int* nbr_in, const int* nbr_n_in) {
    Dev D = a.c->D;
    D.cell_start = t.cell_start; D.cell_count = t.cell_count; D.cell_atoms = t.cell_atoms;
    D.cell_of = t.cell_of; D.cell_slot = t.cell_slot;
    if (second_half) {
        D.r = t.r1; D.s = t.s2; D.nbr = t.nbr; D.nbr_n = t.nbr_n;
    } else {
        D.r = t.r0; D.s = t.s0; D.nbr = const_cast<int*>(nbr_in); D.nbr_n = const_cast<int*>(nbr_n_in);
    }
    return D;
}

void sweeps_rev(const Adj& a, const Dev& D, double dt, const double4* s0, const double4* mid,
                const double4* s1) {
    sld_ctx* c = a.c;
    const auto& G = c->G;
    double h = dt / 2e0;
    // the backward sweep first (its groups in the forward order), then the forward sweep
    for (int g = 0; g < G.ngroups; ++g)
        adj_sweep_rev(D, a.A, a.K, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g], h,
                      true, g, mid, s1);
    for (int g = G.ngroups - 1; g >= 0; --g)
        adj_sweep_rev(D, a.A, a.K, c->st, c->d_gcells + G.gstart[g], G.gstart[g + 1] - G.gstart[g], h,
                      false, g, s0, mid);
    int rows = 0;
    for (int g = 0; g < G.ngroups; ++g) rows = std::max(rows, (G.gstart[g + 1] - G.gstart[g] + 3) / 4);
    adj_theta_flush(a.A, c->st, rows);
}

// One step reversed.  In: the adjoints of the step's end state (rb, pb, sb)
// and of its force pass (fb, from the next step's first kick or the loss).
// Out: the adjoints of its start state, and fb of the previous force pass.
void step_reverse(const Adj& a, const Tape& t, const int* nbr_in, const int* nbr_n_in) {
    sld_ctx* c = a.c;
    cudaStream_t st = c->st;
    double dt = c->P.step;
    adj_kick_rev(c->D, a.A, st, dt / 2e0, t.ppre2);
    Dev D2 = tape_dev(a, t, true, nullptr, nullptr);
    AdjDev A2 = a.A;
    A2.rho = t.rho1;
    A2.dF = t.dF1;
    adj_force_rev(D2, A2, a.K, st);
    cudaMemsetAsync(a.A.fb, 0, sizeof(double4) * a.n, st);
    sweeps_rev(a, D2, dt / 2e0, t.s1, t.sB, t.s2);
    adj_rho_rev(D2, A2, a.K, st);
    adj_drift_rev(c->D, a.A, st, dt);
    Dev D1 = tape_dev(a, t, false, nbr_in, nbr_n_in);
    sweeps_rev(a, D1, dt / 2e0, t.s0, t.sA, t.s1);
    adj_kick_rev(c->D, a.A, st, dt / 2e0, t.ppre1);
}

int check_ctx(sld_ctx* c) {
    if (!c) return SLD_ERR_ARG;
    const sld_params& P = c->P;
    // the NVE spin-lattice step of the reference: no thermostats, no electrons
    if (P.spinlang || P.lattlang || P.eltemp || P.change_step || P.pressure_control ||
        P.stress_control || P.hamiltonian != SLD_HAM_SLDHL || c->D.hext || c->D.fext)
        return SLD_ERR_ARG;
    return SLD_OK;
}

int finish(sld_ctx* c) {
    cudaError_t e = cudaStreamSynchronize(c->st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "sld adjoint: %s\n", cudaGetErrorString(e));
        return SLD_ERR_CUDA;
    }
    unsigned err = 0;
    ACK(cudaMemcpy(&err, &c->D.ctl->err, sizeof err, cudaMemcpyDeviceToHost));
    if (err & SLD_FLAG_CAPACITY) return SLD_ERR_CAPACITY;
    if (err & SLD_FLAG_NAN) return SLD_ERR_NAN;
    return SLD_OK;
}

}  // namespace

extern "C" {

int sld_adjoint_theta_default(double* theta) {
    if (!theta) return SLD_ERR_ARG;
    sld::pot_theta(theta);
    return SLD_OK;
}

int sld_adjoint_config(sld_ctx* c, const double* theta, double* out4, double* dE, double* dL) {
    int rc = check_ctx(c);
    if (rc) return rc;
    SLD_DEVICE_OF(c);
    if (!theta || !out4) return SLD_ERR_ARG;
    Adj a;
    rc = alloc_adj(a, c, theta);
    if (rc) return rc;
    cudaStream_t st = c->st;
    double4* f_keep = a.pool.get<double4>(a.n);
    if (!a.pool.ok) return SLD_ERR_NOMEM;
    ACK(cudaDeviceSynchronize());   // the pool's clearing memsets
    dcopy(f_keep, c->D.f, a.n, st);
    launch_pairs(c->D, st, false);
    fields(a);
    double el[2];
    ACK(cudaMemcpyAsync(el, a.el2, sizeof el, cudaMemcpyDeviceToHost, st));
    // the field's share of the loss: sum |H|^2
    std::vector<double4> H(a.n), f(a.n);
    ACK(cudaMemcpyAsync(H.data(), a.A.H, sizeof(double4) * a.n, cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(f.data(), c->D.f, sizeof(double4) * a.n, cudaMemcpyDeviceToHost, st));
    if (dE) {
        adj_energy_grad(c->D, a.A, a.K, st);
        ACK(cudaMemcpyAsync(dE, a.A.theta_bar, sizeof(double) * ADJ_NTHETA, cudaMemcpyDeviceToHost, st));
    }
    if (dL) {
        cudaMemsetAsync(a.A.theta_bar, 0, sizeof(double) * ADJ_NTHETA, st);
        adj_seed_loss(c->D, a.A, st);
        adj_force_rev(c->D, a.A, a.K, st);
        adj_field_rev(c->D, a.A, a.K, st);
        adj_rho_rev(c->D, a.A, a.K, st);
        ACK(cudaMemcpyAsync(dL, a.A.theta_bar, sizeof(double) * ADJ_NTHETA, cudaMemcpyDeviceToHost, st));
    }
    dcopy(c->D.f, f_keep, a.n, st);
    rc = finish(c);
    if (rc) return rc;
    double fs = 0, hs = 0;
    for (size_t i = 0; i < a.n; ++i) {
        fs += f[i].x * f[i].x + f[i].y * f[i].y + f[i].z * f[i].z;
        hs += H[i].x * H[i].x + H[i].y * H[i].y + H[i].z * H[i].z;
    }
    out4[0] = el[0];
    out4[1] = el[1];
    out4[2] = fs;
    out4[3] = hs;
    return SLD_OK;
}

int sld_adjoint_jacobians(sld_ctx* c, const double* theta, double* f, double* H, double* dF,
                          double* dH) {
    int rc = check_ctx(c);
    if (rc) return rc;
    SLD_DEVICE_OF(c);
    if (!theta || !dF) return SLD_ERR_ARG;
    Adj a;
    rc = alloc_adj(a, c, theta);
    if (rc) return rc;
    cudaStream_t st = c->st;
    const size_t n = a.n, w = 3 * ADJ_NTHETA;
    double4* f_keep = a.pool.get<double4>(n);
    double* drho = a.pool.get<double>(12 * n);
    double* ddf = a.pool.get<double>(w * n);
    double* ddh = a.pool.get<double>(w * n);
    if (!a.pool.ok) return SLD_ERR_NOMEM;
    ACK(cudaDeviceSynchronize());   // the pool's clearing memsets
    dcopy(f_keep, c->D.f, n, st);
    launch_pairs(c->D, st, false);
    fields(a);
    adj_jacobians(c->D, a.A, a.K, st, drho, ddf, ddh);
    std::vector<double> hf(w * n), hh(w * n);
    std::vector<double4> fv(n), Hv(n);
    ACK(cudaMemcpyAsync(hf.data(), ddf, sizeof(double) * w * n, cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(hh.data(), ddh, sizeof(double) * w * n, cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(fv.data(), c->D.f, sizeof(double4) * n, cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(Hv.data(), a.A.H, sizeof(double4) * n, cudaMemcpyDeviceToHost, st));
    dcopy(c->D.f, f_keep, n, st);
    rc = finish(c);
    if (rc) return rc;
    // slot order to the caller's atom order
    for (size_t q = 0; q < n; ++q) {
        size_t i = (size_t)c->id_of_slot[q];
        std::copy(hf.begin() + q * w, hf.begin() + (q + 1) * w, dF + i * w);
        if (dH) std::copy(hh.begin() + q * w, hh.begin() + (q + 1) * w, dH + i * w);
        if (f) { f[3 * i] = fv[q].x; f[3 * i + 1] = fv[q].y; f[3 * i + 2] = fv[q].z; }
        if (H) { H[3 * i] = Hv[q].x; H[3 * i + 1] = Hv[q].y; H[3 * i + 2] = Hv[q].z; }
    }
    return SLD_OK;
}

int sld_adjoint_trajectory(sld_ctx* c, const double* theta, int nsteps, int checkpoint_every,
                           double* L, double* dL) {
    int rc = check_ctx(c);
    if (rc) return rc;
    SLD_DEVICE_OF(c);
    if (!theta || !L || nsteps < 0 || checkpoint_every < 1) return SLD_ERR_ARG;
    Adj a;
    rc = alloc_adj(a, c, theta);
    if (rc) return rc;
    cudaStream_t st = c->st;
    const int C = checkpoint_every;
    const int nseg = (nsteps + C - 1) / C;
    Snap orig{};
    rc = alloc_snap(a.pool, a, orig);
    std::vector<Snap> ck(dL ? nseg : 0);
    for (auto& s : ck)
        if (!rc) rc = alloc_snap(a.pool, a, s);
    std::vector<Tape> tape(dL ? std::min(C, std::max(nsteps, 1)) : 0);
    for (auto& t : tape)
        if (!rc) rc = alloc_tape(a.pool, a, t);
    if (rc) return rc;
    ACK(cudaDeviceSynchronize());   // the pool's clearing memsets
    save(a, orig);

    // forward: the start state's lists and forces, then the steps
    launch_pairs(c->D, st, false);
    fields(a);
    for (int k = 0; k < nsteps; ++k) {
        if (dL && k % C == 0) save(a, ck[k / C]);
        step_forward(a, nullptr);
    }
    double el[2];
    ACK(cudaMemcpyAsync(el, a.el2, sizeof el, cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    *L = el[1];

    if (dL) {
        // seeds: the loss of the end state
        adj_seed_loss(c->D, a.A, st);
        adj_field_rev(c->D, a.A, a.K, st);
        for (int g = nseg - 1; g >= 0; --g) {
            int k0 = g * C, k1 = std::min(nsteps, k0 + C);
            restore(a, ck[g]);
            // the lists the segment's first sweeps read
            const int* nbr_in = ck[g].nbr;
            const int* nbr_n_in = ck[g].nbr_n;
            // forces of the checkpoint's state were restored with it; the
            // densities of the segment's first step are taped by the step
            for (int k = k0; k < k1; ++k) step_forward(a, &tape[k - k0]);
            for (int k = k1 - 1; k >= k0; --k) {
                const Tape& t = tape[k - k0];
                const int* ni = k == k0 ? nbr_in : tape[k - k0 - 1].nbr;
                const int* nni = k == k0 ? nbr_n_in : tape[k - k0 - 1].nbr_n;
                step_reverse(a, t, ni, nni);
            }
        }
        // the start state's force pass (read by the first kick) and its densities
        restore(a, orig);
        launch_pairs(c->D, st, false);
        adj_rho(c->D, a.A, a.K, st);
        adj_force_rev(c->D, a.A, a.K, st);
        adj_rho_rev(c->D, a.A, a.K, st);
        ACK(cudaMemcpyAsync(dL, a.A.theta_bar, sizeof(double) * ADJ_NTHETA, cudaMemcpyDeviceToHost, st));
    }
    restore(a, orig);
    launch_pairs(c->D, st, false);
    return finish(c);
}

}  // extern "C"
