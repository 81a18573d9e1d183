// core_dTe (core_dTe_CPU.cpp:47-200): nloop substeps of
// A(h/2) B(h/2) C(h) B(h/2) A(h/2) on the electron-temperature cells.
//   A  C dTe/dt = Gel Tl + Ges Ts_L     (cell-local)
//   B  C dTe/dt = -(Gel + Ges) Te       (cell-local, RK4)
//   C  C dTe/dt = kappa Laplacian Te    (colour sweep forward and back over
//      the cells, then the total Ee rescaled to its value before the sweep)
// Three kernels, by mesh size:
//   k_dte_hub      meshes up to kHubMaxCells: an 8-CTA cluster, the sweep on
//                  one CTA's shared memory, with the colour lists and a
//                  neighbour table there too (the default);
//   k_dte_cluster  any mesh: the cells spread over a cluster, Te in global
//                  memory, a cluster barrier per colour phase;
//   k_dte          any mesh, one CTA, global memory (no clusters).
// Each is compiled with the reference's heat-capacity expressions (FP64
// form) and with the fitted ones (sld_te.cuh; split form and its FP64 twin).
#include <cooperative_groups.h>

#include <cstdlib>

#include "sld_te.cuh"

namespace cg = cooperative_groups;

struct DteGeom {
    double dx2, dy2, dz2, pre;   // squared Te-cell edges; C's prefactor for a step h
    double idx2, idy2, idz2;     // their reciprocals (fitted form)
};

__device__ __forceinline__ DteGeom dte_geom(const Dev& D, double h) {
    DteGeom g;
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    g.dx2 = lx * lx;
    g.dy2 = ly * ly;
    g.dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    g.pre = h / 2.0 * cond * volume_factor / SLD_BOLTZ;
    g.idx2 = 1.0 / g.dx2;
    g.idy2 = 1.0 / g.dy2;
    g.idz2 = 1.0 / g.dz2;
    return g;
}

// the six face neighbours of Te cell k (periodic)
struct Nbr6 {
    int xp, xm, yp, ym, zp, zm;
};
__device__ __forceinline__ Nbr6 te_nbr6(const Dev& D, int k) {
    const int tx = D.tx, ty = D.ty, tz = D.tz;
    int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
    int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
    int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
    int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
    return {xp + (y + z * ty) * tx, xm + (y + z * ty) * tx, x + (yp + z * ty) * tx,
            x + (ym + z * ty) * tx, x + (y + zp * ty) * tx, x + (y + zm * ty) * tx};
}

// core_dTe_CPU.cpp:158-171: the Laplacian term of one cell (the fitted
// form multiplies by the reciprocal squared edges instead of dividing, with
// every rounding written out, so that the hub's two sweep schedules, whose
// code the compiler contracts differently, form the same bits)
template <bool FAST>
__device__ __forceinline__ double te_lap(const DteGeom& g, double T, double xp, double xm,
                                         double yp, double ym, double zp, double zm) {
    if constexpr (FAST) {
        const double t2 = 2.0 * T;
        const double ex = __dsub_rn(__dadd_rn(xp, xm), t2);
        const double ey = __dsub_rn(__dadd_rn(yp, ym), t2);
        const double ez = __dsub_rn(__dadd_rn(zp, zm), t2);
        return __dmul_rn(g.pre, __fma_rn(ez, g.idz2, __fma_rn(ey, g.idy2, __dmul_rn(ex, g.idx2))));
    } else {
        double ex = xp + xm - 2.0 * T;
        double ey = yp + ym - 2.0 * T;
        double ez = zp + zm - 2.0 * T;
        return g.pre * (ex / g.dx2 + ey / g.dy2 + ez / g.dz2);
    }
}

// Gel Tl + Ges Ts_L and (Gel + Ges) hh / boltz of cell k
// (core_dTe_CPU.cpp:66-122: the lattice's and the spins' coupling, by what
// the Hamiltonian has; Ts_R for the Heisenberg Hamiltonians)
__device__ __forceinline__ double te_src(const Dev& D, int k) {
    double dE = 0.0;
    if (D.latt) dE += D.Gel[k] * D.Tl[k];
    if (D.spin) dE += D.Ges[k] * (D.landau_on ? D.TsL[k] : D.TsR[k]);
    return dE;
}
__device__ __forceinline__ double te_rate(const Dev& D, int k, double hh) {
    double g = 0.0;
    if (D.latt) g += D.Gel[k];
    if (D.spin) g += D.Ges[k];
    g *= hh / SLD_BOLTZ;
    return g;
}

// ---------------------------------------------------------------------
// one CTA, global memory

template <bool FAST>
__device__ __forceinline__ void dte_A(const Dev& D, double dt) {
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = te_E<FAST>(D.Te[k]);
        Ee += dt * te_src(D, k);
        D.Ee[k] = Ee;
        D.Te[k] = te_T<FAST>(Ee);
    }
}

template <bool FAST>
__device__ __forceinline__ void dte_B(const Dev& D, double dt) {
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x)
        D.Te[k] = te_rk4<FAST>(D.Te[k], te_rate(D, k, dt), dt);
}

template <bool FAST>
__device__ __forceinline__ double dte_total_Ee(const Dev& D, double* sh) {
    double acc = 0.0;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double e = te_E<FAST>(D.Te[k]);
        D.Ee[k] = e;
        acc += e;
    }
    double t = block_sum(acc, sh);
    __shared__ double tot;
    if (threadIdx.x == 0) tot = t;
    __syncthreads();
    return tot;
}

template <bool FAST>
__device__ __forceinline__ void dte_C(const Dev& D, double dt, double* sh) {
    double start = dte_total_Ee<FAST>(D, sh);
    const DteGeom gm = dte_geom(D, dt);
    for (int pass = 0; pass < 2; ++pass) {
        for (int gg = 0; gg < D.te_ngroups; ++gg) {
            int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
            int b = D.te_gstart[g], e = D.te_gstart[g + 1];
            for (int m = b + threadIdx.x; m < e; m += blockDim.x) {
                int k = D.te_gcells[m];
                const Nbr6 q = te_nbr6(D, k);
                const double* Te = D.Te;
                double T = Te[k];
                double Ee = te_E<FAST>(T);
                Ee += te_lap<FAST>(gm, T, Te[q.xp], Te[q.xm], Te[q.yp], Te[q.ym], Te[q.zp], Te[q.zm]);
                D.Ee[k] = Ee;
                D.Te[k] = te_T<FAST>(Ee);
            }
            __syncthreads();
        }
    }
    double end = dte_total_Ee<FAST>(D, sh);
    double fac = start / end;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = D.Ee[k] * fac;
        D.Ee[k] = Ee;
        D.Te[k] = te_T<FAST>(Ee);
    }
    __syncthreads();
}

template <bool FAST>
__global__ void __launch_bounds__(1024) k_dte(Dev D, double dt) {
    __shared__ double sh[32];
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop;
    for (int it = 0; it < nloop; ++it) {
        dte_A<FAST>(D, h / 2.0);
        __syncthreads();
        dte_B<FAST>(D, h / 2.0);
        __syncthreads();
        dte_C<FAST>(D, h, sh);
        dte_B<FAST>(D, h / 2.0);
        __syncthreads();
        dte_A<FAST>(D, h / 2.0);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------
// core_dTe on a thread-block cluster: the Te cells are split over the
// cluster's CTAs (each thread owns the same cells in every phase, so A and B
// need no barrier); the colour phases of the diffusion sweep and the two
// energy sums of C synchronise the cluster with its hardware barrier.  Te is
// read across CTAs through L2 (ld.global.cg) after the barrier.

__device__ __forceinline__ double cl_total(double v, double* sh, double* slot_base,
                                           cg::cluster_group& cl) {
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) __stcg(slot_base + cl.block_rank(), t);
    cl.sync();
    double tot = 0.0;
    for (unsigned r = 0; r < cl.num_blocks(); ++r) tot += __ldcg(slot_base + r);
    return tot;
}

template <bool FAST>
__global__ void __launch_bounds__(256) k_dte_cluster(Dev D, double dt) {
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double sh[32];
    const int nb = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int per = (D.nte + nb - 1) / nb;
    const int k0 = rank * per, k1 = min(D.nte, k0 + per);
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    const double h = dt / nloop, hh = h / 2.0;
    const DteGeom gm = dte_geom(D, h);
    double* slots = D.red;   // 2 x num_blocks partial sums
    for (int it = 0; it < nloop; ++it) {
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {   // A(h/2), B(h/2)
            double Ee = te_E<FAST>(__ldcg(D.Te + k));
            Ee += hh * te_src(D, k);
            double T = te_T<FAST>(Ee);
            __stcg(D.Te + k, te_rk4<FAST>(T, te_rate(D, k, hh), hh));
        }
        // C(h): start sum, colour sweep forward and back, end sum, rescale
        double part = 0.0;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) part += te_E<FAST>(__ldcg(D.Te + k));
        double start = cl_total(part, sh, slots, cl);
        for (int pass = 0; pass < 2; ++pass) {
            for (int gg = 0; gg < D.te_ngroups; ++gg) {
                int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
                for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
                    if (D.te_color[k] != g) continue;
                    const Nbr6 q = te_nbr6(D, k);
                    double T = __ldcg(D.Te + k);
                    double Ee = te_E<FAST>(T);
                    Ee += te_lap<FAST>(gm, T, __ldcg(D.Te + q.xp), __ldcg(D.Te + q.xm),
                                 __ldcg(D.Te + q.yp), __ldcg(D.Te + q.ym), __ldcg(D.Te + q.zp),
                                 __ldcg(D.Te + q.zm));
                    __stcg(D.Te + k, te_T<FAST>(Ee));
                }
                cl.sync();
            }
        }
        part = 0.0;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) part += te_E<FAST>(__ldcg(D.Te + k));
        double end = cl_total(part, sh, slots + nb, cl);
        double fac = start / end;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {   // rescale, B(h/2), A(h/2)
            double T = te_T<FAST>(te_E<FAST>(__ldcg(D.Te + k)) * fac);
            T = te_rk4<FAST>(T, te_rate(D, k, hh), hh);
            double Ee = te_E<FAST>(T) + hh * te_src(D, k);
            D.Ee[k] = Ee;
            __stcg(D.Te + k, te_T<FAST>(Ee));
        }
        cl.sync();   // the next substep reads neighbours' Te and reuses the slots
    }
}

// ---------------------------------------------------------------------
#define HUB_CL 8
// Cluster "hub" form: every CTA of an 8-CTA cluster does the cell-local A and
// B parts for its share of the cells in parallel; CTA 0 holds all Te and
// Te_to_Ee(Te) in its shared memory (the others read and write them through
// distributed shared memory) and runs C's diffusion sweep with block
// barriers.  Two cluster barriers per substep instead of one per colour
// phase.
//   - The cells are stored in colour order (position m holds te_gcells[m]),
//     so the cells of a colour group are consecutive and so, in a regular
//     mesh, are their neighbours in each direction: a warp's shared-memory
//     loads of the sweep hit distinct banks.  A table gives each position
//     the positions of its six face neighbours, one 16-byte record.
//   - Each CTA keeps its cells' coupling source Gel Tl + Ges Ts_L and rate
//     (Gel + Ges) h/2/boltz in its own shared memory: they do not change
//     during core_dTe, so the substeps read no global memory.
//   - The sweep runs by colour phases (one barrier per phase) or by levels
//     (te_levels: one barrier per level, fewer than the phases).
//   - Reference expressions: half of the hub's threads update the Te of a
//     phase's (level's) cells, the chain the next one waits for, while the
//     other half evaluate Te_to_Ee for the cells of the previous one, which
//     nothing of this one reads.  A cell updated in two consecutive phases
//     (the last forward colour) has its Te_to_Ee evaluated in place; by
//     levels, such a pair of updates is one task.  Every value is the one of
//     the plain sequence.
//   - Fitted expressions: an update keeps the energy it converts to Te (what
//     Te_to_Ee would return, up to rounding), so the sweep evaluates no
//     Te_to_Ee at all.
static const int kHubMaxCells = 6000;   // 8 (2 n + 10 + 2 n / 8) + 16 n + 4 n bytes of shared memory

// the positions of the six face neighbours of position m
__device__ __forceinline__ void hub_nb(const uint4* sNb, int m, int (&q)[6]) {
    const uint4 v = sNb[m];
    q[0] = (int)(v.x & 0xffffu);
    q[1] = (int)(v.x >> 16);
    q[2] = (int)(v.y & 0xffffu);
    q[3] = (int)(v.y >> 16);
    q[4] = (int)(v.z & 0xffffu);
    q[5] = (int)(v.z >> 16);
}

// one update of the fitted form (two for a double task) at position t & 0x7fff:
// its new Te and energy, which it returns; nothing is stored
__device__ __forceinline__ int hub_task_fast(const double* hsm, int n, const uint4* sNb, unsigned t,
                                             const DteGeom& gm, double& T, double& x) {
    const int m = (int)(t & 0x7fffu);
    int q[6];
    hub_nb(sNb, m, q);
    const double a0 = hsm[q[0]], a1 = hsm[q[1]], a2 = hsm[q[2]], a3 = hsm[q[3]], a4 = hsm[q[4]],
                 a5 = hsm[q[5]];
    T = hsm[m];
    x = __dadd_rn(hsm[n + m], te_lap<true>(gm, T, a0, a1, a2, a3, a4, a5));
    T = te_T<true>(x);
    if (t & 0x8000u) {
        x = __dadd_rn(x, te_lap<true>(gm, T, a0, a1, a2, a3, a4, a5));
        T = te_T<true>(x);
    }
    return m;
}

// one update (two for a double task) of the reference form: the new Te
__device__ __forceinline__ int hub_task_ref(const double* hsm, int n, const uint4* sNb, unsigned t,
                                            const DteGeom& gm, double& T) {
    const int m = (int)(t & 0x7fffu);
    int q[6];
    hub_nb(sNb, m, q);
    const double a0 = hsm[q[0]], a1 = hsm[q[1]], a2 = hsm[q[2]], a3 = hsm[q[3]], a4 = hsm[q[4]],
                 a5 = hsm[q[5]];
    T = hsm[m];
    T = te_T<false>(hsm[n + m] + te_lap<false>(gm, T, a0, a1, a2, a3, a4, a5));
    if (t & 0x8000u) {
        const double E = te_E<false>(T);
        T = te_T<false>(E + te_lap<false>(gm, T, a0, a1, a2, a3, a4, a5));
    }
    return m;
}

// C's diffusion sweep on the hub.  By levels (LEV) the tasks of a level read
// no value another task of the level writes; by phases a phase is one colour
// group, positions te_gstart[g]..te_gstart[g+1].  The fitted form takes two
// tasks per thread and iteration, whose chains interleave.  The reference
// form splits the threads into workers and helpers (above).
template <bool FAST, bool LEV>
__device__ __forceinline__ void hub_sweep(const Dev& D, double* hsm, int n,
                                          const unsigned short* sTk, const uint4* sNb,
                                          const DteGeom& gm) {
    const int G = D.te_ngroups;
    const int nph = LEV ? D.te_nlevels : 2 * G;
    // tasks of phase (level) l: [b, e), as positions (phases) or task entries
    auto range = [&](int l, int& b, int& e) {
        if constexpr (LEV) {
            b = D.te_lstart[l];
            e = D.te_lstart[l + 1];
        } else {
            const int g = l < G ? l : 2 * G - 1 - l;
            b = D.te_gstart[g];
            e = D.te_gstart[g + 1];
        }
    };
    auto task = [&](int m) -> unsigned { return LEV ? (unsigned)sTk[m] : (unsigned)m; };
    if constexpr (FAST) {
        const int bd = blockDim.x;
        for (int l = 0; l < nph; ++l) {
            int b, e;
            range(l, b, e);
            for (int m = b + threadIdx.x; m < e; m += 2 * bd) {
                if (m + bd < e) {   // two tasks: both chains in flight together
                    double T1, x1, T2, x2;
                    const int k1 = hub_task_fast(hsm, n, sNb, task(m), gm, T1, x1);
                    const int k2 = hub_task_fast(hsm, n, sNb, task(m + bd), gm, T2, x2);
                    hsm[k1] = T1;
                    hsm[n + k1] = x1;
                    hsm[k2] = T2;
                    hsm[n + k2] = x2;
                } else {
                    double T1, x1;
                    const int k1 = hub_task_fast(hsm, n, sNb, task(m), gm, T1, x1);
                    hsm[k1] = T1;
                    hsm[n + k1] = x1;
                }
            }
            __syncthreads();
        }
    } else {
        const int half = blockDim.x / 2;
        const bool worker = threadIdx.x < half;
        const int lane = worker ? threadIdx.x : threadIdx.x - half;
        int pb = 0, pe = 0;   // the previous phase's tasks, whose Te_to_Ee is due
        for (int l = 0; l < nph; ++l) {
            int b, e;
            range(l, b, e);
            // by phases, the last forward colour is updated again at once
            const bool inplace = !LEV && l == G - 1;
            if (worker) {
                for (int m = b + lane; m < e; m += half) {
                    double T;
                    const int k = hub_task_ref(hsm, n, sNb, task(m), gm, T);
                    hsm[k] = T;
                    if (inplace) hsm[n + k] = te_E<false>(T);
                }
            } else {
                for (int m = pb + lane; m < pe; m += half) {
                    const int k = (int)(task(m) & 0x7fffu);
                    hsm[n + k] = te_E<false>(hsm[k]);
                }
            }
            __syncthreads();
            pb = inplace ? 0 : b;
            pe = inplace ? 0 : e;
        }
        for (int m = pb + threadIdx.x; m < pe; m += blockDim.x) {
            const int k = (int)(task(m) & 0x7fffu);
            hsm[n + k] = te_E<false>(hsm[k]);
        }
    }
}

template <bool FAST, bool LEV>
__global__ void __launch_bounds__(1024) k_dte_hub(Dev D, double dt, int per) {
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) double hsm[];
    const int n = D.nte;
    const int rank = (int)cl.block_rank();
    double* hT = cl.map_shared_rank(hsm, 0);   // the hub's arrays, by position
    double* hE = hT + n;
    double* hpart = hT + 2 * n + 2;            // each CTA's sum of Ee after A and B
    double* hfac = hT + 2 * n;
    // myE: the energy each A step starts from, the value this CTA last gave
    // the position, in this CTA's own shared memory (every CTA's has the hub's
    // layout): the hub's Te-to-Ee array on the hub, the unused slots of the
    // hub's Te array elsewhere
    double* myE = rank == 0 ? hsm + n : hsm;
    double* mySrc = hsm + 2 * n + 2 + HUB_CL;  // this CTA's own positions
    double* myG = mySrc + per;
    uint4* sNb = reinterpret_cast<uint4*>(myG + per);                      // hub: neighbours
    unsigned short* sTk = reinterpret_cast<unsigned short*>(sNb + n);      // hub: level tasks
    __shared__ double sh[32];
    const int p0 = rank * per, p1 = min(n, p0 + per);
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop, hh = h / 2.0;
    for (int m = p0 + threadIdx.x; m < p1; m += blockDim.x) {
        const int k = D.te_gcells[m];
        double T = D.Te[k];
        hT[m] = T;
        myE[m] = te_E<FAST>(T);
        mySrc[m - p0] = te_src(D, k);
        myG[m - p0] = te_rate(D, k, hh);
    }
    if (rank == 0) {
        for (int m = threadIdx.x; m < n; m += blockDim.x) sNb[m] = D.te_lnb[m];
        if constexpr (LEV) {
            for (int m = threadIdx.x; m < D.te_lstart[D.te_nlevels]; m += blockDim.x)
                sTk[m] = D.te_ltasks[m];
        }
    }
    cl.sync();
    const DteGeom gm = dte_geom(D, h);
    double lastE[4];   // this thread's last A-step energies (per <= 4096 -> <= 4 per thread)
    const int ncta = (int)cl.num_blocks();
    for (int it = 0; it < nloop; ++it) {
        double part = 0.0;   // C's starting energy, summed per CTA
        for (int m = p0 + threadIdx.x; m < p1; m += blockDim.x) {   // A(h/2), B(h/2)
            double T = te_T<FAST>(myE[m] + hh * mySrc[m - p0]);
            T = te_rk4<FAST>(T, myG[m - p0], hh);
            hT[m] = T;
            const double E = te_E<FAST>(T);
            hE[m] = E;
            part += E;
        }
        // sh was last read before the previous cluster barrier
        part = block_sum_after_barrier(part, sh);
        if (threadIdx.x == 0) hpart[rank] = part;
        cl.sync();
        if (rank == 0) {   // C(h) on the hub
            // C's starting energy, valid in thread 0: the fitted form keeps it in
            // the slot after the factor's rather than in a register through its
            // sweep, which holds two updates' chains in flight
            double start = 0.0;
            if (threadIdx.x == 0) {
                for (int r = 0; r < ncta; ++r) start += hsm[2 * n + 2 + r];
                if constexpr (FAST) hsm[2 * n + 1] = start;
            }
            hub_sweep<FAST, LEV>(D, hsm, n, sTk, sNb, gm);
            if constexpr (!FAST) __syncthreads();   // the fitted sweep ends on a barrier
            double acc = 0.0;
            for (int m = threadIdx.x; m < n; m += blockDim.x) acc += hsm[n + m];
            const double t = block_sum_after_barrier(acc, sh);
            if (threadIdx.x == 0) hsm[2 * n] = (FAST ? hsm[2 * n + 1] : start) / t;
        }
        cl.sync();
        const double fac = *hfac;
        int q = 0;
        for (int m = p0 + threadIdx.x; m < p1; m += blockDim.x, ++q) {   // rescale, B, A
            double T = te_T<FAST>(hE[m] * fac);
            T = te_rk4<FAST>(T, myG[m - p0], hh);
            double Ee = te_E<FAST>(T) + hh * mySrc[m - p0];
            if (FAST && it + 1 < nloop) {
                // the fitted form keeps the energy: the next substep's A
                // continues from it without the round trip through Te
                myE[m] = Ee;
            } else {
                T = te_T<FAST>(Ee);
                hT[m] = T;
                myE[m] = te_E<FAST>(T);
            }
            if (q < 4) lastE[q] = Ee;
        }
    }
    int q = 0;
    for (int m = p0 + threadIdx.x; m < p1; m += blockDim.x, ++q) {
        const int k = D.te_gcells[m];
        D.Te[k] = hT[m];
        if (q < 4) D.Ee[k] = lastE[q];
    }
    cl.sync();   // keep the hub's shared memory alive until every CTA is done
}

// ---------------------------------------------------------------------
// launch

static bool g_dte_inited = false;
static int g_dte_cluster = 0;   // cluster size of k_dte_cluster, 0: clusters unavailable
static int g_dte_mode = 3;      // 3: hub by levels when the mesh fits, 2: hub by colour
                                // phases; 1: cluster; 0: one CTA
static bool g_hub_ok = false;

// dynamic shared memory of k_dte_hub for n Te cells: the hub's Te, f(Te),
// factor and the CTAs' partial sums, each CTA's own source and rate, the
// hub's neighbour records and level tasks
static size_t hub_smem(int n) {
    const int per = (n + HUB_CL - 1) / HUB_CL;
    return sizeof(double) * (2 * (size_t)n + 2 + HUB_CL + 2 * (size_t)per) + sizeof(uint4) * (size_t)n +
           sizeof(unsigned short) * 2 * (size_t)n;
}

static cudaLaunchConfig_t cluster_cfg(int cs, int threads, size_t smem, cudaStream_t st,
                                      cudaLaunchAttribute* at) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

template <bool FAST>
static void dte_attributes() {
    cudaFuncSetAttribute(k_dte_hub<FAST, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)hub_smem(kHubMaxCells));
    cudaFuncSetAttribute(k_dte_hub<FAST, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)hub_smem(kHubMaxCells));
    cudaFuncSetAttribute(k_dte_cluster<FAST>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

int dte_init(int device) {
    (void)device;
    // the kernel choice is read at every context creation (tests switch it)
    const char* m = getenv("SLD_DTE_MODE");
    g_dte_mode = m && m[0] >= '0' && m[0] <= '3' ? m[0] - '0' : 3;
    if (g_dte_inited) return g_dte_cluster;
    g_dte_inited = true;
    dte_attributes<false>();
    dte_attributes<true>();
    cudaLaunchAttribute at[1];
    {
        cudaLaunchConfig_t cfg = cluster_cfg(HUB_CL, 1024, hub_smem(kHubMaxCells), nullptr, at);
        int nclu = 0, nclu2 = 0;
        int nclu3 = 0, nclu4 = 0;
        g_hub_ok =
            cudaOccupancyMaxActiveClusters(&nclu, k_dte_hub<false, false>, &cfg) == cudaSuccess &&
            nclu > 0 &&
            cudaOccupancyMaxActiveClusters(&nclu2, k_dte_hub<true, false>, &cfg) == cudaSuccess &&
            nclu2 > 0 &&
            cudaOccupancyMaxActiveClusters(&nclu3, k_dte_hub<false, true>, &cfg) == cudaSuccess &&
            nclu3 > 0 &&
            cudaOccupancyMaxActiveClusters(&nclu4, k_dte_hub<true, true>, &cfg) == cudaSuccess &&
            nclu4 > 0;
        cudaGetLastError();
    }
    for (int cs : {16, 8, 4}) {
        cudaLaunchConfig_t cfg = cluster_cfg(cs, 256, 0, nullptr, at);
        int n = 0, n2 = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_dte_cluster<false>, &cfg) == cudaSuccess && n > 0 &&
            cudaOccupancyMaxActiveClusters(&n2, k_dte_cluster<true>, &cfg) == cudaSuccess && n2 > 0) {
            g_dte_cluster = cs;
            break;
        }
        cudaGetLastError();
    }
    return g_dte_cluster;
}

template <bool FAST>
static void launch_dte_form(const Dev& D, cudaStream_t st, double dt) {
    cudaLaunchAttribute at[1];
    const int hub_per = (D.nte + HUB_CL - 1) / HUB_CL;
    const int mode = D.tune.dte_mode >= 0 ? D.tune.dte_mode : g_dte_mode;
    // a hub thread keeps the energies of at most four of its CTA's cells
    int threads = D.tune.dte_threads > 0 ? D.tune.dte_threads : 1024;
    if (hub_per > 4 * threads) threads = 1024;
    if (mode >= 2 && g_hub_ok && D.nte <= kHubMaxCells && D.te_nlevels > 0 &&
        hub_per <= 4 * 1024) {
        cudaLaunchConfig_t cfg = cluster_cfg(HUB_CL, threads, hub_smem(D.nte), st, at);
        if (mode == 3)
            cudaLaunchKernelEx(&cfg, k_dte_hub<FAST, true>, D, dt, hub_per);
        else
            cudaLaunchKernelEx(&cfg, k_dte_hub<FAST, false>, D, dt, hub_per);
        return;
    }
    if (mode >= 1 && g_dte_cluster > 0) {
        cudaLaunchConfig_t cfg = cluster_cfg(g_dte_cluster, 256, 0, st, at);
        cudaLaunchKernelEx(&cfg, k_dte_cluster<FAST>, D, dt);
        return;
    }
    k_dte<FAST><<<1, 1024, 0, st>>>(D, dt);
}

void launch_dte(const Dev& D, cudaStream_t st, double dt) {
    if (D.split || D.analytic) launch_dte_form<true>(D, st, dt);
    else launch_dte_form<false>(D, st, dt);
}
