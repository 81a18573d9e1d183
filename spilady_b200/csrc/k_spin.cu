// Suzuki-Trotter spin sweeps (core_ds_CPU.cpp:35-83), one launch per colour
// group and direction.
//
// The reference visits the cells of colour group 0..G-1 (then G-1..0), each
// cell's atoms in list order head -> tail (then tail -> head), and each visit
// (calculate_spin_CPU.cpp:33-199) evaluates Heff_H = sum_j J(r_ij) s_j with
// the spins as they are at that moment.  Cells of one colour share no
// neighbour, so during a group's launch every spin outside the group's cells
// is frozen and only a cell's own atoms change while it is walked: a thread
// walks one cell.  The walks (below) differ in how a visit's neighbour spins
// reach the thread.
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "sld_pot32.cuh"
#include "sld_spin.cuh"

// the sweep kernels' `backward` argument: bit 0 the backward sweep (tail ->
// head, the second visit record); bit 1 no H, HL, sum J stores (the step
// graph overwrites them later in the same step)
#define SW_BACKWARD 1
#define SW_NO_FIELDS 2

__device__ __forceinline__ void visit_store(const Dev& D, int i, double3 s, double3 H, double3 HL,
                                            double sumJ, bool fields) {
    double s0 = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
    if (!isfinite(s0)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
    D.s[i] = make_double4(s.x, s.y, s.z, s0);
    if (D.split) D.s32[i] = make_float4((float)s.x, (float)s.y, (float)s.z, (float)s0);
    if (fields) {
        D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
        D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
        if (D.spinlang) D.sumJ[i] = sumJ;
    }
}

// The visit records of both sweeps of one core_ds call, made for every atom
// in one parallel pass before the sweeps: rho (which the sweeps do not
// change) and the noise increment dS = sqrt(2 T gamma_S_HL / dt) xi (the
// draw is counter-based, so it does not depend on when it is made, and the
// temperature does not change during core_ds).  A visit then reads one
// 32-byte record; the sweeps' serial chains only read them.
__global__ void __launch_bounds__(256) k_spin_noise(Dev D, int epoch_off, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned long long e0 = D.ctl->epoch + (unsigned long long)epoch_off;
    double T = D.eltemp ? D.Te[D.node[i]] : D.temperature;
    const double rho = D.rho[i];
    for (int v = 0; v < 2; ++v) {
        const unsigned id = (unsigned)D.id[i];
        const double3 xi = D.split ? normals3_f32(D.seed, D.replica, id, e0 + v)
                                   : normals3(D.seed, D.replica, id, e0 + v);
        double3 x = spin_noise_dS(D, T, xi, dt);
        D.vrec[2 * (size_t)i + v] = make_double4(rho, x.x, x.y, x.z);
    }
}

void launch_spin_noise(const Dev& D, cudaStream_t st, int epoch_off, double dt) {
    k_spin_noise<<<div_up(D.natom, 256), 256, 0, st>>>(D, epoch_off, dt);
}

__device__ __forceinline__ double4 visit_record(const Dev& D, int i, int sweep) {
    return D.vrec[2 * (size_t)i + sweep];
}

// one visit entirely from global memory (the fallback path)
__device__ void visit_global(const Dev& D, int i, double dt, int sweep, bool fields) {
    double3 H;
    double sumJ;
    exchange_field(D, i, H, sumJ, [](int) { return false; }, [](int, double) {});
    double4 s4 = D.s[i];
    double rho = 0.0;
    double3 dS = make_double3(0.0, 0.0, 0.0);
    if (D.spinlang) {
        const double4 q = visit_record(D, i, sweep);
        rho = q.x;
        dS = make_double3(q.y, q.z, q.w);
    }
    double3 HL;
    double3 s = spin_integrate_dS(D, make_double3(s4.x, s4.y, s4.z), H, sumJ, rho, dS, dt, HL);
    visit_store(D, i, s, H, HL, sumJ, fields);
}

// the spin as a prefetched neighbour slot holds it (FP32 copy in the split form)
template <bool SPLIT>
__device__ __forceinline__ typename std::conditional<SPLIT, float4, double4>::type spin_reg(
    const double4& s) {
    if constexpr (SPLIT) {
        return make_float4((float)s.x, (float)s.y, (float)s.z, (float)s.w);
    } else {
        return s;
    }
}

// one thread per cell for the whole visit, reading the spins from global
// memory (no shared-memory phases)
__global__ void __launch_bounds__(128) k_sweep_cell(Dev D, const int* __restrict__ gcells,
                                                    int ncell_g, double dt, int backward) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell_g) return;
    int c = gcells[t];
    int st = D.cell_start[c], n = cell_n(D, c);
    const bool bwd = (backward & SW_BACKWARD) != 0;
    const bool fields = bwd && !(backward & SW_NO_FIELDS);
    for (int m = 0; m < n; ++m) {
        int i = D.cell_atoms[st + (bwd ? n - 1 - m : m)];
        visit_global(D, i, dt, bwd ? 1 : 0, fields);
    }
}

// ---------------------------------------------------------------------
// One thread per cell, software-pipelined.  A visit's inputs sit behind a
// chain of dependent loads (cell list -> atom -> exchange row -> neighbour
// spins), and a thread walks its cell's atoms one after another, so without
// overlap every visit pays that chain in full.  Here the loads of later
// visits are issued before visit m is integrated:
//   - the atom index three visits ahead;
//   - the first SC_PJ exchange-list indices of the atom two visits ahead
//     (split form; the FP64 form, short of registers, loads them one visit
//     ahead and waits for them);
//   - for the next atom: its couplings J, the spins of its first SC_PJ
//     exchange neighbours, its own spin, rho and noise increment.
// During visit m only atom m's spin changes (cells of one colour group share
// no neighbour), so a prefetched neighbour spin is stale only if that
// neighbour is atom m; it is replaced by atom m's new spin right after the
// store.  Entries beyond SC_PJ (rare in bcc Fe) are read when used.  The
// field is summed in exchange-list order with exchange_field's arithmetic,
// so the result is the one of k_sweep_cell.  The split form gathers the FP32
// copy of the spins (16 bytes per neighbour, the values its FP32 sums use).
// Exchange entries prefetched per visit.  In bcc Fe the exchange cutoff
// (3.75 A) takes the 14 atoms of the first two shells (the third is at
// 4.05 A); rare longer rows read their extra entries when used.  The row
// indices are loaded 16 at a time (four 16-byte loads).
#define SC_PJ 14
#define SC_ROW 16

// the exchange-list indices of one atom, as loaded (not yet masked by nj)
struct RowIdx {
    int i, nj;
    int4 w[SC_ROW / 4];
};

__device__ __forceinline__ void row_load(const Dev& D, int i, RowIdx& r) {
    r.i = i;
    r.nj = __ldg(D.jl_n + i);
    const int* row = D.jl + (size_t)i * SLD_MAXJ;
#pragma unroll
    for (int q = 0; q < SC_ROW / 8; ++q) ldg32_i8_once(row + 8 * q, r.w[2 * q], r.w[2 * q + 1]);
}

template <bool SPLIT>
struct VisitRegs {
    using JT = typename std::conditional<SPLIT, float, double>::type;
    using ST = typename std::conditional<SPLIT, float4, double4>::type;
    int i, nj;
    int jj[SC_PJ];
    JT J[SC_PJ];
    ST sj[SC_PJ];
    double4 si;
    double rho;
    double3 dS;
};

// Spin loads.  CG: through L2 only (ld.global.cg), for a kernel in which
// other blocks update spins while it runs, so that no stale copy in this
// SM's L1 is read.  The gathered neighbours keep L2's normal priority (the
// streamed rows and records are marked evict-first instead).
template <bool CG>
__device__ __forceinline__ double4 ld_spin(const double4* p) {
    if constexpr (CG) return ld32cg_d4(p);
    else return ld32_d4(p);
}
template <bool CG>
__device__ __forceinline__ float4 ld_spin(const float4* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}
// a visit's own FP64 spin in the split form (read once per visit and gathered
// by no one: streamed)
template <bool CG>
__device__ __forceinline__ double4 ld_own_spin(const double4* p) {
    if constexpr (CG) return ld32cg_d4(p);
    else return ld32_d4_once(p);
}

// everything of one visit but the indices: couplings, neighbour spins, the
// atom's own spin, rho and noise increment
template <bool SPLIT, bool CG>
__device__ __forceinline__ void visit_fetch(const Dev& D, const RowIdx& r, int sweep,
                                            VisitRegs<SPLIT>& v) {
    const int i = r.i, nj = r.nj;
    v.i = i;
    v.nj = nj;
#pragma unroll
    for (int u = 0; u < SC_PJ; ++u) {
        const int4 w = r.w[u / 4];
        const int x = (u & 3) == 0 ? w.x : (u & 3) == 1 ? w.y : (u & 3) == 2 ? w.z : w.w;
        v.jj[u] = u < nj ? x : -1;
    }
    const size_t row = (size_t)i * SLD_MAXJ;
    if constexpr (SPLIT) {
        float4 jw[SC_ROW / 4];
#pragma unroll
        for (int q = 0; q < SC_ROW / 8; ++q) ldg32_f8_once(D.jvf + row + 8 * q, jw[2 * q], jw[2 * q + 1]);
#pragma unroll
        for (int u = 0; u < SC_PJ; ++u) {
            const float4 w = jw[u / 4];
            v.J[u] = (u & 3) == 0 ? w.x : (u & 3) == 1 ? w.y : (u & 3) == 2 ? w.z : w.w;
        }
#pragma unroll
        for (int u = 0; u < SC_PJ; ++u)
            v.sj[u] = v.jj[u] >= 0 ? ld_spin<CG>(D.s32 + v.jj[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
#pragma unroll
        for (int q = 0; q < SC_ROW / 4; ++q) {
            const double4 w = ldg32_d4_once(D.jv + row + 4 * q);
            const double e[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (4 * q + u < SC_PJ) v.J[4 * q + u] = e[u];
        }
#pragma unroll
        for (int u = 0; u < SC_PJ; ++u)
            v.sj[u] = v.jj[u] >= 0 ? ld_spin<CG>(D.s + v.jj[u]) : make_double4(0, 0, 0, 0);
    }
    if constexpr (SPLIT) v.si = ld_own_spin<CG>(D.s + i);
    else v.si = ld_spin<CG>(D.s + i);
    if (D.spinlang) {
        const double4 q = ldg32_d4_once(D.vrec + 2 * (size_t)i + sweep);
        v.rho = q.x;
        v.dS = make_double3(q.y, q.z, q.w);
    } else {
        v.rho = 0.0;
        v.dS = make_double3(0.0, 0.0, 0.0);
    }
}

// sum_j J s_j and sum_j J |s_j| in exchange-list order (exchange_field's
// arithmetic: FP64, or FP32 products in Kahan sums for the split form)
template <bool SPLIT, bool CG>
__device__ __forceinline__ void visit_field(const Dev& D, const VisitRegs<SPLIT>& v, double3& H,
                                            double& sumJ) {
    double hx = 0, hy = 0, hz = 0, hj = 0;
    double4 hext = make_double4(0.0, 0.0, 0.0, 0.0);
    if (D.hext) {
        // the reference starts the field at the external one (calculate_spin_CPU.cpp:35-40)
        hext = D.hext[v.i];
        if constexpr (!SPLIT) { hx = hext.x; hy = hext.y; hz = hext.z; }
    }
    float ks[4] = {0, 0, 0, 0}, kc[4] = {0, 0, 0, 0};
    auto add32 = [&](float J, float4 s) { exch_add32(ks, kc, J, s); };
    auto add64 = [&](double J, double4 s) { exch_add64(hx, hy, hz, hj, J, s); };
#pragma unroll
    for (int u = 0; u < SC_PJ; ++u) {
        if constexpr (SPLIT) exch_add32_if(u < v.nj, ks, kc, v.J[u], v.sj[u]);
        else exch_add64_if(u < v.nj, hx, hy, hz, hj, v.J[u], v.sj[u]);
    }
    for (int e = SC_PJ; e < v.nj; ++e) {
        const size_t at = (size_t)v.i * SLD_MAXJ + e;
        const int j = D.jl[at];
        if constexpr (SPLIT) add32(D.jvf[at], ld_spin<CG>(D.s32 + j));
        else add64(D.jv[at], ld_spin<CG>(D.s + j));
    }
    if constexpr (SPLIT) {
        hx = hext.x + ((double)ks[0] - (double)kc[0]);
        hy = hext.y + ((double)ks[1] - (double)kc[1]);
        hz = hext.z + ((double)ks[2] - (double)kc[2]);
        hj = (double)ks[3] - (double)kc[3];
    }
    H = make_double3(hx, hy, hz);
    sumJ = hj;
}

// the walk of one cell c in the reference's order (backward: tail -> head);
// INTEG 0: the Heisenberg-Landau visit, 1: the Heisenberg one (SDH, SLDH)
template <bool SPLIT, bool CG, int INTEG = 0>
__device__ __forceinline__ void cell_walk(const Dev& D, int c, double dt, int backward) {
    constexpr bool kDeep = SPLIT;   // indices two visits ahead
    const int n = cell_n(D, c);
    if (n <= 0) return;
    const int* ca = D.cell_atoms + D.cell_start[c];
    const bool bwd = (backward & SW_BACKWARD) != 0;
    // the backward sweep is each atom's last visit of the call
    const bool fields = bwd && !(backward & SW_NO_FIELDS);
    const int sweep = bwd ? 1 : 0;
    auto atom_at = [&](int m) { return __ldg(ca + (bwd ? n - 1 - m : m)); };
    VisitRegs<SPLIT> v;
    RowIdx r;
    row_load(D, atom_at(0), r);
    visit_fetch<SPLIT, CG>(D, r, sweep, v);
    int i_after;          // the atom whose indices are loaded next
    if (kDeep) {
        if (n > 1) row_load(D, atom_at(1), r);
        i_after = n > 2 ? atom_at(2) : -1;
    } else {
        i_after = n > 1 ? atom_at(1) : -1;
    }
    for (int m = 0; m < n; ++m) {
        const int i = v.i;
        double3 H;
        double sumJ;
        visit_field<SPLIT, CG>(D, v, H, sumJ);
        const double3 s_old = make_double3(v.si.x, v.si.y, v.si.z);
        const double s0_old = v.si.w;
        const double rho = v.rho;
        const double3 dS = v.dS;
        const bool more = m + 1 < n;
        if (more) {
            if (kDeep) {
                visit_fetch<SPLIT, CG>(D, r, sweep, v);        // r: indices of atom m+1
                if (m + 2 < n) row_load(D, i_after, r);    // indices of atom m+2
                i_after = m + 3 < n ? atom_at(m + 3) : -1;
            } else {
                row_load(D, i_after, r);
                visit_fetch<SPLIT, CG>(D, r, sweep, v);
                i_after = m + 2 < n ? atom_at(m + 2) : -1;
            }
        }
        double3 HL = make_double3(0.0, 0.0, 0.0);
        double3 s;
        if constexpr (INTEG == 1)
            s = spin_integrate_H(D, s_old, s0_old, H, dS, dt);
        else
            s = spin_integrate_dS(D, s_old, H, sumJ, rho, dS, dt, HL);
        double s0 = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
        if (!isfinite(s0)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
        const double4 s4 = make_double4(s.x, s.y, s.z, s0);
        if constexpr (SPLIT) st32_d4_once(D.s + i, s4);
        else st32_d4(D.s + i, s4);
        const auto sr = spin_reg<SPLIT>(s4);
        if constexpr (SPLIT) D.s32[i] = sr;
        if (fields) {
            st32_d4_once(D.H + i, make_double4(H.x, H.y, H.z, 0.0));
            if constexpr (INTEG == 0) st32_d4_once(D.HL + i, make_double4(HL.x, HL.y, HL.z, 0.0));
            if (D.spinlang) D.sumJ[i] = sumJ;
        }
        if (more) {
#pragma unroll
            for (int u = 0; u < SC_PJ; ++u)
                if (v.jj[u] == i) v.sj[u] = sr;
        }
    }
}

template <bool SPLIT, int INTEG>
__global__ void __launch_bounds__(128) k_sweep_pipe(Dev D, const int* __restrict__ gcells,
                                                    int ncell_g, double dt, int backward) {
    // one cell per thread; a capped grid walks several cells per thread
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell_g; t += gridDim.x * blockDim.x)
        cell_walk<SPLIT, false, INTEG>(D, gcells[t], dt, backward);
}

// ---------------------------------------------------------------------
// Both sweeps of one core_ds call in one persistent launch, scheduled by
// data flow instead of a grid-wide barrier per colour group.
//
// The reference's order gives each visit of a cell c of group g a fixed view
// of its 26 neighbour cells:
//   forward:  neighbours of groups < g already swept forward, of groups > g
//             not yet;
//   backward: neighbours of groups > g already swept backward, of groups < g
//             swept forward but not yet backward.
// Any schedule that keeps these views gives the reference's result bit for
// bit.  Work is handed out in the reference's order (forward groups 0..G-1,
// then backward G-1..0) in tasks of at most 32 cells of one group (one warp
// each), through an atomic counter.  A cell's flag holds the tag of its last
// finished sweep (tagF = forward of this call, tagB = backward); before a
// warp walks its cells it waits until
//   forward:  every neighbour of a lower group shows tagF;
//   backward: the cell itself shows tagF, every neighbour of a higher group
//             tagB and every one of a lower group tagF.
// A neighbour that must not have moved yet cannot have: its own wait needs
// this cell's flag.  Every task depends only on earlier tasks, and a task is
// taken only by a running warp, so the earliest unfinished task can always
// proceed.  The waits are bounded: a wait that runs out sets SLD_FLAG_WAIT
// and every warp leaves; the host reports SLD_ERR_TIMEOUT.
// Tags grow by 2 per call (sync[0]); flags and tags are never reset, so
// stale flags from earlier calls are always below this call's tags.
#define FLOW_POLLS (1 << 21)     // default polls of one cell's waits (~0.2 s with the sleeps)

__device__ __forceinline__ int ld_flag(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}

__device__ __forceinline__ bool flow_wait_one(const Dev& D, const int* flag, int need, int& budget) {
    while (ld_flag(flag) < need) {
        if (--budget <= 0) return false;
        if ((budget & 255) == 0 &&
            (*reinterpret_cast<const volatile unsigned*>(&D.ctl->err) & SLD_FLAG_WAIT))
            return false;
        __nanosleep(64);
    }
    return true;
}

// The waits of one cell: all its flags and groups are read at once, and only
// the flags not yet set are polled.
__device__ bool flow_wait(const Dev& D, const SweepFlow& F, int c, int g, bool bwd, int tagF,
                          int tagB) {
    int budget = F.polls;
    int cx, cy, cz;
    cell_xyz(D, c, cx, cy, cz);
    int nb[26], fl[26], gr[26];
#pragma unroll
    for (int k = 0; k < 26; ++k) nb[k] = nbr_cell(D, cx, cy, cz, k);
#pragma unroll
    for (int k = 0; k < 26; ++k) {
        fl[k] = ld_flag(F.cell_flag + nb[k]);
        gr[k] = __ldg(F.cell_group + nb[k]);
    }
    if (bwd && !flow_wait_one(D, F.cell_flag + c, tagF, budget)) return false;
#pragma unroll
    for (int k = 0; k < 26; ++k) {
        int need;
        if (!bwd) {
            if (gr[k] > g) continue;
            need = tagF;
        } else {
            need = gr[k] > g ? tagB : tagF;
        }
        if (fl[k] < need && !flow_wait_one(D, F.cell_flag + nb[k], need, budget)) return false;
    }
    return true;
}

template <bool SPLIT>
__global__ void __launch_bounds__(128) k_sweep_flow(Dev D, SweepFlow F, double dt, int flags) {
    const int lane = threadIdx.x & 31;
    // the tags this call's waits need (F.stall > 0 asks for tags no warp
    // writes: every wait on a neighbour then runs out)
    const int tagF = F.sync[0] + 1 + F.stall, tagB = tagF + 1;
    const int putF = F.sync[0] + 1, putB = putF + 1;
    int task = 0;
    if (lane == 0) task = atomicAdd(F.sync + 1, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    while (task < F.ntasks) {
        const bool stop =
            (*reinterpret_cast<const volatile unsigned*>(&D.ctl->err) & SLD_FLAG_WAIT) != 0;
        if (__any_sync(0xffffffffu, stop)) break;
        // the warp's next task, taken now so that the atomic's round trip
        // overlaps this task (tasks stay in order per warp, so the earliest
        // unfinished task can still always proceed)
        int next = 0;
        if (lane == 0) next = atomicAdd(F.sync + 1, 1);
        const int4 tk = __ldg(F.tasks + task);   // backward, first, count, group
        const bool bwd = tk.x != 0;
        const int c = lane < tk.z ? __ldg(F.gcells + tk.y + lane) : -1;
        bool ok = c < 0 || flow_wait(D, F, c, tk.w, bwd, tagF, tagB);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicOr(&D.ctl->err, SLD_FLAG_WAIT);
            break;
        }
        if (c >= 0) {
            __threadfence();                  // the flags above before the spins below
            cell_walk<SPLIT, true>(D, c, dt, (bwd ? SW_BACKWARD : 0) | flags);
            __threadfence();                  // this cell's spins before its flag
            atomicExch(F.cell_flag + c, bwd ? putB : putF);
        }
        task = __shfl_sync(0xffffffffu, next, 0);
    }
}

// after a flow launch: the next call's tags, and the task counter back to 0
__global__ void k_flow_next(SweepFlow F) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        F.sync[0] += 2;
        F.sync[1] = 0;
    }
}

static int g_flow_blocks[2] = {0, 0};
// the waits' bound and the stall of the data-flow schedule, from the
// environment at context creation (SLD_FLOW_POLLS, SLD_FLOW_STALL): a test
// makes the waits run out with a small bound and a stall, and expects
// SLD_ERR_TIMEOUT instead of a hang
static int g_flow_polls = FLOW_POLLS, g_flow_stall = 0;

void launch_sweep_flow(const Dev& D, cudaStream_t st, const SweepFlow& F0, double dt, bool fields) {
    SweepFlow F = F0;
    F.polls = g_flow_polls;
    F.stall = g_flow_stall;
    const int flags = fields ? 0 : SW_NO_FIELDS;
    const int k = D.split ? 1 : 0;
    if (D.split)
        k_sweep_flow<true><<<g_flow_blocks[k], 128, 0, st>>>(D, F, dt, flags);
    else
        k_sweep_flow<false><<<g_flow_blocks[k], 128, 0, st>>>(D, F, dt, flags);
    k_flow_next<<<1, 32, 0, st>>>(F);
}

static int g_sms = 148;        // SMs of the device (capped sweep grids)
static int g_sweep_mode = 2;   // 1: one thread per cell, 2: one thread per cell,
                               // pipelined; one launch per group
                               // 3: the pipelined walk, scheduled by data flow

void sweep_init() {
    const char* v = getenv("SLD_SWEEP_MODE");
    if (v && v[0] >= '1' && v[0] <= '3') g_sweep_mode = v[0] - '0';
    g_flow_polls = FLOW_POLLS;
    g_flow_stall = 0;
    if (const char* q = getenv("SLD_FLOW_POLLS")) {
        long n = strtol(q, nullptr, 10);
        if (n >= 1 && n <= FLOW_POLLS) g_flow_polls = (int)n;
    }
    if (const char* q = getenv("SLD_FLOW_STALL")) {
        long n = strtol(q, nullptr, 10);
        if (n >= 0 && n <= 1000) g_flow_stall = (int)n;
    }
    int dev = 0, sms = 0, b0 = 0, b1 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms > 0) g_sms = sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_sweep_flow<false>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_sweep_flow<true>, 128, 0);
    g_flow_blocks[0] = (b0 > 0 ? b0 : 1) * sms;
    g_flow_blocks[1] = (b1 > 0 ? b1 : 1) * sms;
}

bool sweep_uses_flow() { return g_sweep_mode == 3; }

void launch_sweep(const Dev& D, cudaStream_t st, const int* gcells, int ncell_g, double dt,
                  bool backward, bool fields) {
    if (ncell_g <= 0) return;
    const int b = (backward ? SW_BACKWARD : 0) | (fields ? 0 : SW_NO_FIELDS);
    if (g_sweep_mode >= 2 || D.hint) {
        // Block sizes that fill the register file: the split form's kernel takes
        // about 200 registers a thread, 9 warps an SM, so blocks of 3 warps
        // (128-thread blocks would leave one warp's registers idle; holding it
        // to 200 registers for a tenth warp measured slower); the FP64 form's
        // 255 registers allow 8 warps, 2 blocks of 4.  The Heisenberg
        // Hamiltonians' visit has its own instance (the other sweep variants
        // have only the Heisenberg-Landau visit).
        const int bs = D.tune.sweep_block > 0 ? D.tune.sweep_block : (D.split ? 96 : 128);
        int nb = div_up(ncell_g, bs);
        // a cap on the CTAs per SM leaves registers for the kernels of the
        // graph's other branch (the pair pass, the EAM forces, core_dTe),
        // which then run beside the sweep instead of after it
        if (D.tune.sweep_cap > 0) nb = std::min(nb, D.tune.sweep_cap * g_sms);
        if (D.split) {
            if (D.hint)
                k_sweep_pipe<true, 1><<<nb, bs, 0, st>>>(D, gcells, ncell_g, dt, b);
            else
                k_sweep_pipe<true, 0><<<nb, bs, 0, st>>>(D, gcells, ncell_g, dt, b);
        } else {
            if (D.hint)
                k_sweep_pipe<false, 1><<<nb, bs, 0, st>>>(D, gcells, ncell_g, dt, b);
            else
                k_sweep_pipe<false, 0><<<nb, bs, 0, st>>>(D, gcells, ncell_g, dt, b);
        }
        return;
    }
    k_sweep_cell<<<div_up(ncell_g, 128), 128, 0, st>>>(D, gcells, ncell_g, dt, b);
}
