// Suzuki-Trotter spin sweeps (core_ds_CPU.cpp:35-83), one launch per colour
// group and direction.
//
// The reference visits the cells of colour group 0..G-1 (then G-1..0), each
// cell's atoms in list order head -> tail (then tail -> head), and each visit
// (calculate_spin_CPU.cpp:33-199) evaluates Heff_H = sum_j J(r_ij) s_j with
// the spins as they are at that moment.  Cells of one colour share no
// neighbour, so during a group's launch every spin outside the group's cells
// is frozen and only a cell's own atoms change while it is walked.  Each block
// takes 32 cells of the group and works in three phases:
//   A  one thread per atom: from the exchange list, sum the field of the
//      neighbours outside the atom's cell (frozen), note the in-cell
//      neighbours, and draw the visit's noise (counter-based, so the draw
//      does not depend on the order);
//   B  one thread per cell: walk the cell in the reference's order, add the
//      in-cell neighbours' current spins (kept in shared memory) and apply the
//      integrator (FP64);
//   C  one thread per atom: write the spins back.
// A block whose cells hold more atoms (or in-cell neighbours) than its
// shared-memory tables falls back to one thread per cell reading everything
// from global memory, with the same arithmetic.
#include <cstdlib>

#include "sld_pot32.cuh"
#include "sld_spin.cuh"

#define SW_CPB 32
#define SW_THREADS 256
#define SW_MAXA 256
#define SW_MAXIN 12

struct SweepShared {
    double s[SW_MAXA][4];           // current spin, |s|
    double h[SW_MAXA][4];           // field of the out-of-cell neighbours, sum J|s|
    double aux[SW_MAXA][5];         // rho, T, noise x y z
    double inJ[SW_MAXA][SW_MAXIN];  // J of the in-cell neighbours
    int slot[SW_MAXA];
    unsigned char inq[SW_MAXA][SW_MAXIN];   // their position in the cell list
    unsigned char inn[SW_MAXA];
    int cell[SW_CPB], cell_n[SW_CPB], cell_start[SW_CPB], cell_base[SW_CPB];
    int total, overflow;
};

__device__ __forceinline__ void visit_store(const Dev& D, int i, double3 s, double3 H, double3 HL,
                                            double sumJ, bool fields) {
    double s0 = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
    if (!isfinite(s0)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
    D.s[i] = make_double4(s.x, s.y, s.z, s0);
    if (fields) {
        D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
        D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
        if (D.spinlang) D.sumJ[i] = sumJ;
    }
}

// The normals of both sweeps of one core_ds call, drawn for every atom in
// one parallel pass before the sweeps (the draw is counter-based, so it does
// not depend on when it is made); the sweeps' serial chains only read them.
__global__ void __launch_bounds__(256) k_spin_noise(Dev D, int epoch_off) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned long long e0 = D.ctl->epoch + (unsigned long long)epoch_off;
    for (int v = 0; v < 2; ++v) {
        double3 x = normals3(D.seed, 0u, (unsigned)D.id[i], e0 + v);
        double* o = D.xi + 6 * (size_t)i + 3 * v;
        o[0] = x.x;
        o[1] = x.y;
        o[2] = x.z;
    }
}

void launch_spin_noise(const Dev& D, cudaStream_t st, int epoch_off) {
    k_spin_noise<<<div_up(D.natom, 256), 256, 0, st>>>(D, epoch_off);
}

__device__ __forceinline__ double3 spin_noise_at(const Dev& D, int i, int sweep) {
    const double* x = D.xi + 6 * (size_t)i + 3 * sweep;
    return make_double3(x[0], x[1], x[2]);
}

// one visit entirely from global memory (the fallback path)
__device__ void visit_global(const Dev& D, int i, double dt, unsigned long long epoch, bool fields) {
    double3 H;
    double sumJ;
    exchange_field(D, i, H, sumJ, [](int) { return false; }, [](int, double) {});
    double4 s4 = D.s[i];
    double T = 0.0, rho = 0.0;
    double3 xi = make_double3(0.0, 0.0, 0.0);
    if (D.spinlang) {
        T = D.eltemp ? D.Te[D.node[i]] : D.temperature;
        rho = D.rho[i];
        xi = spin_noise_at(D, i, fields ? 1 : 0);
        (void)epoch;
    }
    double3 HL;
    double3 s = spin_integrate(D, make_double3(s4.x, s4.y, s4.z), H, sumJ, rho, T, xi, dt, HL);
    visit_store(D, i, s, H, HL, sumJ, fields);
}

__global__ void __launch_bounds__(SW_THREADS) k_sweep(Dev D, const int* __restrict__ gcells,
                                                      int ncell_g, double dt, int backward,
                                                      int epoch_off) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SweepShared& S = *reinterpret_cast<SweepShared*>(smem_raw);
    const int cbeg = blockIdx.x * SW_CPB;
    const int ncb = min(SW_CPB, ncell_g - cbeg);
    const unsigned long long epoch = D.ctl->epoch + (unsigned long long)epoch_off;
    const bool fields = backward != 0;   // the backward sweep is each atom's last visit
    if (threadIdx.x < 32) {
        int lane = threadIdx.x, n = 0, st = 0, c = -1;
        if (lane < ncb) {
            c = gcells[cbeg + lane];
            n = D.cell_count[c];
            st = D.cell_start[c];
        }
        int inc = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane < ncb) {
            S.cell[lane] = c;
            S.cell_n[lane] = n;
            S.cell_start[lane] = st;
            S.cell_base[lane] = inc - n;
        }
        int total = __shfl_sync(0xffffffffu, inc, 31);
        if (lane == 0) {
            S.total = total;
            S.overflow = total > SW_MAXA ? 1 : 0;
        }
    }
    __syncthreads();
    const int total = S.total;
    if (!S.overflow) {
        // phase A
        for (int a = threadIdx.x; a < total; a += blockDim.x) {
            int q = 0;
            while (q + 1 < ncb && S.cell_base[q + 1] <= a) ++q;
            int i = D.cell_atoms[S.cell_start[q] + (a - S.cell_base[q])];
            int c = S.cell[q];
            S.slot[a] = i;
            double4 si = D.s[i];
            S.s[a][0] = si.x; S.s[a][1] = si.y; S.s[a][2] = si.z; S.s[a][3] = si.w;
            int nin = 0;
            const int cst = S.cell_start[q], cn = S.cell_n[q];
            double3 Ho;
            double hjo;
            exchange_field(
                D, i, Ho, hjo, [&](int j) { return D.cell_of[j] == c; },
                [&](int j, double J) {
                    int pos = 0;
                    while (pos < cn && D.cell_atoms[cst + pos] != j) ++pos;
                    if (nin < SW_MAXIN) {
                        S.inq[a][nin] = (unsigned char)pos;
                        S.inJ[a][nin] = J;
                    }
                    ++nin;
                });
            S.h[a][0] = Ho.x; S.h[a][1] = Ho.y; S.h[a][2] = Ho.z; S.h[a][3] = hjo;
            S.inn[a] = (unsigned char)(nin < SW_MAXIN ? nin : SW_MAXIN);
            if (nin > SW_MAXIN) S.overflow = 1;
            if (D.spinlang) {
                double3 xi = spin_noise_at(D, i, fields ? 1 : 0);
                S.aux[a][0] = D.rho[i];
                S.aux[a][1] = D.eltemp ? D.Te[D.node[i]] : D.temperature;
                S.aux[a][2] = xi.x; S.aux[a][3] = xi.y; S.aux[a][4] = xi.z;
            }
        }
        __syncthreads();
        if (!S.overflow) {
            // phase B
            if (threadIdx.x < ncb) {
                int q = threadIdx.x, n = S.cell_n[q], b = S.cell_base[q];
                for (int t = 0; t < n; ++t) {
                    int a = b + (backward ? n - 1 - t : t);
                    double3 H = make_double3(S.h[a][0], S.h[a][1], S.h[a][2]);
                    double sumJ = S.h[a][3];
                    for (int e = 0; e < S.inn[a]; ++e) {
                        int a2 = b + S.inq[a][e];
                        double J = S.inJ[a][e];
                        H.x += J * S.s[a2][0]; H.y += J * S.s[a2][1]; H.z += J * S.s[a2][2];
                        sumJ += J * S.s[a2][3];
                    }
                    double3 HL;
                    double3 s = spin_integrate(
                        D, make_double3(S.s[a][0], S.s[a][1], S.s[a][2]), H, sumJ, S.aux[a][0],
                        S.aux[a][1], make_double3(S.aux[a][2], S.aux[a][3], S.aux[a][4]), dt, HL);
                    double s0 = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
                    S.s[a][0] = s.x; S.s[a][1] = s.y; S.s[a][2] = s.z; S.s[a][3] = s0;
                    if (fields) {
                        int i = S.slot[a];
                        D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
                        D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
                        if (D.spinlang) D.sumJ[i] = sumJ;
                    }
                }
            }
            __syncthreads();
            // phase C
            for (int a = threadIdx.x; a < total; a += blockDim.x) {
                double s0 = S.s[a][3];
                if (!isfinite(s0)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
                D.s[S.slot[a]] = make_double4(S.s[a][0], S.s[a][1], S.s[a][2], s0);
            }
            return;
        }
    }
    // fallback: one thread per cell, from global memory
    if (threadIdx.x < ncb) {
        int q = threadIdx.x, n = S.cell_n[q], st = S.cell_start[q];
        for (int t = 0; t < n; ++t) {
            int i = D.cell_atoms[st + (backward ? n - 1 - t : t)];
            visit_global(D, i, dt, epoch, fields);
        }
    }
}

// one thread per cell for the whole visit, reading the spins from global
// memory (no shared-memory phases)
__global__ void __launch_bounds__(128) k_sweep_cell(Dev D, const int* __restrict__ gcells,
                                                    int ncell_g, double dt, int backward,
                                                    int epoch_off) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell_g) return;
    int c = gcells[t];
    int st = D.cell_start[c], n = D.cell_count[c];
    unsigned long long epoch = D.ctl->epoch + (unsigned long long)epoch_off;
    bool fields = backward != 0;
    for (int m = 0; m < n; ++m) {
        int i = D.cell_atoms[st + (backward ? n - 1 - m : m)];
        visit_global(D, i, dt, epoch, fields);
    }
}

static size_t sweep_smem() { return sizeof(SweepShared); }
static int g_sweep_mode = 1;   // 0: two-level (shared memory), 1: one thread per cell

void sweep_init() {
    cudaFuncSetAttribute(k_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem());
    const char* v = getenv("SLD_SWEEP_MODE");
    if (v && (v[0] == '0' || v[0] == '1')) g_sweep_mode = v[0] - '0';
}

void launch_sweep(const Dev& D, cudaStream_t st, const int* gcells, int ncell_g, double dt,
                  bool backward, int epoch_off) {
    if (ncell_g <= 0) return;
    if (g_sweep_mode == 1) {
        k_sweep_cell<<<div_up(ncell_g, 128), 128, 0, st>>>(D, gcells, ncell_g, dt, backward ? 1 : 0,
                                                          epoch_off);
        return;
    }
    k_sweep<<<div_up(ncell_g, SW_CPB), SW_THREADS, sweep_smem(), st>>>(D, gcells, ncell_g, dt,
                                                                       backward ? 1 : 0, epoch_off);
}
