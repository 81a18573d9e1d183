// Electron-temperature subsystem and the energy bookkeeping.
//
//   calculate_temperature  calculate_temperature_CPU.cpp:35-148
//   core_dTe               core_dTe_CPU.cpp:47-217 (A B C B A per substep)
//   check_energy           check_energy_CPU.cpp:33-111 (renormalisation)
//
// Te cells are the link cells (as in the reference) or the nodes of a mesh
// decoupled from them.  core_dTe is one launch of a single 1024-thread block
// that runs every substep: the Te arrays are small (one value per cell) and
// the colour-ordered diffusion sweep needs a barrier between colour groups,
// which a block barrier gives cheaply.
#include <cooperative_groups.h>
#include <cstdlib>

#include "sld_pot32.cuh"

// Heff_H and sum_j J |s_j| (inner_spin / inner_sum_Jij_sj) from the
// exchange list
__device__ __forceinline__ void gather_field_t(const Dev& D, int i, double3& H, double& sumJ) {
    exchange_field(D, i, H, sumJ, [](int) { return false; }, [](int, double) {});
}

// per-atom terms of calculate_temperature; writes H, HL, sumJ and returns
// the five sums (R_up, R_dn, L_up, L_dn) it contributes
__device__ __forceinline__ void temp_atom(const Dev& D, int i, double& Rup, double& Rdn, double& Lup,
                                          double& Ldn) {
    double3 H;
    double sumJ;
    gather_field_t(D, i, H, sumJ);
    double4 s4 = D.s[i];
    double3 s = make_double3(s4.x, s4.y, s4.z);
    double cx_ = s.y * H.z - H.y * s.z, cy_ = s.z * H.x - H.z * s.x, cz_ = s.x * H.y - H.x * s.y;
    Rup = cx_ * cx_ + cy_ * cy_ + cz_ * cz_;
    Rdn = s.x * H.x + s.y * H.y + s.z * H.z;
    double rho = D.rho[i];
    double A = interp_const(D.landau[0], rho, D.inv_rho);
    double B = interp_const(D.landau[1], rho, D.inv_rho);
    double C = interp_const(D.landau[2], rho, D.inv_rho);
    double Dd = interp_const(D.landau[3], rho, D.inv_rho);
    double s_sq = s.x * s.x + s.y * s.y + s.z * s.z;
    double s0 = sqrt(s_sq);
    double c = -(2.0 * A + 4.0 * B * s_sq + 6.0 * C * (s_sq * s_sq) + 8.0 * Dd * (s_sq * s_sq * s_sq));
    double k = -sumJ / s0;
    double3 HL = make_double3(c * s.x + k * s.x, c * s.y + k * s.y, c * s.z + k * s.z);
    double hx = H.x + HL.x, hy = H.y + HL.y, hz = H.z + HL.z;
    Lup = hx * hx + hy * hy + hz * hz;
    Ldn = 6.0 * A + 20.0 * B * s_sq + 42.0 * C * (s_sq * s_sq) + 72.0 * Dd * (s_sq * s_sq * s_sq);
    Ldn += 2.0 * sumJ / s0;
    D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
    D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
    D.sumJ[i] = sumJ;
}

// per-Te-cell results from the sums (calculate_temperature_CPU.cpp:118-142)
__device__ __forceinline__ void temp_finish(const Dev& D, int k, double n, double sum_ke, double apx,
                                            double apy, double apz, double Rup, double Rdn, double Lup,
                                            double Ldn) {
    double per = (double)D.natom / (double)D.nte;
    if (D.localcolmot) {
        apx = apx / n; apy = apy / n; apz = apz / n;
        sum_ke -= n * (apx * apx + apy * apy + apz * apz) / 2.0 / D.atmass;
        D.Tl[k] = 2.0 / 3.0 * sum_ke / (n - 1.0) / SLD_BOLTZ;
        D.Gel[k] = 3.0 * (n - 1.0) * SLD_BOLTZ * D.gamma_L / D.atmass / per;
    } else {
        D.Tl[k] = sum_ke * 2.0 / 3.0 / n / SLD_BOLTZ;
        D.Gel[k] = 3.0 * n * SLD_BOLTZ * D.gamma_L / D.atmass / per;
    }
    D.TsR[k] = Rup / Rdn / 2.0 / SLD_BOLTZ;
    D.TsL[k] = Lup / Ldn / SLD_BOLTZ;
    D.Ges[k] = SLD_BOLTZ * D.gamma_S_HL * Ldn / per;
}

// Te on link cells: one thread per cell, atoms in list order (the
// reference's summation order)
__global__ void __launch_bounds__(128) k_temp_cell(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.ncells) return;
    int st = D.cell_start[c], n = D.cell_count[c];
    double ke = 0, ax = 0, ay = 0, az = 0, Rup = 0, Rdn = 0, Lup = 0, Ldn = 0;
    for (int m = 0; m < n; ++m) {
        int i = D.cell_atoms[st + m];
        ke += D.ke[i];
        double4 p = D.p[i];
        ax += p.x; ay += p.y; az += p.z;
        double a, b, e, f;
        temp_atom(D, i, a, b, e, f);
        Rup += a; Rdn += b; Lup += e; Ldn += f;
    }
    temp_finish(D, c, (double)n, ke, ax, ay, az, Rup, Rdn, Lup, Ldn);
}

// Te on a mesh: per-atom terms added into the node accumulators
__global__ void __launch_bounds__(128) k_temp_atom(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double a, b, e, f;
    temp_atom(D, i, a, b, e, f);
    double4 p = D.p[i];
    // Atoms are stored cell by cell, so neighbouring lanes mostly share a
    // node: a segmented warp scan (segments = runs of equal node, marked by
    // head flags) sums each run, and the run's last lane does the atomics.
    // Lanes past natom have returned; the active lanes are a prefix.
    int node = D.node[i];
    double v[8] = {D.ke[i], p.x, p.y, p.z, a, b, e, f};
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    int prev = __shfl_up_sync(act, node, 1);
    int head = (lane == 0 || prev != node) ? 1 : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int th = __shfl_up_sync(act, head, o);
        double t[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) t[q] = __shfl_up_sync(act, v[q], o);
        if (lane >= o) {
            if (!head) {
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] += t[q];
            }
            head |= th;
        }
    }
    int nxt = __shfl_down_sync(act, node, 1);
    bool last = lane == 31 || !((act >> (lane + 1)) & 1u) || nxt != node;
    if (last) {
        double* acc = D.acc + 9 * (size_t)node;
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(acc + q, v[q]);
    }
}

__global__ void k_temp_node(Dev D) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nte) return;
    const double* a = D.acc + 9 * (size_t)k;
    temp_finish(D, k, (double)D.te_count[k], a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]);
}

void launch_temperature(const Dev& D, cudaStream_t st) {
    if (D.te_mesh > 0) {
        cudaMemsetAsync(D.acc, 0, sizeof(double) * 9 * (size_t)D.nte, st);
        k_temp_atom<<<div_up(D.natom, 128), 128, 0, st>>>(D);
        k_temp_node<<<div_up(D.nte, 128), 128, 0, st>>>(D);
    } else {
        k_temp_cell<<<div_up(D.ncells, 128), 128, 0, st>>>(D);
    }
}

// ---------------------------------------------------------------------
// core_dTe: nloop substeps of A(h/2) B(h/2) C(h) B(h/2) A(h/2)

__device__ __forceinline__ void dte_A(const Dev& D, double dt) {
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = te_to_Ee(D.Te[k]);
        double dE = 0.0;
        dE += D.Gel[k] * D.Tl[k];
        dE += D.Ges[k] * D.TsL[k];
        Ee += dt * dE;
        D.Ee[k] = Ee;
        D.Te[k] = Ee_to_te(Ee);
    }
}

__device__ __forceinline__ void dte_B(const Dev& D, double dt) {
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double g = 0.0;
        g += D.Gel[k];
        g += D.Ges[k];
        g *= dt / SLD_BOLTZ;
        double T0 = D.Te[k];
        double k1 = T0 * (exp(-g / te_Ce(T0)) - 1.0) / dt;
        double T1 = T0 + k1 * dt / 2.0;
        double k2 = T1 * (exp(-g / te_Ce(T1)) - 1.0) / dt;
        double T2 = T0 + k2 * dt / 2.0;
        double k3 = T2 * (exp(-g / te_Ce(T2)) - 1.0) / dt;
        double T3 = T0 + k3 * dt;
        double k4 = T3 * (exp(-g / te_Ce(T3)) - 1.0) / dt;
        D.Te[k] = T0 + dt / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
    }
}

__device__ __forceinline__ double dte_total_Ee(const Dev& D, double* sh) {
    double acc = 0.0;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double e = te_to_Ee(D.Te[k]);
        D.Ee[k] = e;
        acc += e;
    }
    double t = block_sum(acc, sh);
    __shared__ double tot;
    if (threadIdx.x == 0) tot = t;
    __syncthreads();
    return tot;
}

__device__ __forceinline__ void dte_C(const Dev& D, double dt, double* sh) {
    double start = dte_total_Ee(D, sh);
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    double dx2 = lx * lx, dy2 = ly * ly, dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    double pre = dt / 2.0 * cond * volume_factor / SLD_BOLTZ;
    int tx = D.tx, ty = D.ty, tz = D.tz;
    for (int pass = 0; pass < 2; ++pass) {
        for (int gg = 0; gg < D.te_ngroups; ++gg) {
            int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
            int b = D.te_gstart[g], e = D.te_gstart[g + 1];
            for (int m = b + threadIdx.x; m < e; m += blockDim.x) {
                int k = D.te_gcells[m];
                int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
                int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
                int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
                int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
                const double* Te = D.Te;
                double T = Te[k];
                double Ee = te_to_Ee(T);
                double ex = Te[xp + (y + z * ty) * tx] + Te[xm + (y + z * ty) * tx] - 2.0 * T;
                double ey = Te[x + (yp + z * ty) * tx] + Te[x + (ym + z * ty) * tx] - 2.0 * T;
                double ez = Te[x + (y + zp * ty) * tx] + Te[x + (y + zm * ty) * tx] - 2.0 * T;
                Ee += pre * (ex / dx2 + ey / dy2 + ez / dz2);
                D.Ee[k] = Ee;
                D.Te[k] = Ee_to_te(Ee);
            }
            __syncthreads();
        }
    }
    double end = dte_total_Ee(D, sh);
    double fac = start / end;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = D.Ee[k] * fac;
        D.Ee[k] = Ee;
        D.Te[k] = Ee_to_te(Ee);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(1024) k_dte(Dev D, double dt) {
    __shared__ double sh[32];
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop;
    for (int it = 0; it < nloop; ++it) {
        dte_A(D, h / 2.0);
        __syncthreads();
        dte_B(D, h / 2.0);
        __syncthreads();
        dte_C(D, h, sh);
        dte_B(D, h / 2.0);
        __syncthreads();
        dte_A(D, h / 2.0);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------
// core_dTe on a thread-block cluster: the Te cells are split over the
// cluster's CTAs (each thread owns the same cells in every phase, so A and B
// need no barrier); the colour phases of the diffusion sweep and the two
// energy sums of C synchronise the cluster with its hardware barrier.  Te is
// read across CTAs through L2 (ld.global.cg) after the barrier.

namespace cg = cooperative_groups;

__device__ __forceinline__ double cl_total(const Dev& D, double v, double* sh, double* slot_base,
                                           cg::cluster_group& cl) {
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) __stcg(slot_base + cl.block_rank(), t);
    cl.sync();
    double tot = 0.0;
    for (unsigned r = 0; r < cl.num_blocks(); ++r) tot += __ldcg(slot_base + r);
    return tot;
}

__global__ void __launch_bounds__(256) k_dte_cluster(Dev D, double dt) {
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double sh[32];
    const int nb = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int per = (D.nte + nb - 1) / nb;
    const int k0 = rank * per, k1 = min(D.nte, k0 + per);
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop;
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    double dx2 = lx * lx, dy2 = ly * ly, dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    double pre = h / 2.0 * cond * volume_factor / SLD_BOLTZ;
    const int tx = D.tx, ty = D.ty, tz = D.tz;
    double* slots = D.red;   // 2 x num_blocks partial sums
    for (int it = 0; it < nloop; ++it) {
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
            // A(h/2), B(h/2)
            double T = __ldcg(D.Te + k);
            double Ee = te_to_Ee(T);
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            Ee += (h / 2.0) * dE;
            T = Ee_to_te(Ee);
            double hh = h / 2.0;
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            double k1_ = T * (exp(-g / te_Ce(T)) - 1.0) / hh;
            double T1 = T + k1_ * hh / 2.0;
            double k2_ = T1 * (exp(-g / te_Ce(T1)) - 1.0) / hh;
            double T2 = T + k2_ * hh / 2.0;
            double k3_ = T2 * (exp(-g / te_Ce(T2)) - 1.0) / hh;
            double T3 = T + k3_ * hh;
            double k4_ = T3 * (exp(-g / te_Ce(T3)) - 1.0) / hh;
            T = T + hh / 6.0 * (k1_ + 2.0 * k2_ + 2.0 * k3_ + k4_);
            __stcg(D.Te + k, T);
        }
        // C(h): start sum, colour sweep forward and back, end sum, rescale
        double part = 0.0;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) part += te_to_Ee(__ldcg(D.Te + k));
        double start = cl_total(D, part, sh, slots, cl);
        for (int pass = 0; pass < 2; ++pass) {
            for (int gg = 0; gg < D.te_ngroups; ++gg) {
                int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
                for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
                    if (D.te_color[k] != g) continue;
                    int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
                    int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
                    int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
                    int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
                    double T = __ldcg(D.Te + k);
                    double Ee = te_to_Ee(T);
                    double ex = __ldcg(D.Te + xp + (y + z * ty) * tx) + __ldcg(D.Te + xm + (y + z * ty) * tx) - 2.0 * T;
                    double ey = __ldcg(D.Te + x + (yp + z * ty) * tx) + __ldcg(D.Te + x + (ym + z * ty) * tx) - 2.0 * T;
                    double ez = __ldcg(D.Te + x + (y + zp * ty) * tx) + __ldcg(D.Te + x + (y + zm * ty) * tx) - 2.0 * T;
                    Ee += pre * (ex / dx2 + ey / dy2 + ez / dz2);
                    __stcg(D.Te + k, Ee_to_te(Ee));
                }
                cl.sync();
            }
        }
        part = 0.0;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) part += te_to_Ee(__ldcg(D.Te + k));
        double end = cl_total(D, part, sh, slots + nb, cl);
        double fac = start / end;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
            // rescale, then B(h/2), A(h/2)
            double Ee = te_to_Ee(__ldcg(D.Te + k)) * fac;
            double T = Ee_to_te(Ee);
            double hh = h / 2.0;
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            double k1_ = T * (exp(-g / te_Ce(T)) - 1.0) / hh;
            double T1 = T + k1_ * hh / 2.0;
            double k2_ = T1 * (exp(-g / te_Ce(T1)) - 1.0) / hh;
            double T2 = T + k2_ * hh / 2.0;
            double k3_ = T2 * (exp(-g / te_Ce(T2)) - 1.0) / hh;
            double T3 = T + k3_ * hh;
            double k4_ = T3 * (exp(-g / te_Ce(T3)) - 1.0) / hh;
            T = T + hh / 6.0 * (k1_ + 2.0 * k2_ + 2.0 * k3_ + k4_);
            Ee = te_to_Ee(T);
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            Ee += (h / 2.0) * dE;
            D.Ee[k] = Ee;
            __stcg(D.Te + k, Ee_to_te(Ee));
        }
        cl.sync();   // the next substep reads neighbours' Te and reuses the slots
    }
}

// The same with the Te cells held in the CTAs' shared memory: CTA r keeps
// cells [r*per, (r+1)*per) and f(Te) = Te_to_Ee(Te) beside each Te; cells of
// other CTAs are read through distributed shared memory.  The value of f is
// refreshed whenever its Te changes, so the reference's repeated
// Te_to_Ee(Te) calls on an unchanged Te become reads.

__device__ __forceinline__ double dte_rk4(double T, double g, double hh) {
    double k1_ = T * (exp(-g / te_Ce(T)) - 1.0) / hh;
    double T1 = T + k1_ * hh / 2.0;
    double k2_ = T1 * (exp(-g / te_Ce(T1)) - 1.0) / hh;
    double T2 = T + k2_ * hh / 2.0;
    double k3_ = T2 * (exp(-g / te_Ce(T2)) - 1.0) / hh;
    double T3 = T + k3_ * hh;
    double k4_ = T3 * (exp(-g / te_Ce(T3)) - 1.0) / hh;
    return T + hh / 6.0 * (k1_ + 2.0 * k2_ + 2.0 * k3_ + k4_);
}

__device__ __forceinline__ double dsm_total(double v, double* sh, double* part, int slot,
                                            cg::cluster_group& cl) {
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) part[slot] = t;
    cl.sync();
    double tot = 0.0;
    for (unsigned r = 0; r < cl.num_blocks(); ++r) tot += cl.map_shared_rank(part, r)[slot];
    return tot;
}

__global__ void __launch_bounds__(256) k_dte_dsm(Dev D, double dt, int per) {
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) double dsm[];
    double* sT = dsm;            // Te of the owned cells
    double* sE = dsm + per;      // Te_to_Ee(Te) of the same cells
    double* part = dsm + 2 * per;
    __shared__ double sh[32];
    const int rank = (int)cl.block_rank();
    const int k0 = rank * per, k1 = min(D.nte, k0 + per), nown = max(0, k1 - k0);
    for (int l = threadIdx.x; l < nown; l += blockDim.x) {
        double T = D.Te[k0 + l];
        sT[l] = T;
        sE[l] = te_to_Ee(T);
    }
    cl.sync();
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop, hh = h / 2.0;
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    double dx2 = lx * lx, dy2 = ly * ly, dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    double pre = h / 2.0 * cond * volume_factor / SLD_BOLTZ;
    const int tx = D.tx, ty = D.ty, tz = D.tz;
    auto Tat = [&](int n) -> double {
        int o = n / per, l = n - o * per;
        return o == rank ? sT[l] : cl.map_shared_rank(sT, o)[l];
    };
    for (int it = 0; it < nloop; ++it) {
        // A(h/2) then B(h/2)
        for (int l = threadIdx.x; l < nown; l += blockDim.x) {
            int k = k0 + l;
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double Ee = sE[l] + hh * dE;
            double T = Ee_to_te(Ee);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            sT[l] = T;
            sE[l] = te_to_Ee(T);
        }
        // C(h)
        double acc = 0.0;
        for (int l = threadIdx.x; l < nown; l += blockDim.x) acc += sE[l];
        double start = dsm_total(acc, sh, part, 0, cl);
        for (int pass = 0; pass < 2; ++pass) {
            for (int gg = 0; gg < D.te_ngroups; ++gg) {
                int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
                for (int l = threadIdx.x; l < nown; l += blockDim.x) {
                    int k = k0 + l;
                    if (D.te_color[k] != g) continue;
                    int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
                    int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
                    int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
                    int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
                    double T = sT[l];
                    double ex = Tat(xp + (y + z * ty) * tx) + Tat(xm + (y + z * ty) * tx) - 2.0 * T;
                    double ey = Tat(x + (yp + z * ty) * tx) + Tat(x + (ym + z * ty) * tx) - 2.0 * T;
                    double ez = Tat(x + (y + zp * ty) * tx) + Tat(x + (y + zm * ty) * tx) - 2.0 * T;
                    double Ee = sE[l] + pre * (ex / dx2 + ey / dy2 + ez / dz2);
                    T = Ee_to_te(Ee);
                    sT[l] = T;
                    sE[l] = te_to_Ee(T);
                }
                cl.sync();
            }
        }
        acc = 0.0;
        for (int l = threadIdx.x; l < nown; l += blockDim.x) acc += sE[l];
        double end = dsm_total(acc, sh, part, 1, cl);
        double fac = start / end;
        // rescale, B(h/2), A(h/2)
        for (int l = threadIdx.x; l < nown; l += blockDim.x) {
            int k = k0 + l;
            double T = Ee_to_te(sE[l] * fac);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double Ee = te_to_Ee(T) + hh * dE;
            T = Ee_to_te(Ee);
            sT[l] = T;
            sE[l] = te_to_Ee(T);
            if (it == nloop - 1) D.Ee[k] = Ee;
        }
    }
    for (int l = threadIdx.x; l < nown; l += blockDim.x) D.Te[k0 + l] = sT[l];
    cl.sync();   // no CTA may exit while another still reads its shared memory
}

// The whole Te mesh in one CTA's shared memory (meshes up to kBlockMaxCells
// cells): block barriers between the colour phases instead of cluster ones.
static const int kBlockMaxCells = 12000;

__global__ void __launch_bounds__(1024) k_dte_block(Dev D, double dt) {
    extern __shared__ __align__(16) double bsm[];
    const int n = D.nte;
    double* sT = bsm;
    double* sE = bsm + n;
    __shared__ double sh[32];
    __shared__ double tot;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double T = D.Te[k];
        sT[k] = T;
        sE[k] = te_to_Ee(T);
    }
    __syncthreads();
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop, hh = h / 2.0;
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    double dx2 = lx * lx, dy2 = ly * ly, dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    double pre = h / 2.0 * cond * volume_factor / SLD_BOLTZ;
    const int tx = D.tx, ty = D.ty, tz = D.tz;
    for (int it = 0; it < nloop; ++it) {
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += blockDim.x) {   // A(h/2), B(h/2)
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double T = Ee_to_te(sE[k] + hh * dE);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            sT[k] = T;
            sE[k] = te_to_Ee(T);
        }
        double acc = 0.0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) acc += sE[k];
        double t = block_sum(acc, sh);
        if (threadIdx.x == 0) tot = t;
        __syncthreads();
        double start = tot;
        for (int pass = 0; pass < 2; ++pass) {
            for (int gg = 0; gg < D.te_ngroups; ++gg) {
                int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
                int b = D.te_gstart[g], e = D.te_gstart[g + 1];
                for (int m = b + threadIdx.x; m < e; m += blockDim.x) {
                    int k = D.te_gcells[m];
                    int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
                    int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
                    int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
                    int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
                    double T = sT[k];
                    double ex = sT[xp + (y + z * ty) * tx] + sT[xm + (y + z * ty) * tx] - 2.0 * T;
                    double ey = sT[x + (yp + z * ty) * tx] + sT[x + (ym + z * ty) * tx] - 2.0 * T;
                    double ez = sT[x + (y + zp * ty) * tx] + sT[x + (y + zm * ty) * tx] - 2.0 * T;
                    T = Ee_to_te(sE[k] + pre * (ex / dx2 + ey / dy2 + ez / dz2));
                    sT[k] = T;
                    sE[k] = te_to_Ee(T);
                }
                __syncthreads();
            }
        }
        acc = 0.0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) acc += sE[k];
        t = block_sum(acc, sh);
        if (threadIdx.x == 0) tot = t;
        __syncthreads();
        double fac = start / tot;
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += blockDim.x) {   // rescale, B(h/2), A(h/2)
            double T = Ee_to_te(sE[k] * fac);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double Ee = te_to_Ee(T) + hh * dE;
            T = Ee_to_te(Ee);
            sT[k] = T;
            sE[k] = te_to_Ee(T);
            if (it == nloop - 1) D.Ee[k] = Ee;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) D.Te[k] = sT[k];
}

// Cluster "hub" form: every CTA of a 4-CTA cluster does the cell-local A and
// B parts for its share of the cells in parallel; CTA 0 holds all Te and
// Te_to_Ee(Te) in its shared memory (the others read and write them through
// distributed shared memory) and runs C's colour phases with block barriers.
// Two cluster barriers per substep instead of one per colour phase.
#define HUB_CL 4
__global__ void __launch_bounds__(1024) k_dte_hub(Dev D, double dt, int per) {
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) double hsm[];
    const int n = D.nte;
    const int rank = (int)cl.block_rank();
    double* hT = cl.map_shared_rank(hsm, 0);   // the hub's arrays
    double* hE = hT + n;
    double* hfac = hT + 2 * n;
    __shared__ double sh[32];
    const int k0 = rank * per, k1 = min(n, k0 + per);
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        double T = D.Te[k];
        hT[k] = T;
        hE[k] = te_to_Ee(T);
    }
    cl.sync();
    int nloop = D.te_nloop > 0 ? D.te_nloop : 50;
    double h = dt / nloop, hh = h / 2.0;
    double cond = D.kappa_e / SLD_EVTOJ / 1e10;
    double lx = D.box_len[0] / D.tx, ly = D.box_len[1] / D.ty, lz = D.box_len[2] / D.tz;
    double dx2 = lx * lx, dy2 = ly * ly, dz2 = lz * lz;
    double atomic_volume = D.box_volume / (double)D.natom;
    double volume_factor = atomic_volume / ((double)D.natom / (double)D.nte);
    double pre = h / 2.0 * cond * volume_factor / SLD_BOLTZ;
    const int tx = D.tx, ty = D.ty, tz = D.tz;
    double lastE[4];   // this thread's last A-step energies (per = 1024 -> <= 1 per thread)
    for (int it = 0; it < nloop; ++it) {
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {   // A(h/2), B(h/2)
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double T = Ee_to_te(hE[k] + hh * dE);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            hT[k] = T;
            hE[k] = te_to_Ee(T);
        }
        cl.sync();
        if (rank == 0) {   // C(h) on the hub
            double acc = 0.0;
            for (int k = threadIdx.x; k < n; k += blockDim.x) acc += hsm[n + k];
            double t = block_sum(acc, sh);
            __shared__ double tot;
            if (threadIdx.x == 0) tot = t;
            __syncthreads();
            double start = tot;
            for (int pass = 0; pass < 2; ++pass) {
                for (int gg = 0; gg < D.te_ngroups; ++gg) {
                    int g = pass == 0 ? gg : D.te_ngroups - 1 - gg;
                    int b = D.te_gstart[g], e = D.te_gstart[g + 1];
                    for (int m = b + threadIdx.x; m < e; m += blockDim.x) {
                        int k = D.te_gcells[m];
                        int x = k % tx, y = (k / tx) % ty, z = k / (tx * ty);
                        int xp = x + 1 == tx ? 0 : x + 1, xm = x == 0 ? tx - 1 : x - 1;
                        int yp = y + 1 == ty ? 0 : y + 1, ym = y == 0 ? ty - 1 : y - 1;
                        int zp = z + 1 == tz ? 0 : z + 1, zm = z == 0 ? tz - 1 : z - 1;
                        const double* sT = hsm;
                        double T = sT[k];
                        double ex = sT[xp + (y + z * ty) * tx] + sT[xm + (y + z * ty) * tx] - 2.0 * T;
                        double ey = sT[x + (yp + z * ty) * tx] + sT[x + (ym + z * ty) * tx] - 2.0 * T;
                        double ez = sT[x + (y + zp * ty) * tx] + sT[x + (y + zm * ty) * tx] - 2.0 * T;
                        T = Ee_to_te(hsm[n + k] + pre * (ex / dx2 + ey / dy2 + ez / dz2));
                        hsm[k] = T;
                        hsm[n + k] = te_to_Ee(T);
                    }
                    __syncthreads();
                }
            }
            acc = 0.0;
            for (int k = threadIdx.x; k < n; k += blockDim.x) acc += hsm[n + k];
            t = block_sum(acc, sh);
            if (threadIdx.x == 0) hsm[2 * n] = start / t;
        }
        cl.sync();
        double fac = *hfac;
        int q = 0;
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x, ++q) {   // rescale, B, A
            double T = Ee_to_te(hE[k] * fac);
            double g = 0.0;
            g += D.Gel[k];
            g += D.Ges[k];
            g *= hh / SLD_BOLTZ;
            T = dte_rk4(T, g, hh);
            double dE = 0.0;
            dE += D.Gel[k] * D.Tl[k];
            dE += D.Ges[k] * D.TsL[k];
            double Ee = te_to_Ee(T) + hh * dE;
            T = Ee_to_te(Ee);
            hT[k] = T;
            hE[k] = te_to_Ee(T);
            if (q < 4) lastE[q] = Ee;
        }
    }
    int q = 0;
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x, ++q) {
        D.Te[k] = hT[k];
        if (q < 4) D.Ee[k] = lastE[q];
    }
    cl.sync();   // keep the hub's shared memory alive until every CTA is done
}

static int g_dte_cluster = 0;   // cluster size in use, 0: single block
static int g_dte_mode = 2;      // 0: one CTA; 1: cluster, cells spread; 2: cluster hub
static bool g_hub_ok = false;
static const int kDsmMaxPer = 12000;   // Te cells per CTA held in shared memory

int dte_init(int device) {
    (void)device;
    if (g_dte_cluster) return g_dte_cluster;
    cudaFuncSetAttribute(k_dte_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double) * 2 * kBlockMaxCells));
    const char* m = getenv("SLD_DTE_MODE");
    if (m && (m[0] == '0' || m[0] == '1' || m[0] == '2')) g_dte_mode = m[0] - '0';
    cudaFuncSetAttribute(k_dte_hub, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double) * (2 * kBlockMaxCells + 2)));
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(HUB_CL);
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = sizeof(double) * (2 * kBlockMaxCells + 2);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = HUB_CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nclu = 0;
        g_hub_ok = cudaOccupancyMaxActiveClusters(&nclu, k_dte_hub, &cfg) == cudaSuccess && nclu > 0;
        cudaGetLastError();
    }
    const char* v = getenv("SLD_DTE_SINGLE");
    if (v && v[0] == '1') return 0;
    cudaFuncSetAttribute(k_dte_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_dte_dsm, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_dte_dsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double) * (2 * kDsmMaxPer + 4)));
    for (int cs : {16, 8, 4}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(256);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_dte_cluster, &cfg) == cudaSuccess && n > 0) {
            g_dte_cluster = cs;
            break;
        }
        cudaGetLastError();
    }
    return g_dte_cluster;
}

void launch_dte(const Dev& D, cudaStream_t st, double dt) {
    int hub_per = (D.nte + HUB_CL - 1) / HUB_CL;
    if (g_dte_mode == 2 && g_hub_ok && D.nte <= kBlockMaxCells && hub_per <= 4 * 1024) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(HUB_CL);
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = sizeof(double) * (2 * D.nte + 2);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = HUB_CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_dte_hub, D, dt, hub_per);
        return;
    }
    if ((g_dte_mode == 0 || g_dte_cluster == 0) && D.nte <= kBlockMaxCells) {
        k_dte_block<<<1, 1024, sizeof(double) * 2 * D.nte, st>>>(D, dt);
        return;
    }
    if (g_dte_cluster > 0 && (D.nte + g_dte_cluster - 1) / g_dte_cluster <= kDsmMaxPer) {
        int per = (D.nte + g_dte_cluster - 1) / g_dte_cluster;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g_dte_cluster);
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = sizeof(double) * (2 * per + 4);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g_dte_cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_dte_dsm, D, dt, per);
        return;
    }
    if (g_dte_cluster > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g_dte_cluster);
        cfg.blockDim = dim3(256);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g_dte_cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_dte_cluster, D, dt);
        return;
    }
    k_dte<<<1, 1024, 0, st>>>(D, dt);
}

// ---------------------------------------------------------------------
// check_energy: averages and, with renormalizeEnergy, the energy error
// moved into the electrons.  mode 0: reference energy (step -1);
// mode 1: main-loop step (renormalise when (step+1) % interval == 0).

__global__ void __launch_bounds__(256) k_energy_partials(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0, b = 0, c = 0, d = 0;
    if (i < D.natom) { a = D.pe[i]; b = D.ke[i]; c = D.me[i]; d = D.me0[i]; }
    __shared__ double sh[32];
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    d = block_sum(d, sh);
    if (threadIdx.x == 0) {
        double* o = D.red + 4 * (size_t)blockIdx.x;
        o[0] = a; o[1] = b; o[2] = c; o[3] = d;
    }
}

__global__ void __launch_bounds__(1024) k_renorm(Dev D, int nb, int mode) {
    __shared__ double sh[32];
    __shared__ double err_s;
    long long cur = D.ctl->steps;
    bool act = mode == 0 || ((cur + 1) % D.print_every == 0);
    if (!act) return;
    double a = 0, b = 0, c = 0, d = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a += D.red[4 * k]; b += D.red[4 * k + 1]; c += D.red[4 * k + 2]; d += D.red[4 * k + 3];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    d = block_sum(d, sh);
    double per = (double)D.natom / (double)D.nte;
    double e = 0.0;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = te_to_Ee(D.Te[k]);
        D.Ee[k] = Ee;
        e += per * Ee;
    }
    e = block_sum(e, sh);
    if (threadIdx.x == 0) {
        double n = (double)D.natom;
        double pe = a / n, ke = b / n, me = c / n, me0 = d / n, Ee = e / n;
        double err = 0.0;
        if (mode == 0) {
            double t = 0.0;
            t += pe; t += ke; t += me; t += me0; t += Ee;
            D.ctl->initial_ave_energy = t;
        } else {
            double t = 0.0;
            t += pe; t += ke; t += me; t += me0; t += Ee;
            err = t - D.ctl->initial_ave_energy;
        }
        err_s = err;
    }
    __syncthreads();
    double err = err_s;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        double Ee = D.Ee[k] - err;
        D.Ee[k] = Ee;
        D.Te[k] = Ee_to_te(Ee);
    }
}

void launch_energy_check(const Dev& D, cudaStream_t st, int mode) {
    int nb = div_up(D.natom, 256);
    k_energy_partials<<<nb, 256, 0, st>>>(D);
    k_renorm<<<1, 1024, 0, st>>>(D, nb, mode);
}

// ---------------------------------------------------------------------
// bookkeeping and read-outs

__global__ void k_advance(Dev D, int epochs, int steps) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        D.ctl->epoch += (unsigned long long)epochs;
        for (int k = 0; k < steps; ++k) D.ctl->total_time += D.step;
        D.ctl->steps += steps;
    }
}

void launch_advance(const Dev& D, cudaStream_t st, int epochs, int steps) {
    k_advance<<<1, 32, 0, st>>>(D, epochs, steps);
}

__global__ void __launch_bounds__(256) k_avg_partials(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < D.natom) {
        v[0] = D.pe[i]; v[1] = D.ke[i]; v[2] = D.me[i]; v[3] = D.me0[i];
        double4 s = D.s[i];
        v[4] = s.x; v[5] = s.y; v[6] = s.z;
    }
    __shared__ double sh[32];
    for (int k = 0; k < 7; ++k) {
        double t = block_sum(v[k], sh);
        if (threadIdx.x == 0) D.red[8 * (size_t)blockIdx.x + k] = t;
    }
}

__global__ void __launch_bounds__(1024) k_avg_final(Dev D, int nb, double* out) {
    __shared__ double sh[32];
    double v[7];
    for (int k = 0; k < 7; ++k) {
        double a = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) a += D.red[8 * b + k];
        v[k] = block_sum(a, sh);
    }
    double e = 0, t = 0;
    if (D.eltemp) {
        double per = (double)D.natom / (double)D.nte;
        for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
            e += per * te_to_Ee(D.Te[k]);
            t += D.Te[k];
        }
    }
    e = block_sum(e, sh);
    t = block_sum(t, sh);
    if (threadIdx.x == 0) {
        double n = (double)D.natom;
        out[0] = v[0] / n; out[1] = v[1] / n; out[2] = v[2] / n; out[3] = v[3] / n;
        out[4] = D.eltemp ? e / n : 0.0;
        out[5] = v[1] * 2.0 / 3.0 / n / SLD_BOLTZ;
        out[6] = D.eltemp ? t / D.nte / SLD_BOLTZ : 0.0;
        out[7] = v[4] / n; out[8] = v[5] / n; out[9] = v[6] / n;
    }
}

void launch_averages(const Dev& D, cudaStream_t st, double* out_dev) {
    int nb = div_up(D.natom, 256);
    k_avg_partials<<<nb, 256, 0, st>>>(D);
    k_avg_final<<<1, 1024, 0, st>>>(D, nb, out_dev);
}

__global__ void __launch_bounds__(256) k_vir_partials(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = i < D.natom ? D.vir[i] : 0.0;
    __shared__ double sh[32];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) D.red[4 * (size_t)blockIdx.x] = v;
}
__global__ void __launch_bounds__(1024) k_vir_final(Dev D, int nb) {
    __shared__ double sh[32];
    double a = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) a += D.red[4 * b];
    a = block_sum(a, sh);
    if (threadIdx.x == 0) D.ctl->virial = a;
}
void launch_virial(const Dev& D, cudaStream_t st) {
    int nb = div_up(D.natom, 256);
    k_vir_partials<<<nb, 256, 0, st>>>(D);
    k_vir_final<<<1, 1024, 0, st>>>(D, nb);
}
