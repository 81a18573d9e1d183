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
#include "sld_common.cuh"

// Heff_H and sum_j J |s_j| (inner_spin / inner_sum_Jij_sj) from the
// exchange list
__device__ __forceinline__ void gather_field_t(const Dev& D, int i, double3& H, double& sumJ) {
    const int N = D.natom;
    H = make_double3(0.0, 0.0, 0.0);
    sumJ = 0.0;
    int nj = D.jl_n[i];
    for (int e = 0; e < nj; ++e) {
        int j = D.jl[(size_t)e * N + i];
        double J = D.jv[(size_t)e * N + i];
        double4 sj = D.s[j];
        H.x += J * sj.x; H.y += J * sj.y; H.z += J * sj.z;
        sumJ += J * sj.w;
    }
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
    double c = -(2.0 * A + 4.0 * B * s_sq + 6.0 * C * (s_sq * s_sq) + 8.0 * Dd * pow(s_sq, 3.0));
    double k = -sumJ / s0;
    double3 HL = make_double3(c * s.x + k * s.x, c * s.y + k * s.y, c * s.z + k * s.z);
    double hx = H.x + HL.x, hy = H.y + HL.y, hz = H.z + HL.z;
    Lup = hx * hx + hy * hy + hz * hz;
    Ldn = 6.0 * A + 20.0 * B * s_sq + 42.0 * C * (s_sq * s_sq) + 72.0 * Dd * pow(s_sq, 3.0);
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
    double* acc = D.acc + 9 * (size_t)D.node[i];
    atomicAdd(acc + 0, D.ke[i]);
    atomicAdd(acc + 1, p.x);
    atomicAdd(acc + 2, p.y);
    atomicAdd(acc + 3, p.z);
    atomicAdd(acc + 4, a);
    atomicAdd(acc + 5, b);
    atomicAdd(acc + 6, e);
    atomicAdd(acc + 7, f);
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

void launch_dte(const Dev& D, cudaStream_t st, double dt) {
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
