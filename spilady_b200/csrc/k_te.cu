// Electron-temperature cells and the energy bookkeeping.
//
//   calculate_temperature  calculate_temperature_CPU.cpp:35-148
//   check_energy           check_energy_CPU.cpp:33-111 (renormalisation)
//   averages and virial    check_energy/check_temperature/check_spin
//
// Te cells are the link cells (as in the reference) or the nodes of a mesh
// decoupled from them.  core_dTe itself is in k_dte.cu.
#include <cstdlib>

#include "sld_pot32.cuh"

// Heff_H and sum_j J |s_j| (inner_spin / inner_sum_Jij_sj) from the
// exchange list
__device__ __forceinline__ void gather_field_t(const Dev& D, int i, double3& H, double& sumJ) {
    exchange_field(D, i, H, sumJ, [](int) { return false; }, [](int, double) {});
}

// per-atom terms of calculate_temperature; writes H, HL, sumJ and returns
// the four sums (R_up, R_dn, L_up, L_dn) it contributes
__device__ __forceinline__ void temp_atom(const Dev& D, int i, double& Rup, double& Rdn, double& Lup,
                                          double& Ldn) {
    Rup = Rdn = Lup = Ldn = 0.0;
    if (!D.spin) return;
    double3 H;
    double sumJ;
    gather_field_t(D, i, H, sumJ);
    temp_spin_terms(D, i, H, sumJ, Rup, Rdn, Lup, Ldn);
}

// per-Te-cell results from the sums (calculate_temperature_CPU.cpp:118-142)
__device__ __forceinline__ void temp_finish(const Dev& D, int k, double n, double sum_ke, double apx,
                                            double apy, double apz, double Rup, double Rdn, double Lup,
                                            double Ldn) {
    double per = (double)D.natom / (double)D.nte;
    if (!D.latt) {
    } else if (D.localcolmot) {
        apx = apx / n; apy = apy / n; apz = apz / n;
        sum_ke -= n * (apx * apx + apy * apy + apz * apz) / 2.0 / D.atmass;
        D.Tl[k] = 2.0 / 3.0 * sum_ke / (n - 1.0) / SLD_BOLTZ;
        D.Gel[k] = 3.0 * (n - 1.0) * SLD_BOLTZ * D.gamma_L / D.atmass / per;
    } else {
        D.Tl[k] = sum_ke * 2.0 / 3.0 / n / SLD_BOLTZ;
        D.Gel[k] = 3.0 * n * SLD_BOLTZ * D.gamma_L / D.atmass / per;
    }
    if (D.spin) D.TsR[k] = Rup / Rdn / 2.0 / SLD_BOLTZ;
    if (D.landau_on) {
        D.TsL[k] = Lup / Ldn / SLD_BOLTZ;
        D.Ges[k] = SLD_BOLTZ * D.gamma_S_HL * Ldn / per;
    } else if (D.spin) {
        // the Heisenberg Hamiltonians (calculate_temperature_CPU.cpp:128-131)
        D.Ges[k] = 2e0 * SLD_BOLTZ * D.gamma_S_H * Rdn / SLD_HBAR / per;
    }
    // the cell sums check_temperature adds up (check_temperature_CPU.cpp:49-55,86-92)
    double* q = D.trl + 4 * (size_t)k;
    q[0] = Rup; q[1] = Rdn; q[2] = Lup; q[3] = Ldn;
}

// Te on link cells: one thread per cell, atoms in list order (the
// reference's summation order)
__global__ void __launch_bounds__(128) k_temp_cell(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.ncells) return;
    int st = D.cell_start[c], n = cell_n(D, c);
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
    double v[8] = {D.ke[i], p.x, p.y, p.z, a, b, e, f};
    node_add<8>(D, D.node[i], v, 0);
}

__global__ void k_temp_node(Dev D) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nte) return;
    const double* a = D.acc + 9 * (size_t)k;
    temp_finish(D, k, (double)D.te_count[k], a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]);
}

void launch_temperature_begin(const Dev& D, cudaStream_t st) {
    cudaMemsetAsync(D.acc, 0, sizeof(double) * 9 * (size_t)D.nte, st);
}
void launch_temperature_end(const Dev& D, cudaStream_t st) {
    k_temp_node<<<div_up(D.nte, 128), 128, 0, st>>>(D);
}

void launch_temperature(const Dev& D, cudaStream_t st) {
    if (D.te_mesh > 0) {
        cudaMemsetAsync(D.acc, 0, sizeof(double) * 9 * (size_t)D.nte, st);
        const int bs = D.tune.temp_block > 0 ? D.tune.temp_block : 128;
        k_temp_atom<<<div_up(D.natom, bs), bs, 0, st>>>(D);
        k_temp_node<<<div_up(D.nte, 128), 128, 0, st>>>(D);
    } else {
        k_temp_cell<<<div_up(D.ncells, 128), 128, 0, st>>>(D);
    }
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
        // the terms of the Hamiltonian's energy (check_energy_CPU.cpp:86-108)
        double t = 0.0;
        if (D.latt) { t += pe; t += ke; }
        if (D.spin) { t += me; t += me0; }
        t += Ee;
        if (mode == 0)
            D.ctl->initial_ave_energy = t;
        else
            err = t - D.ctl->initial_ave_energy;
        err_s = err;
        // what check_energy prints for this step (check_energy_CPU.cpp:113-130)
        D.ctl->chk[0] = pe; D.ctl->chk[1] = ke; D.ctl->chk[2] = me; D.ctl->chk[3] = me0;
        D.ctl->chk[4] = Ee;
        D.ctl->chk_tag = mode == 0 ? 1 : cur + 2;
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

// ---------------------------------------------------------------------
// Sums behind the print-out lines of check() (check.cpp:31-47): per-atom
// energies (check_energy_CPU.cpp:35-60), spins (check_spin_CPU.cpp:35-50),
// virial and stresses (check_pressure_CPU.cpp:35-38,
// check_stress_CPU.cpp:35-50), and the spin-temperature sums
// (check_temperature_CPU.cpp:43-130).  Without eltemp the reference forms the
// latter from freshly computed fields, overwriting Heff_H, Heff_L and
// sum_Jij_sj of every atom; ATOM_TEMP does the same through temp_atom.  With
// eltemp it adds up the cell sums of the last calculate_temperature.
// Fixed-order block sums, so a check is bit-reproducible.

template <bool ATOM_TEMP>
__global__ void __launch_bounds__(256) k_check_partials(Dev D, double* part) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[SLD_CHK_ATOM];
#pragma unroll
    for (int k = 0; k < SLD_CHK_ATOM; ++k) v[k] = 0.0;
    if (i < D.natom) {
        v[SLD_CHK_PE] = D.pe[i]; v[SLD_CHK_KE] = D.ke[i];
        v[SLD_CHK_ME] = D.me[i]; v[SLD_CHK_ME0] = D.me0[i];
        double4 s = D.s[i];
        v[SLD_CHK_SX] = s.x; v[SLD_CHK_SY] = s.y; v[SLD_CHK_SZ] = s.z;
        v[SLD_CHK_VIR] = D.vir[i];
        const double* st = D.stress + 6 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[SLD_CHK_STRESS + k] = st[k];
        if (ATOM_TEMP)
            temp_atom(D, i, v[SLD_CHK_RUP], v[SLD_CHK_RDN], v[SLD_CHK_LUP], v[SLD_CHK_LDN]);
    }
    __shared__ double sh[32];
    for (int k = 0; k < SLD_CHK_ATOM; ++k) {
        double t = block_sum(v[k], sh);
        if (threadIdx.x == 0) part[SLD_CHK_ATOM * (size_t)blockIdx.x + k] = t;
    }
}

__global__ void __launch_bounds__(1024) k_check_final(Dev D, const double* part, int nb,
                                                      bool atom_temp, double* out) {
    __shared__ double sh[32];
    for (int k = 0; k < SLD_CHK_ATOM; ++k) {
        double a = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) a += part[SLD_CHK_ATOM * (size_t)b + k];
        a = block_sum(a, sh);
        if (threadIdx.x == 0) out[k] = a;
    }
    if (!D.eltemp) return;
    double per = (double)D.natom / (double)D.nte;
    double r[4] = {0, 0, 0, 0}, te = 0, ee = 0;
    for (int k = threadIdx.x; k < D.nte; k += blockDim.x) {
        const double* q = D.trl + 4 * (size_t)k;
        r[0] += q[0]; r[1] += q[1]; r[2] += q[2]; r[3] += q[3];
        double t = D.Te[k];
        te += t;
        ee += per * te_to_Ee(t);
    }
    for (int k = 0; k < 4; ++k) r[k] = block_sum(r[k], sh);
    te = block_sum(te, sh);
    ee = block_sum(ee, sh);
    if (threadIdx.x == 0) {
        if (!atom_temp)
            for (int k = 0; k < 4; ++k) out[SLD_CHK_RUP + k] = r[k];
        out[SLD_CHK_TE] = te;
        out[SLD_CHK_EE] = ee;
    }
}

// part: SLD_CHK_ATOM doubles per 256 atoms; out: SLD_CHK_N doubles
void launch_check_sums(const Dev& D, cudaStream_t st, double* part, double* out) {
    int nb = div_up(D.natom, 256);
    bool atom_temp = !D.eltemp;
    if (atom_temp)
        k_check_partials<true><<<nb, 256, 0, st>>>(D, part);
    else
        k_check_partials<false><<<nb, 256, 0, st>>>(D, part);
    k_check_final<<<1, 1024, 0, st>>>(D, part, nb, atom_temp, out);
}
