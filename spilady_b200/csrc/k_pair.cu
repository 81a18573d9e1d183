// EAM density and force/energy passes, FP64 form.
//
// The reference walks a half shell (13 neighbour cells plus the head of the
// own list) and scatters every pair into both atoms with OpenMP atomics
// (calculate_rho_CPU.cpp:33-69, calculate_force_energy_CPU.cpp:33-216).  On
// the GPU each thread owns one atom and gathers its full shell (26 cells in
// the reference's neighbour order, then its own cell), so there are no
// atomics and every per-atom sum is formed by one thread.  Each pair term is
// the reference's, evaluated from the same interpolated tables; only the
// order of the additions differs.
#include "sld_common.cuh"

__device__ __forceinline__ void cell_xyz(const Dev& D, int c, int& cx, int& cy, int& cz) {
    cx = c % D.nx;
    int t = c / D.nx;
    cy = t % D.ny;
    cz = t / D.ny;
}

__global__ void __launch_bounds__(128) k_rho64(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned* err = &D.ctl->err;
    double4 ri = D.r[i];
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    double rho = 0.0;
    for (int k = 0; k < 27; ++k) {
        int c = k == 26 ? c0 : nbr_cell(D, cx, cy, cz, k);
        int st = D.cell_start[c], n = D.cell_count[c];
        for (int m = 0; m < n; ++m) {
            int j = D.cell_atoms[st + m];
            if (j == i) continue;
            double4 rj = D.r[j];
            double3 d = find_image(D, make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z));
            double r0 = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
            if (r0 < D.rcut_pot) rho += interp(D.tf, r0, D.inv_r, err);
        }
    }
    D.rho[i] = rho;
}

__global__ void __launch_bounds__(128) k_force64(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned* err = &D.ctl->err;
    double4 ri = D.r[i];
    double4 si = D.s[i];
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    double rho_i = D.rho[i];
    double dF_i = interp(D.tdF, rho_i, D.inv_rho, err);
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    double fx = 0, fy = 0, fz = 0, pe = 0, me = 0, me0 = 0, vir = 0;
    double s11 = 0, s22 = 0, s33 = 0, s12 = 0, s23 = 0, s31 = 0;
    for (int k = 0; k < 27; ++k) {
        int c = k == 26 ? c0 : nbr_cell(D, cx, cy, cz, k);
        int st = D.cell_start[c], n = D.cell_count[c];
        for (int m = 0; m < n; ++m) {
            int j = D.cell_atoms[st + m];
            if (j == i) continue;
            double4 rj = D.r[j];
            double3 d = find_image(D, make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z));
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            if (rsq >= D.rcut_max_sq) continue;
            double r0 = sqrt(rsq);
            double dudr = 0.0, dudr_spin = 0.0;
            if (r0 < D.rcut_pot) {
                double df = interp(D.tdf, r0, D.inv_r, err);
                double dF_j = interp(D.tdF, D.rho[j], D.inv_rho, err);
                dudr = (dF_i + dF_j) * df + interp(D.tdphi, r0, D.inv_r, err);
                // the Landau tables are rho-independent, so their
                // derivative tables are zero and add nothing here
                pe += 0.5 * interp(D.tphi, r0, D.inv_r, err);
            }
            if (r0 < D.rcut_mag) {
                double4 sj = D.s[j];
                double sj_sq = sj.x * sj.x + sj.y * sj.y + sj.z * sj.z;
                double dot = si.x * sj.x + si.y * sj.y + si.z * sj.z;
                double times = sqrt(si_sq * sj_sq);
                dudr_spin = -interp(D.tdJ, r0, D.inv_r, err) * (dot - times);
                double Jh = interp(D.tJ, r0, D.inv_r, err) / 2.0;
                me0 += Jh * times;
                me += -Jh * dot;
            }
            dudr += dudr_spin;
            double force = -dudr / r0;
            double gx = force * d.x, gy = force * d.y, gz = force * d.z;
            fx += gx; fy += gy; fz += gz;
            s11 += gx * d.x; s22 += gy * d.y; s33 += gz * d.z;
            s12 += gx * d.y; s23 += gy * d.z; s31 += gz * d.x;
            vir += -force * rsq;
        }
    }
    pe += interp(D.tF, rho_i, D.inv_rho, err);
    double A = interp_const(D.landau[0], rho_i, D.inv_rho);
    double B = interp_const(D.landau[1], rho_i, D.inv_rho);
    double C = interp_const(D.landau[2], rho_i, D.inv_rho);
    double Dd = interp_const(D.landau[3], rho_i, D.inv_rho);
    me += A * si_sq + B * (si_sq * si_sq) + C * pow(si_sq, 3.0) + Dd * pow(si_sq, 4.0);
    D.f[i] = make_double4(fx, fy, fz, 0.0);
    D.pe[i] = pe;
    D.me[i] = me;
    D.me0[i] = me0;
    D.vir[i] = 0.5 * vir;   // each pair's virial split evenly between its atoms
    // calculate_force_energy_CPU.cpp:262-296: local volume V/N, kinetic part
    double4 p = D.p[i];
    double m = D.atmass, V = D.box_volume / D.natom;
    double* st = D.stress + 6 * (size_t)i;
    st[0] = ((p.x * p.x) / m + s11 / 2.0) / V;
    st[1] = ((p.y * p.y) / m + s22 / 2.0) / V;
    st[2] = ((p.z * p.z) / m + s33 / 2.0) / V;
    st[3] = ((p.x * p.y) / m + s12 / 2.0) / V;
    st[4] = ((p.y * p.z) / m + s23 / 2.0) / V;
    st[5] = ((p.z * p.x) / m + s31 / 2.0) / V;
    if (!isfinite(fx + fy + fz + pe + me)) atomicOr(err, SLD_FLAG_NAN);
}

void launch_rho64(const Dev& D, cudaStream_t st) {
    k_rho64<<<div_up(D.natom, 128), 128, 0, st>>>(D);
}
void launch_force64(const Dev& D, cudaStream_t st) {
    k_force64<<<div_up(D.natom, 128), 128, 0, st>>>(D);
}
