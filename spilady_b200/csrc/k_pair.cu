// Pair passes, FP64 form: the per-step neighbour lists with the EAM density,
// and the force/energy pass.
//
// The reference finds pairs by walking link cells in every pass: a half
// shell with OpenMP atomics for rho and forces (calculate_rho_CPU.cpp:33-69,
// calculate_force_energy_CPU.cpp:33-216) and the full shell for each of the
// spin-field evaluations (calculate_spin_CPU.cpp:201-274).  Positions change
// only in core_dr, so here one pass after each drift (k_pairs) walks the 26
// neighbour cells and the own cell in the reference's order, computes rho,
// and records every pair within rcut_max (nbr) and every exchange pair
// within rcut_mag with its J(r_ij) (jl/jv); the force pass, the spin sweeps
// and calculate_temperature then read those lists.  Each thread owns one
// atom and gathers its full shell, so there are no atomics.  The minimum
// image is applied with the reference's arithmetic (find_image) and only to
// pairs whose cells are neighbours across the periodic boundary; for all
// other pairs the reference's find_image leaves the vector unchanged.
#include "sld_common.cuh"

__global__ void __launch_bounds__(128) k_pairs(Dev D, int write_rho) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned* err = &D.ctl->err;
    const int N = D.natom;
    double4 ri = D.r[i];
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    double rho = 0.0;
    int nn = 0, nj = 0;
    for (int k = 0; k < 27; ++k) {
        bool wrap = false;
        int c = k == 26 ? c0 : nbr_cell_w(D, cx, cy, cz, k, wrap);
        int st = D.cell_start[c], n = D.cell_count[c];
        for (int m = 0; m < n; ++m) {
            int j = D.cell_atoms[st + m];
            if (j == i) continue;
            double4 rj = D.r[j];
            double3 d = make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z);
            if (wrap) d = find_image(D, d);
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            if (rsq >= D.rcut_max_sq) continue;
            if (nn < SLD_MAXNB) D.nbr[(size_t)nn * N + i] = j | (wrap ? SLD_WRAP : 0);
            ++nn;
            double r0 = sqrt(rsq);
            if (r0 < D.rcut_pot) rho += interp(D.tf, r0, D.inv_r, err);
            if (rsq < D.rcut_mag_sq) {
                if (nj < SLD_MAXJ) {
                    D.jl[(size_t)nj * N + i] = j;
                    D.jv[(size_t)nj * N + i] = interp(D.tJ, r0, D.inv_r, err);
                }
                ++nj;
            }
        }
    }
    if (nn > SLD_MAXNB || nj > SLD_MAXJ) atomicOr(err, SLD_FLAG_CAPACITY);
    D.nbr_n[i] = nn < SLD_MAXNB ? nn : SLD_MAXNB;
    D.jl_n[i] = nj < SLD_MAXJ ? nj : SLD_MAXJ;
    if (write_rho) D.rho[i] = rho;
}

__global__ void __launch_bounds__(128) k_force(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    unsigned* err = &D.ctl->err;
    const int N = D.natom;
    double4 ri = D.r[i];
    double4 si = D.s[i];
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    double rho_i = D.rho[i];
    double dF_i = interp(D.tdF, rho_i, D.inv_rho, err);
    double fx = 0, fy = 0, fz = 0, pe = 0, me = 0, me0 = 0, vir = 0;
    double s11 = 0, s22 = 0, s33 = 0, s12 = 0, s23 = 0, s31 = 0;
    int nn = D.nbr_n[i];
    for (int e = 0; e < nn; ++e) {
        int pk = D.nbr[(size_t)e * N + i];
        int j = pk & SLD_JMASK;
        double4 rj = D.r[j];
        double3 d = make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z);
        if (pk & SLD_WRAP) d = find_image(D, d);
        double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
        double r0 = sqrt(rsq);
        double dudr = 0.0, dudr_spin = 0.0;
        if (r0 < D.rcut_pot) {
            double df = interp(D.tdf, r0, D.inv_r, err);
            double dF_j = interp(D.tdF, D.rho[j], D.inv_rho, err);
            dudr = (dF_i + dF_j) * df + interp(D.tdphi, r0, D.inv_r, err);
            // the Landau tables are rho-independent: their derivative
            // tables are zero and add nothing to dudr
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
    double* out = D.stress + 6 * (size_t)i;
    out[0] = ((p.x * p.x) / m + s11 / 2.0) / V;
    out[1] = ((p.y * p.y) / m + s22 / 2.0) / V;
    out[2] = ((p.z * p.z) / m + s33 / 2.0) / V;
    out[3] = ((p.x * p.y) / m + s12 / 2.0) / V;
    out[4] = ((p.y * p.z) / m + s23 / 2.0) / V;
    out[5] = ((p.z * p.x) / m + s31 / 2.0) / V;
    if (!isfinite(fx + fy + fz + pe + me)) atomicOr(err, SLD_FLAG_NAN);
}

void launch_pairs(const Dev& D, cudaStream_t st, bool write_rho) {
    k_pairs<<<div_up(D.natom, 128), 128, 0, st>>>(D, write_rho ? 1 : 0);
}
void launch_force(const Dev& D, cudaStream_t st) {
    k_force<<<div_up(D.natom, 128), 128, 0, st>>>(D);
}
