// Spin effective field and the Suzuki-Trotter colour sweeps, FP64 form.
//
// core_ds (core_ds_CPU.cpp:35-83) visits every atom twice: colour groups
// 0..G-1 with each cell walked head -> tail, then groups G-1..0 walked
// tail -> head.  Cells of one colour share no neighbour, so one launch per
// (group, direction) updates all cells of the group at once, one thread per
// cell, each walking its list in the reference's order (the in-cell update
// is Gauss-Seidel: a later atom sees the spins already rotated before it).
//
// A visit (calculate_spin_CPU.cpp:33-199) gathers Heff_H = sum_j J(r_ij) s_j
// over the 26 neighbour cells and the own cell in the reference's order
// (inner_spin, :201-235); with the Langevin thermostat it also gathers
// sum_j J(r_ij) |s_j| (inner_sum_Jij_sj, :238-274) in the same pass, since
// no neighbour spin changes between the two sums.  NVE visits apply the
// exact rotation (core_ds_CPU.cpp:90-127); Langevin visits apply the
// reference's five-part scheme with counter-based normal noise.
#include "sld_common.cuh"

__device__ __forceinline__ double3 spin_rotation(double3 H, double3 s, double dt) {
    double3 w = make_double3(H.x / -SLD_HBAR, H.y / -SLD_HBAR, H.z / -SLD_HBAR);
    double w0 = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
    if (w0 > 0.0) w = make_double3(w.x / w0, w.y / w0, w.z / w0);
    else w = make_double3(0.0, 0.0, 0.0);
    double w12 = w.x * w.y, w23 = w.y * w.z, w13 = w.x * w.z;
    double w1s = w.x * w.x, w2s = w.y * w.y, w3s = w.z * w.z;
    double A, cw;
    sincos(w0 * dt, &A, &cw);
    double B = 1.0 - cw;
    double3 o;
    o.x = s.x + (s.x * B * (-w2s - w3s) + s.y * (B * w12 - A * w.z) + s.z * (A * w.y + B * w13));
    o.y = s.y + (s.y * B * (-w1s - w3s) + s.z * (B * w23 - A * w.x) + s.x * (A * w.z + B * w12));
    o.z = s.z + (s.z * B * (-w1s - w2s) + s.x * (B * w13 - A * w.y) + s.y * (A * w.x + B * w23));
    return o;
}

// Landau field plus the exchange correction (calculate_spin_CPU.cpp:127-136)
__device__ __forceinline__ double3 landau_field(const double L[4], double sumJ, double3 x) {
    double s_sq = x.x * x.x + x.y * x.y + x.z * x.z;
    double c = -(2.0 * L[0] + 4.0 * L[1] * s_sq + 6.0 * L[2] * (s_sq * s_sq) +
                 8.0 * L[3] * pow(s_sq, 3.0));
    double3 HL = make_double3(c * x.x, c * x.y, c * x.z);
    double s0 = sqrt(s_sq);
    if (s0 > 0.0) {
        double k = -sumJ / s0;
        HL.x += k * x.x; HL.y += k * x.y; HL.z += k * x.z;
    }
    return HL;
}

__device__ __forceinline__ void cell_xyz(const Dev& D, int c, int& cx, int& cy, int& cz) {
    cx = c % D.nx;
    int t = c / D.nx;
    cy = t % D.ny;
    cz = t / D.ny;
}

// Heff_H and (optionally) sum_j J |s_j| for atom i
__device__ __forceinline__ void gather_field(const Dev& D, int i, double4 ri, int c0, bool want_sumJ,
                                             double3& H, double& sumJ, unsigned* err) {
    int cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    H = make_double3(0.0, 0.0, 0.0);
    sumJ = 0.0;
    for (int k = 0; k < 27; ++k) {
        int c = k == 26 ? c0 : nbr_cell(D, cx, cy, cz, k);
        int st = D.cell_start[c], n = D.cell_count[c];
        for (int m = 0; m < n; ++m) {
            int j = D.cell_atoms[st + m];
            if (j == i) continue;
            double4 rj = D.r[j];
            double3 d = find_image(D, make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z));
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            if (rsq < D.rcut_mag_sq) {
                double J = interp(D.tJ, sqrt(rsq), D.inv_r, err);
                double4 sj = D.s[j];
                H.x += J * sj.x; H.y += J * sj.y; H.z += J * sj.z;
                if (want_sumJ) sumJ += J * sj.w;
            }
        }
    }
}

__device__ void spin_visit(const Dev& D, int i, double dt, unsigned long long epoch) {
    unsigned* err = &D.ctl->err;
    double4 ri = D.r[i];
    double4 s4 = D.s[i];
    double3 s = make_double3(s4.x, s4.y, s4.z);
    double3 H;
    double sumJ;
    gather_field(D, i, ri, D.cell_of[i], D.spinlang != 0, H, sumJ, err);
    double3 HL = make_double3(0.0, 0.0, 0.0);
    if (!D.spinlang) {
        s = spin_rotation(H, s, dt);
    } else {
        double dt_half = dt / 2.0, dt_quad = dt / 4.0, g = D.gamma_S_HL;
        double rho = D.rho[i];
        double L[4];
        for (int k = 0; k < 4; ++k) L[k] = interp_const(D.landau[k], rho, D.inv_rho);
        s = spin_rotation(H, s, dt_half);                                   // part 1
        HL = landau_field(L, sumJ, s);                                      // part 2
        double a = g * dt_quad;
        double3 t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
        HL = landau_field(L, sumJ, t);
        a = g * dt_half;
        s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
        double T = D.eltemp ? D.Te[D.node[i]] : D.temperature;              // part 3
        double amp = sqrt(2.0 * T * g / dt);
        double3 xi = normals3(D.seed, 0u, (unsigned)D.id[i], epoch);
        double3 dS = make_double3(amp * xi.x, amp * xi.y, amp * xi.z);
        s = make_double3(s.x + dt * dS.x, s.y + dt * dS.y, s.z + dt * dS.z);
        HL = landau_field(L, sumJ, s);                                      // part 4
        a = g * dt_quad;
        t = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
        HL = landau_field(L, sumJ, t);
        a = g * dt_half;
        s = make_double3(s.x + a * (H.x + HL.x), s.y + a * (H.y + HL.y), s.z + a * (H.z + HL.z));
        s = spin_rotation(H, s, dt_half);                                   // part 5
        D.sumJ[i] = sumJ;
    }
    double s0 = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
    if (!isfinite(s0)) atomicOr(err, SLD_FLAG_NAN);
    D.s[i] = make_double4(s.x, s.y, s.z, s0);
    D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
    D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
}

__global__ void __launch_bounds__(128) k_sweep64(Dev D, const int* __restrict__ gcells, int ncell_g,
                                                 double dt, int backward, int epoch_off) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell_g) return;
    int c = gcells[t];
    int st = D.cell_start[c], n = D.cell_count[c];
    unsigned long long epoch = D.ctl->epoch + (unsigned long long)epoch_off;
    if (!backward) {
        for (int m = 0; m < n; ++m) spin_visit(D, D.cell_atoms[st + m], dt, epoch);
    } else {
        for (int m = n - 1; m >= 0; --m) spin_visit(D, D.cell_atoms[st + m], dt, epoch);
    }
}

void launch_sweep64(const Dev& D, cudaStream_t st, const int* gcells, int ncell_g, double dt,
                    bool backward, int epoch_off) {
    if (ncell_g <= 0) return;
    k_sweep64<<<div_up(ncell_g, 128), 128, 0, st>>>(D, gcells, ncell_g, dt, backward ? 1 : 0,
                                                    epoch_off);
}
