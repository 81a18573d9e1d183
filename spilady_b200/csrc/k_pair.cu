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
#include <algorithm>
#include <cstdlib>

#include "sld_pot32.cuh"

// pair vector (FP64, minimum image with the reference's arithmetic)
__device__ __forceinline__ double3 pair_d(const Dev& D, double4 ri, int pk) {
    double4 rj = D.r[pk & SLD_JMASK];
    double3 d = make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z);
    if (pk & SLD_WRAP) d = find_image(D, d);
    return d;
}

// MODE 0: FP64 tables (the reference's arithmetic); 1: split form (FP32
// analytic); 2: the analytic forms in FP64.
//
// Two passes per atom.  The first walks the 27 cells with a loose cutoff
// test in FP32 on the cell-ordered FP32 positions (one contiguous 16-byte
// load and a few FP32 operations per candidate; a neighbour cell across the
// box is shifted by its box vector), writing the slots that pass to the
// atom's list in traversal order.  The second walks that list, applies the
// reference's exact test (FP64 pair vector with find_image), compacts the
// list in place to the atom indices that pass, and does the per-pair work
// (density, exchange list).  The lists and sums are those of one exact pass.
// In one pass, some lane of a warp accepts almost every candidate (about 26
// of 162 pass), so the per-pair body would run, divergent, for nearly every
// candidate of every lane.
//
// The loose test keeps every pair the exact one keeps: with coordinates
// below B in magnitude, each FP32 rounding moves a coordinate by at most
// e = ulp(B)/2; a pair-vector component collects four of them (two
// positions, the box shift, the difference), so r^2 near the cutoff moves by
// at most 2 r_max (4 sqrt(3) e) + (4 sqrt(3) e)^2 plus the FP32 rounding of
// the sum.  D.pair_loose, set on the host from the box, is twice that.

template <int MODE>
__device__ __forceinline__ bool pair_accept(const Dev& D, double3 d) {
    if constexpr (MODE == 1) {
        float dx = (float)d.x, dy = (float)d.y, dz = (float)d.z;
        return dx * dx + dy * dy + dz * dz < (float)D.rcut_max_sq;
    } else {
        return d.x * d.x + d.y * d.y + d.z * d.z < D.rcut_max_sq;
    }
}

template <int MODE>
__device__ void pairs_one(const Dev& D, int i, int write_rho) {
    constexpr bool SPLIT = MODE == 1;
    unsigned* err = &D.ctl->err;
    const int N = D.natom;
    const double4 ri = D.r[i];
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    // pass 1: loose cutoff test in the reference's traversal order
    int nn = 0;
    const int myslot = D.cell_slot[i];
    auto keep = [&](int slot, bool wrap) {
        if (nn < SLD_MAXNB) D.nbr[(size_t)nn * N + i] = slot | (wrap ? SLD_WRAP : 0);
        ++nn;
    };
    if (!D.small_grid) {
        const float rx = (float)ri.x, ry = (float)ri.y, rz = (float)ri.z;
        const float cut = (float)D.rcut_max_sq + D.pair_loose;
        const float ax = (float)D.d[0];
        const float bx = (float)D.d[1], by = (float)D.d[2];
        const float qx = (float)D.d[3], qy = (float)D.d[4], qz = (float)D.d[5];
        for (int k = 0; k < 27; ++k) {
            int sx = 0, sy = 0, sz = 0;
            const int c = k == 26 ? c0 : nbr_cell_s(D, cx, cy, cz, k, sx, sy, sz);
            const bool wrap = (sx | sy | sz) != 0;
            // this atom seen from the neighbour cell's image (its atoms
            // + sx a + sy b + sz c)
            const float ex = rx - (sx * ax + sy * bx + sz * qx);
            const float ey = ry - (sy * by + sz * qy);
            const float ez = rz - sz * qz;
            const int st = __ldg(D.cell_start + c), n = min(__ldg(D.cell_count + c), SLD_MAXC);
            for (int m0 = 0; m0 < n; m0 += 4) {
                float4 q[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    q[u] = m0 + u < n ? __ldg(D.r32s + st + m0 + u) : make_float4(1e30f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int slot = st + m0 + u;
                    const float dx = ex - q[u].x, dy = ey - q[u].y, dz = ez - q[u].z;
                    if (dx * dx + dy * dy + dz * dz < cut && slot != myslot) keep(slot, wrap);
                }
            }
        }
    } else {
        // three cells along an axis: the image is the reference's minimum
        // image of each pair
        for (int k = 0; k < 27; ++k) {
            bool wrap = false;
            const int c = k == 26 ? c0 : nbr_cell_w(D, cx, cy, cz, k, wrap);
            const int st = D.cell_start[c], n = cell_n(D, c);
            for (int m = 0; m < n; ++m) {
                const int slot = st + m;
                if (slot == myslot) continue;
                const double4 rj = D.r[D.cell_atoms[slot]];
                if (pair_accept<MODE>(
                        D, find_image(D, make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z))))
                    keep(slot, true);
            }
        }
    }
    const int nl = nn < SLD_MAXNB ? nn : SLD_MAXNB;
    // pass 2: density and exchange list over the accepted pairs
    double rho = 0.0;
    Kahan rho32;
    const float rmag2f = (float)D.rcut_mag_sq;
    const float rpotf = (float)D.rcut_pot;
    int nj = 0, w = 0;
    for (int e = 0; e < nl; ++e) {
        const int ps = D.nbr[(size_t)e * N + i];
        const int j = D.cell_atoms[ps & SLD_JMASK];
        const int pk = j | (ps & SLD_WRAP);
        double3 d = pair_d(D, ri, pk);
        if (!pair_accept<MODE>(D, d)) continue;
        D.nbr[(size_t)w * N + i] = pk;
        ++w;
        if constexpr (!SPLIT) {
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            double r0 = sqrt(rsq);
            if (r0 < D.rcut_pot) {
                if constexpr (MODE == 0) {
                    rho += interp(D.tf, r0, D.inv_r, err);
                } else {
                    double f, df;
                    dens64(D, r0, f, df);
                    rho += f;
                }
            }
            if (rsq < D.rcut_mag_sq) {
                if (nj < SLD_MAXJ) {
                    D.jl[(size_t)i * SLD_MAXJ + nj] = j;
                    double J, dJ;
                    if constexpr (MODE == 0) J = interp(D.tJ, r0, D.inv_r, err);
                    else exch64(r0, J, dJ);
                    D.jv[(size_t)i * SLD_MAXJ + nj] = J;
                }
                ++nj;
            }
        } else {
            float dx = (float)d.x, dy = (float)d.y, dz = (float)d.z;
            float rsq = dx * dx + dy * dy + dz * dz;
            double r64 = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
            float f, df;
            if ((float)r64 < rpotf) {
                dens32r(D, r64, f, df);
                rho32.add(f);
            }
            if (rsq < rmag2f) {
                if (nj < SLD_MAXJ) {
                    float J, dJ;
                    exch32r(r64, J, dJ);
                    D.jl[(size_t)i * SLD_MAXJ + nj] = j;
                    D.jvf[(size_t)i * SLD_MAXJ + nj] = J;
                }
                ++nj;
            }
        }
    }
    if (nn > SLD_MAXNB || nj > SLD_MAXJ) atomicOr(err, SLD_FLAG_CAPACITY);
    D.nbr_n[i] = w;
    D.jl_n[i] = nj < SLD_MAXJ ? nj : SLD_MAXJ;
    if (write_rho) D.rho[i] = SPLIT ? rho32.value() : rho;
}

template <int MODE>
__global__ void __launch_bounds__(128) k_pairs(Dev D, int write_rho) {
    // one atom per thread; a capped grid walks several atoms per thread
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x)
        pairs_one<MODE>(D, i, write_rho);
}

// F'(rho) per atom (the force pass needs it for both atoms of every pair):
// from the reference's FP64 tables (FP64 and split forms), or the analytic
// derivative (FP64_ANALYTIC)
template <int MODE>
__global__ void __launch_bounds__(256) k_embed(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    if constexpr (MODE == 2) {
        double F, dF;
        emb64(D.rho[i], F, dF);
        D.dF[i] = dF;
    } else {
        D.dF[i] = interp(D.tdF, D.rho[i], D.inv_rho, &D.ctl->err);
    }
}

// Parts of the force pass.  The lattice (EAM) terms do not depend on the
// spins, the magnetic ones do; the step runs the EAM part beside the spin
// sweeps and adds the magnetic part after them (the sum is the reference's
// dudr = dudr_EAM + dudr_spin per pair, added in two passes).
enum { PART_ALL = 3, PART_EAM = 1, PART_MAG = 2 };

// on-site terms and outputs
template <int PART>
__device__ __forceinline__ void force_finish(const Dev& D, int i, double si_sq, double rho_i,
                                             double F_i, double fx, double fy, double fz, double pe,
                                             double me, double me0, double vir, const double st6[6]) {
    double m = D.atmass, V = D.box_volume / D.natom;
    double* out = D.stress + 6 * (size_t)i;
    if (PART & PART_EAM) {
        pe += F_i;
        D.pe[i] = pe;
    }
    if (PART & PART_MAG) {
        if (D.hext) {   // calculate_force_energy_CPU.cpp:200-202
            double4 s = D.s[i], h = D.hext[i];
            me -= s.x * h.x + s.y * h.y + s.z * h.z;
        }
        if (D.landau_on) {   // the Heisenberg-Landau Hamiltonians
            double A = interp_const(D.landau[0], rho_i, D.inv_rho);
            double B = interp_const(D.landau[1], rho_i, D.inv_rho);
            double C = interp_const(D.landau[2], rho_i, D.inv_rho);
            double Dd = interp_const(D.landau[3], rho_i, D.inv_rho);
            double s4 = si_sq * si_sq;
            me += A * si_sq + B * s4 + C * (s4 * si_sq) + Dd * (s4 * s4);
        }
        D.me[i] = me;
        D.me0[i] = me0;
    }
    if (PART == PART_MAG) {
        // add to what the EAM part wrote
        double4 f = D.f[i];
        D.f[i] = make_double4(f.x + fx, f.y + fy, f.z + fz, 0.0);
        D.vir[i] += 0.5 * vir;
        for (int k = 0; k < 6; ++k) out[k] += st6[k] / 2.0 / V;
        if (!isfinite(fx + fy + fz + me)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
        return;
    }
    D.f[i] = make_double4(fx, fy, fz, 0.0);
    D.vir[i] = 0.5 * vir;   // each pair's virial split evenly between its atoms
    // calculate_force_energy_CPU.cpp:262-296: local volume V/N, kinetic part
    double4 p = D.p[i];
    out[0] = ((p.x * p.x) / m + st6[0] / 2.0) / V;
    out[1] = ((p.y * p.y) / m + st6[1] / 2.0) / V;
    out[2] = ((p.z * p.z) / m + st6[2] / 2.0) / V;
    out[3] = ((p.x * p.y) / m + st6[3] / 2.0) / V;
    out[4] = ((p.y * p.z) / m + st6[4] / 2.0) / V;
    out[5] = ((p.z * p.x) / m + st6[5] / 2.0) / V;
    if (!isfinite(fx + fy + fz + pe)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
}

// FP64 force pass; AN: the analytic forms instead of the tables
template <bool AN, int PART>
__device__ __forceinline__ void force64_one(const Dev& D, int i) {
    unsigned* err = &D.ctl->err;
    const int N = D.natom;
    double4 ri = D.r[i];
    // the EAM part runs beside the spin sweeps and must not read the spins
    double4 si = (PART & PART_MAG) ? D.s[i] : make_double4(0, 0, 0, 0);
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    double rho_i = D.rho[i];
    double dF_i = (PART & PART_EAM) ? D.dF[i] : 0.0;
    double fx = 0, fy = 0, fz = 0, pe = 0, me = 0, me0 = 0, vir = 0;
    double st6[6] = {0, 0, 0, 0, 0, 0};
    int nn = D.nbr_n[i];
    for (int e0 = 0; e0 < nn; e0 += 4) {
      int pkb[4];
      double4 rjb[4];
      double dFb[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) pkb[u] = e0 + u < nn ? D.nbr[(size_t)(e0 + u) * N + i] : -1;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
          int j = pkb[u] & SLD_JMASK;
          rjb[u] = pkb[u] >= 0 ? D.r[j] : ri;
          dFb[u] = (pkb[u] >= 0 && (PART & PART_EAM)) ? D.dF[j] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int pk = pkb[u];
        if (pk < 0) continue;
        int j = pk & SLD_JMASK;
        double3 d = make_double3(ri.x - rjb[u].x, ri.y - rjb[u].y, ri.z - rjb[u].z);
        if (pk & SLD_WRAP) d = find_image(D, d);
        double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
        double r0 = sqrt(rsq);
        double dudr = 0.0, dudr_spin = 0.0;
        if ((PART & PART_EAM) && r0 < D.rcut_pot) {
            double df, dphi, phi;
            if constexpr (AN) {
                double f;
                dens64(D, r0, f, df);
                pair64(D, r0, phi, dphi);
            } else {
                df = interp(D.tdf, r0, D.inv_r, err);
                dphi = interp(D.tdphi, r0, D.inv_r, err);
                phi = interp(D.tphi, r0, D.inv_r, err);
            }
            dudr = (dF_i + dFb[u]) * df + dphi;
            // the Landau tables are rho-independent: their derivative
            // tables are zero and add nothing to dudr
            pe += 0.5 * phi;
        }
        if ((PART & PART_MAG) && r0 < D.rcut_mag) {
            double4 sj = D.s[j];
            double sj_sq = sj.x * sj.x + sj.y * sj.y + sj.z * sj.z;
            double dot = si.x * sj.x + si.y * sj.y + si.z * sj.z;
            double times = sqrt(si_sq * sj_sq);
            double J, dJ;
            if constexpr (AN) {
                exch64(r0, J, dJ);
            } else {
                dJ = interp(D.tdJ, r0, D.inv_r, err);
                J = interp(D.tJ, r0, D.inv_r, err);
            }
            dudr_spin = -dJ * (dot - times);
            double Jh = J / 2.0;
            me0 += Jh * times;
            me += -Jh * dot;
        }
        dudr += dudr_spin;
        if (dudr == 0.0 && PART != PART_ALL) continue;
        double force = -dudr / r0;
        double gx = force * d.x, gy = force * d.y, gz = force * d.z;
        fx += gx; fy += gy; fz += gz;
        st6[0] += gx * d.x; st6[1] += gy * d.y; st6[2] += gz * d.z;
        st6[3] += gx * d.y; st6[4] += gy * d.z; st6[5] += gz * d.x;
        vir += -force * rsq;
      }
    }
    double F_i = 0.0;
    if (PART & PART_EAM) {
        if constexpr (AN) {
            double dF_unused;
            emb64(rho_i, F_i, dF_unused);
        } else {
            F_i = interp(D.tF, rho_i, D.inv_rho, err);
        }
    }
    force_finish<PART>(D, i, si_sq, rho_i, F_i, fx, fy, fz, pe, me, me0, vir, st6);
}

// split form: FP32 pair terms from the analytic potential, Kahan sums
template <bool AN, int PART>
__global__ void __launch_bounds__(128) k_force64(Dev D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x)
        force64_one<AN, PART>(D, i);
}

template <int PART>
__device__ __forceinline__ void force32_one(const Dev& D, int i) {
    const int N = D.natom;
    double4 ri = D.r[i];
    double4 si = (PART & PART_MAG) ? D.s[i] : make_double4(0, 0, 0, 0);
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    float sx = (float)si.x, sy = (float)si.y, sz = (float)si.z;
    float si_sqf = sx * sx + sy * sy + sz * sz;
    double rho_i = D.rho[i];
    float dF_i = (PART & PART_EAM) ? (float)D.dF[i] : 0.f;
    const float rpot = (float)D.rcut_pot, rmag = (float)D.rcut_mag;
    Kahan fx, fy, fz, pe, me, me0;
    float vir = 0.f, st6f[6] = {0, 0, 0, 0, 0, 0};
    int nn = D.nbr_n[i];
    for (int e = 0; e < nn; ++e) {
        int pk = D.nbr[(size_t)e * N + i];
        int j = pk & SLD_JMASK;
        double3 dd = pair_d(D, ri, pk);
        float dx = (float)dd.x, dy = (float)dd.y, dz = (float)dd.z;
        double r64 = sqrt(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z);
        float r0 = (float)r64, rsq = r0 * r0;
        float dudr = 0.f;
        if ((PART & PART_EAM) && r0 < rpot) {
            float f, df, phi, dphi;
            dens32r(D, r64, f, df);
            pair32r(D, r64, phi, dphi);
            dudr = (dF_i + (float)D.dF[j]) * df + dphi;
            pe.add(0.5f * phi);
        }
        if ((PART & PART_MAG) && r0 < rmag) {
            const float4 sj4 = D.s32[j];   // (float) of the spin
            float tx = sj4.x, ty = sj4.y, tz = sj4.z;
            float sj_sq = tx * tx + ty * ty + tz * tz;
            float dot = sx * tx + sy * ty + sz * tz;
            float times = sqrtf(si_sqf * sj_sq);
            float J, dJ;
            exch32r(r64, J, dJ);
            dudr += -dJ * (dot - times);
            float Jh = 0.5f * J;
            me0.add(Jh * times);
            me.add(-Jh * dot);
        }
        if (dudr == 0.f && PART != PART_ALL) continue;
        float force = -dudr / r0;
        float gx = force * dx, gy = force * dy, gz = force * dz;
        fx.add(gx); fy.add(gy); fz.add(gz);
        st6f[0] += gx * dx; st6f[1] += gy * dy; st6f[2] += gz * dz;
        st6f[3] += gx * dy; st6f[4] += gy * dz; st6f[5] += gz * dx;
        vir += -force * rsq;
    }
    double F = 0.0;
    if (PART & PART_EAM) F = interp(D.tF, rho_i, D.inv_rho, &D.ctl->err);
    double st6[6];
    for (int k = 0; k < 6; ++k) st6[k] = st6f[k];
    force_finish<PART>(D, i, si_sq, rho_i, F, fx.value(), fy.value(), fz.value(),
                       pe.value(), me.value(), me0.value(), (double)vir, st6);
}

template <int PART>
__global__ void __launch_bounds__(128) k_force32(Dev D) {
    // one atom per thread; a capped grid walks several atoms per thread
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x)
        force32_one<PART>(D, i);
}

// a cap on the CTAs per SM (0: none) for the kernels of the step graph's side
// branch, which run beside the spin sweeps: a capped grid leaves room for the
// sweep's next launch instead of filling every free slot
static int capped_grid(int nb, int cap) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            sms <= 0)
            sms = 148;
    }
    return cap > 0 ? std::min(nb, cap * sms) : nb;
}

template <int PART>
static void launch_force_part(const Dev& D, cudaStream_t st) {
    const int bs = D.tune.force_block > 0 ? D.tune.force_block : 128;
    int nb = div_up(D.natom, bs);
    if (PART == PART_EAM) nb = capped_grid(nb, D.tune.force_cap);
    if (D.split) k_force32<PART><<<nb, bs, 0, st>>>(D);
    else if (D.analytic) k_force64<true, PART><<<nb, bs, 0, st>>>(D);
    else k_force64<false, PART><<<nb, bs, 0, st>>>(D);
}

void launch_pairs(const Dev& D, cudaStream_t st, bool write_rho) {
    int w = write_rho ? 1 : 0;
    const int bs = D.tune.pair_block > 0 ? D.tune.pair_block : 128;
    int nb = capped_grid(div_up(D.natom, bs), D.tune.pair_cap);
    if (D.split) k_pairs<1><<<nb, bs, 0, st>>>(D, w);
    else if (D.analytic) k_pairs<2><<<nb, bs, 0, st>>>(D, w);
    else k_pairs<0><<<nb, bs, 0, st>>>(D, w);
}
void launch_embed(const Dev& D, cudaStream_t st) {
    int nb = div_up(D.natom, 256);
    if (D.split) k_embed<1><<<nb, 256, 0, st>>>(D);
    else if (D.analytic) k_embed<2><<<nb, 256, 0, st>>>(D);
    else k_embed<0><<<nb, 256, 0, st>>>(D);
}
// all terms of the Hamiltonian: MD has no spins
void launch_force(const Dev& D, cudaStream_t st) {
    launch_embed(D, st);
    if (D.spin)
        launch_force_part<PART_ALL>(D, st);
    else
        launch_force_part<PART_EAM>(D, st);
}
void launch_force_eam(const Dev& D, cudaStream_t st) {
    launch_embed(D, st);
    launch_force_part<PART_EAM>(D, st);
}
void launch_force_mag(const Dev& D, cudaStream_t st) { launch_force_part<PART_MAG>(D, st); }
