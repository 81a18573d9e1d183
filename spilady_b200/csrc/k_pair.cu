// Pair passes: the per-step neighbour lists with the EAM density, and the
// force/energy pass.
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
// atom and gathers its full shell, so there are no atomics.
//
// Candidates are tested on fixed-point positions relative to their link
// cell (fxs, cell_fix): the pair vector of an atom and a candidate in
// neighbour cell k is M (f_i - f_j - delta_k), exact in integers up to the
// products with the cell matrix, so a neighbour cell across the periodic
// boundary is its nearest image and the FP32 vector has one rounding per
// term, whatever the box.
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

// find_image_CPU.cpp:31-53 with a flag: true when it moved the vector
__device__ __forceinline__ double3 find_image_f(const Dev& D, double3 rij, bool& moved) {
    double3 q = to_frac(D, rij.x, rij.y, rij.z);
    int idx = 0;
    if (q.x < -0.5) { q.x += 1.0; ++idx; }
    if (q.x >= 0.5) { q.x -= 1.0; ++idx; }
    if (q.y < -0.5) { q.y += 1.0; ++idx; }
    if (q.y >= 0.5) { q.y -= 1.0; ++idx; }
    if (q.z < -0.5) { q.z += 1.0; ++idx; }
    if (q.z >= 0.5) { q.z -= 1.0; ++idx; }
    moved = idx != 0;
    return moved ? to_cart(D, q) : rij;
}

// ---------------------------------------------------------------------
// FP64 forms.  MODE 0: the reference's tables; 2: the analytic forms in
// FP64 with exact derivatives.
//
// Two passes per atom.  The first walks the 27 cells with a loose cutoff
// test in FP32 on the cell-relative positions (one contiguous 16-byte load
// and a few FP32 operations per candidate), writing the slots that pass to
// the atom's list in traversal order.  The second walks that list, applies
// the reference's exact test (FP64 pair vector of the positions with
// find_image, which the reference applies to every pair and which leaves a
// vector that needs no image unchanged), compacts the list in place to the
// atom indices that pass (with SLD_WRAP where find_image moved the vector),
// and does the per-pair work (density, exchange list).  The lists and sums
// are those of one exact pass.  In one pass, some lane of a warp accepts
// almost every candidate (about 26 of 162 pass), so the per-pair body would
// run, divergent, for nearly every candidate of every lane.
//
// The loose test keeps every pair the exact one keeps: with coordinates
// below B in magnitude, each FP32 rounding moves a coordinate by at most
// e = ulp(B)/2; a pair-vector component collects five of them (two
// positions, the cell offset, two differences), so r^2 near the cutoff moves
// by at most 2 r_max (5 sqrt(3) e) + (5 sqrt(3) e)^2 plus the FP32 rounding of
// the sum.  D.pair_loose, set on the host from the cell size, is twice that.
template <int MODE, bool ORTHO>
__device__ void pairs_one(const Dev& D, int i, int write_rho) {
    unsigned* err = &D.ctl->err;
    const int N = D.natom;
    const double4 ri = D.r[i];
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    // pass 1: loose cutoff test in the reference's traversal order
    int nn = 0;
    const int myslot = D.cell_slot[i];
    {
        const int4 fi = __ldg(D.fxs + myslot);
        const FxMat M = fx_mat(D);
        const float cut = (float)D.rcut_max_sq + D.pair_loose;
        for (int k = 0; k < 27; ++k) {
            const int c = k == 26 ? c0 : nbr_cell(D, cx, cy, cz, k);
            // this atom seen from the neighbour cell
            const int ex = fi.x - kNbr[k][0] * SLD_FX_ONE, ey = fi.y - kNbr[k][1] * SLD_FX_ONE,
                      ez = fi.z - kNbr[k][2] * SLD_FX_ONE;
            const int st = __ldg(D.cell_start + c), n = min(__ldg(D.cell_count + c), SLD_MAXC);
            for (int m0 = 0; m0 < n; m0 += 4) {
                int4 q[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    q[u] = m0 + u < n ? __ldg(D.fxs + st + m0 + u) : make_int4(ex, ey, ez, 0);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int slot = st + m0 + u;
                    const float3 d = fx_vec<ORTHO>(M, ex - q[u].x, ey - q[u].y, ez - q[u].z);
                    if (m0 + u < n && d.x * d.x + d.y * d.y + d.z * d.z < cut && slot != myslot) {
                        if (nn < SLD_MAXNB) D.nbr[(size_t)nn * N + i] = slot;
                        ++nn;
                    }
                }
            }
        }
    }
    const int nl = nn < SLD_MAXNB ? nn : SLD_MAXNB;
    // pass 2: the exact test, density and exchange list over the candidates
    double rho = 0.0;
    int nj = 0, w = 0;
    for (int e = 0; e < nl; ++e) {
        const int ps = D.nbr[(size_t)e * N + i];
        const int j = D.cell_atoms[ps];
        const double4 rj = D.r[j];
        bool moved;
        const double3 d = find_image_f(D, make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z), moved);
        const double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
        if (!(rsq < D.rcut_max_sq)) continue;
        D.nbr[(size_t)w * N + i] = j | (moved ? SLD_WRAP : 0);
        ++w;
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
    }
    if (nn > SLD_MAXNB || nj > SLD_MAXJ) atomicOr(err, SLD_FLAG_CAPACITY);
    D.nbr_n[i] = w;
    D.jl_n[i] = nj < SLD_MAXJ ? nj : SLD_MAXJ;
    if (write_rho) D.rho[i] = rho;
}

template <int MODE, bool ORTHO>
__global__ void __launch_bounds__(128) k_pairs(Dev D, int write_rho) {
    // one atom per thread; a capped grid walks several atoms per thread
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x)
        pairs_one<MODE, ORTHO>(D, i, write_rho);
}

// ---------------------------------------------------------------------
// Split form: pair distances in FP32 from the cell-relative positions.
//
// Pass 1 walks the 27 cells and keeps every candidate with |d|^2 < rcut_max^2
// in FP32 (its slot and neighbour cell k, packed slot | k << 27); pass 2
// forms the same d again from the list, writes the atom index (nbr, with
// SLD_WRAP on every entry so that FP64 readers apply find_image, which
// leaves a vector that needs no image unchanged) and k (nbk), and adds the
// density and the exchange row.  A pair within a few 1e-7 A of the cutoff
// may be kept or dropped otherwise than in FP64; every term is zero there
// (the density and pair terms' last knots, 3.0 and 4.1 A, and the exchange's
// 3.75 A lie inside the cutoffs).
#define SLD_SPLIT_SLOT_BITS 27
template <bool ORTHO>
__device__ void pairs_split_one(const Dev& D, const int4* koff, int i, int write_rho) {
    const int N = D.natom;
    int c0 = D.cell_of[i], cx, cy, cz;
    cell_xyz(D, c0, cx, cy, cz);
    const int myslot = D.cell_slot[i];
    const int4 fi = __ldg(D.fxs + myslot);
    const FxMat M = fx_mat(D);
    const float cut = (float)D.rcut_max_sq;
    int nn = 0;
    for (int k = 0; k < 27; ++k) {
        const int c = k == 26 ? c0 : nbr_cell(D, cx, cy, cz, k);
        const int ex = fi.x - kNbr[k][0] * SLD_FX_ONE, ey = fi.y - kNbr[k][1] * SLD_FX_ONE,
                  ez = fi.z - kNbr[k][2] * SLD_FX_ONE;
        const int st = __ldg(D.cell_start + c), n = min(__ldg(D.cell_count + c), SLD_MAXC);
        for (int m0 = 0; m0 < n; m0 += 4) {
            int4 q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                q[u] = m0 + u < n ? __ldg(D.fxs + st + m0 + u) : make_int4(ex, ey, ez, 0);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int slot = st + m0 + u;
                const float3 d = fx_vec<ORTHO>(M, ex - q[u].x, ey - q[u].y, ez - q[u].z);
                if (m0 + u < n && d.x * d.x + d.y * d.y + d.z * d.z < cut && slot != myslot) {
                    if (nn < SLD_MAXNB)
                        D.nbr[(size_t)nn * N + i] =
                            (int)((unsigned)slot | ((unsigned)k << SLD_SPLIT_SLOT_BITS));
                    ++nn;
                }
            }
        }
    }
    const int nl = nn < SLD_MAXNB ? nn : SLD_MAXNB;
    Kahan rho;
    const float rmag2 = (float)D.rcut_mag_sq, rpot = (float)D.rcut_pot;
    const Knots32 K = knots32(D);
    int nj = 0;
    for (int e0 = 0; e0 < nl; e0 += 4) {
        int sb[4], kb[4], jb[4];
        int4 qb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int ps = e0 + u < nl ? D.nbr[(size_t)(e0 + u) * N + i] : 0;
            sb[u] = ps & ((1 << SLD_SPLIT_SLOT_BITS) - 1);
            kb[u] = (unsigned)ps >> SLD_SPLIT_SLOT_BITS;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            jb[u] = e0 + u < nl ? __ldg(D.cell_atoms + sb[u]) : 0;
            qb[u] = __ldg(D.fxs + sb[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (e0 + u >= nl) break;
            const int e = e0 + u, k = kb[u];
            const int4 o = koff[k];
            const float3 d = fx_vec<ORTHO>(M, fi.x - o.x - qb[u].x, fi.y - o.y - qb[u].y,
                                           fi.z - o.z - qb[u].z);
            const float rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            const float ir = rsqrtf(rsq), r = rsq * ir;
            D.nbr[(size_t)e * N + i] = jb[u] | SLD_WRAP;
            D.nbk[(size_t)e * N + i] = (unsigned char)k;
            if (r < rpot) {
                float f, df;
                dens32f(D, K, r, ir, f, df);
                rho.add(f);
            }
            if (rsq < rmag2) {
                if (nj < SLD_MAXJ) {
                    float J, dJ;
                    exch32f(r, ir, J, dJ);
                    D.jl[(size_t)i * SLD_MAXJ + nj] = jb[u];
                    D.jvf[(size_t)i * SLD_MAXJ + nj] = J;
                    D.jlk[(size_t)i * SLD_MAXJ + nj] = (unsigned char)k;
                }
                ++nj;
            }
        }
    }
    if (nn > SLD_MAXNB || nj > SLD_MAXJ) atomicOr(&D.ctl->err, SLD_FLAG_CAPACITY);
    D.nbr_n[i] = nl;
    D.jl_n[i] = nj < SLD_MAXJ ? nj : SLD_MAXJ;
    if (write_rho) D.rho[i] = rho.value();
}

template <bool ORTHO>
__global__ void __launch_bounds__(128) k_pairs_split(Dev D, int write_rho) {
    __shared__ int4 koff[27];
    fx_offsets_load(koff);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x)
        pairs_split_one<ORTHO>(D, koff, i, write_rho);
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
        if (D.fm) {
            // the terms that the add below would add, kept apart
            D.fm[i] = make_double4(fx, fy, fz, 0.0);
            D.virm[i] = 0.5 * vir;
            double* om = D.stressm + 6 * (size_t)i;
            for (int k = 0; k < 6; ++k) om[k] = st6[k] / 2.0 / V;
        } else {
            // add to what the EAM part wrote
            double4 f = D.f[i];
            D.f[i] = make_double4(f.x + fx, f.y + fy, f.z + fz, 0.0);
            D.vir[i] += 0.5 * vir;
            for (int k = 0; k < 6; ++k) out[k] += st6[k] / 2.0 / V;
        }
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

// The magnetic part over the exchange rows (ROWS): an exchange entry is
// appended for a neighbour-list entry exactly when its pair vector passes
// the exchange cutoff, so the rows hold the neighbour list's magnetic pairs
// in its order and the sums are those of the pass over the neighbour list,
// with 14 entries per atom to gather instead of 26 (bcc Fe).

// FP64 force pass; AN: the analytic forms instead of the tables.  TEMP
// (with ROWS): also the spin terms of calculate_temperature into tv[0..3],
// from the exchange field summed as exchange_field does (the rows' J and the
// neighbours' spins, in row order).
template <bool AN, int PART, bool ROWS = false, bool TEMP = false>
__device__ __forceinline__ void force64_one(const Dev& D, int i, double4& tv) {
    static_assert(!ROWS || PART == PART_MAG, "the exchange rows hold the magnetic pairs only");
    static_assert(!TEMP || ROWS, "the temperature terms come from the exchange rows");
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
    double hx = 0, hy = 0, hz = 0, hj = 0;   // the exchange field (TEMP)
    if (TEMP && D.hext) {
        const double4 h = D.hext[i];
        hx = h.x; hy = h.y; hz = h.z;
    }
    const int nn = ROWS ? D.jl_n[i] : D.nbr_n[i];
    for (int e0 = 0; e0 < nn; e0 += 4) {
      int pkb[4];
      double4 rjb[4];
      double dFb[4];
      double4 sjb[4];
      double Jb[4];
      if constexpr (ROWS) {
          // find_image on every entry, which leaves a vector that needs no
          // image unchanged (the list's SLD_WRAP marks where it moves one)
          const int4 w = __ldg(reinterpret_cast<const int4*>(D.jl + (size_t)i * SLD_MAXJ + e0));
          const int q[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) pkb[u] = e0 + u < nn ? (q[u] | SLD_WRAP) : -1;
      } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) pkb[u] = e0 + u < nn ? D.nbr[(size_t)(e0 + u) * N + i] : -1;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
          int j = pkb[u] & SLD_JMASK;
          rjb[u] = pkb[u] >= 0 ? D.r[j] : ri;
          dFb[u] = (pkb[u] >= 0 && (PART & PART_EAM)) ? D.dF[j] : 0.0;
          if constexpr (TEMP) {
              sjb[u] = pkb[u] >= 0 ? D.s[j] : make_double4(0, 0, 0, 0);
              Jb[u] = pkb[u] >= 0 ? D.jv[(size_t)i * SLD_MAXJ + e0 + u] : 0.0;
          }
      }
      if constexpr (TEMP) {
#pragma unroll
          for (int u = 0; u < 4; ++u)
              if (pkb[u] >= 0) exch_add64(hx, hy, hz, hj, Jb[u], sjb[u]);
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
            double4 sj;
            if constexpr (TEMP) sj = sjb[u];
            else sj = D.s[j];
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
    if constexpr (TEMP)
        temp_spin_terms(D, i, make_double3(hx, hy, hz), hj, tv.x, tv.y, tv.z, tv.w);
}

template <bool AN, int PART, bool ROWS = false>
__global__ void __launch_bounds__(128) k_force64(Dev D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x) {
        double4 unused;
        force64_one<AN, PART, ROWS>(D, i, unused);
    }
}

// the magnetic part and the spin terms of calculate_temperature, one atom a
// thread (the node sums need the lanes of a warp on consecutive atoms)
template <bool AN>
__global__ void __launch_bounds__(128) k_force64_temp(Dev D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double4 t;
    force64_one<AN, PART_MAG, true, true>(D, i, t);
    double v[4] = {t.x, t.y, t.z, t.w};
    node_add<4>(D, D.node[i], v, 4);
}

// Split form: FP32 pair vectors from the fixed-point cell positions (fxa, the
// neighbour cell of each entry in nbk), the potential's FP32 forms with the
// reference's derivatives, compensated (Kahan) FP32 sums for the forces and
// energies; the stress and virial products (FP32) are summed in FP64.  Four
// entries' loads are issued together.
template <int PART, bool ORTHO, bool ROWS = false, bool TEMP = false>
__device__ __forceinline__ void force32_one(const Dev& D, const int4* koff, int i, double4& tv) {
    static_assert(!ROWS || PART == PART_MAG, "the exchange rows hold the magnetic pairs only");
    static_assert(!TEMP || ROWS, "the temperature terms come from the exchange rows");
    const int N = D.natom;
    const int4 fi = __ldg(D.fxa + i);
    const FxMat M = fx_mat(D);
    double4 si = (PART & PART_MAG) ? D.s[i] : make_double4(0, 0, 0, 0);
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    float sx = (float)si.x, sy = (float)si.y, sz = (float)si.z;
    float si_sqf = sx * sx + sy * sy + sz * sz;
    double rho_i = D.rho[i];
    float dF_i = (PART & PART_EAM) ? (float)D.dF[i] : 0.f;
    const float rpot = (float)D.rcut_pot, rmag2 = (float)D.rcut_mag_sq;
    const Knots32 K = knots32(D);
    Kahan fx, fy, fz, pe, me, me0;
    double st[6] = {0, 0, 0, 0, 0, 0}, vir = 0.0;
    float ks[4] = {0, 0, 0, 0}, kc[4] = {0, 0, 0, 0};   // the exchange field (TEMP)
    const int nn = ROWS ? D.jl_n[i] : D.nbr_n[i];
    for (int e0 = 0; e0 < nn; e0 += 4) {
        int jb[4], kb[4];
        int4 qb[4];
        float4 sb[4];
        float dFb[4];
        float4 Jw = make_float4(0.f, 0.f, 0.f, 0.f);
        if constexpr (ROWS) {
            const size_t at = (size_t)i * SLD_MAXJ + e0;
            const int4 w = __ldg(reinterpret_cast<const int4*>(D.jl + at));
            const unsigned kw = __ldg(reinterpret_cast<const unsigned*>(D.jlk + at));
            if constexpr (TEMP) Jw = __ldg(reinterpret_cast<const float4*>(D.jvf + at));
            const int q[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in = e0 + u < nn;
                jb[u] = in ? q[u] : i;
                kb[u] = in ? (int)((kw >> (8 * u)) & 255u) : 26;
            }
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in = e0 + u < nn;
                jb[u] = in ? (D.nbr[(size_t)(e0 + u) * N + i] & SLD_JMASK) : i;
                kb[u] = in ? D.nbk[(size_t)(e0 + u) * N + i] : 26;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            qb[u] = __ldg(D.fxa + jb[u]);
            dFb[u] = (PART & PART_EAM) ? (float)__ldg(D.dF + jb[u]) : 0.f;
            sb[u] = (PART & PART_MAG) ? __ldg(D.s32 + jb[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if constexpr (TEMP) {
            const float Jq[4] = {Jw.x, Jw.y, Jw.z, Jw.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (e0 + u < nn) exch_add32(ks, kc, Jq[u], sb[u]);
        }
        // the batch's stress and virial products, summed in FP32 and added
        // to the FP64 sums once per batch
        float bst[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (e0 + u >= nn) break;
            const int4 o = koff[kb[u]];
            const float3 d = fx_vec<ORTHO>(M, fi.x - o.x - qb[u].x, fi.y - o.y - qb[u].y,
                                           fi.z - o.z - qb[u].z);
            const float dx = d.x, dy = d.y, dz = d.z;
            const float rsq = dx * dx + dy * dy + dz * dz;
            const float ir = rsqrtf(rsq);
            const float r0 = rsq * ir;
            float dudr = 0.f;
            if ((PART & PART_EAM) && r0 < rpot) {
                float f, df, phi, dphi;
                dens32f(D, K, r0, ir, f, df);
                pair32f(D, K, r0, ir, phi, dphi);
                dudr = (dF_i + dFb[u]) * df + dphi;
                pe.add(0.5f * phi);
            }
            if ((PART & PART_MAG) && rsq < rmag2) {
                const float tx = sb[u].x, ty = sb[u].y, tz = sb[u].z;
                float sj_sq = tx * tx + ty * ty + tz * tz;
                float dot = sx * tx + sy * ty + sz * tz;
                float times = sqrtf(si_sqf * sj_sq);
                float J, dJ;
                exch32f(r0, ir, J, dJ);
                dudr += -dJ * (dot - times);
                float Jh = 0.5f * J;
                me0.add(Jh * times);
                me.add(-Jh * dot);
            }
            if (dudr == 0.f && PART != PART_ALL) continue;
            const float force = -dudr * ir;
            const float gx = force * dx, gy = force * dy, gz = force * dz;
            fx.add(gx); fy.add(gy); fz.add(gz);
            bst[0] += gx * dx; bst[1] += gy * dy; bst[2] += gz * dz;
            bst[3] += gx * dy; bst[4] += gy * dz; bst[5] += gz * dx;
            bst[6] += -force * rsq;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) st[k] += (double)bst[k];
        vir += (double)bst[6];
    }
    double F = 0.0;
    if (PART & PART_EAM) F = interp(D.tF, rho_i, D.inv_rho, &D.ctl->err);
    force_finish<PART>(D, i, si_sq, rho_i, F, fx.value(), fy.value(), fz.value(),
                       pe.value(), me.value(), me0.value(), vir, st);
    if constexpr (TEMP) {
        // exchange_field's split-form result: the compensated sums, then the
        // external field added in FP64
        double hx = (double)ks[0] - (double)kc[0], hy = (double)ks[1] - (double)kc[1],
               hz = (double)ks[2] - (double)kc[2];
        const double hj = (double)ks[3] - (double)kc[3];
        if (D.hext) {
            const double4 h = D.hext[i];
            hx = h.x + hx; hy = h.y + hy; hz = h.z + hz;
        }
        temp_spin_terms(D, i, make_double3(hx, hy, hz), hj, tv.x, tv.y, tv.z, tv.w);
    }
}

template <int PART, bool ORTHO, bool ROWS = false>
__global__ void __launch_bounds__(128) k_force32(Dev D) {
    // one atom per thread; a capped grid walks several atoms per thread
    __shared__ int4 koff[27];
    fx_offsets_load(koff);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.natom; i += gridDim.x * blockDim.x) {
        double4 unused;
        force32_one<PART, ORTHO, ROWS>(D, koff, i, unused);
    }
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
    if (D.split) {
        if (box_ortho(D)) k_force32<PART, true><<<nb, bs, 0, st>>>(D);
        else k_force32<PART, false><<<nb, bs, 0, st>>>(D);
    }
    else if (D.analytic) k_force64<true, PART><<<nb, bs, 0, st>>>(D);
    else k_force64<false, PART><<<nb, bs, 0, st>>>(D);
}

void launch_pairs(const Dev& D, cudaStream_t st, bool write_rho) {
    int w = write_rho ? 1 : 0;
    const int bs = D.tune.pair_block > 0 ? D.tune.pair_block : 128;
    int nb = capped_grid(div_up(D.natom, bs), D.tune.pair_cap);
    const bool ortho = box_ortho(D);
    if (D.split) {
        if (ortho) k_pairs_split<true><<<nb, bs, 0, st>>>(D, w);
        else k_pairs_split<false><<<nb, bs, 0, st>>>(D, w);
    } else if (D.analytic) {
        if (ortho) k_pairs<2, true><<<nb, bs, 0, st>>>(D, w);
        else k_pairs<2, false><<<nb, bs, 0, st>>>(D, w);
    } else {
        if (ortho) k_pairs<0, true><<<nb, bs, 0, st>>>(D, w);
        else k_pairs<0, false><<<nb, bs, 0, st>>>(D, w);
    }
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
template <bool ORTHO>
__global__ void __launch_bounds__(128) k_force32_temp(Dev D) {
    __shared__ int4 koff[27];
    fx_offsets_load(koff);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double4 t;
    force32_one<PART_MAG, ORTHO, true, true>(D, koff, i, t);
    double v[4] = {t.x, t.y, t.z, t.w};
    node_add<4>(D, D.node[i], v, 4);
}

// f, vir and stress plus the magnetic parts kept apart (D.fm): the same
// single addition per element as the magnetic pass's add.  f is left out
// when an external force is set: the kick then stores its f + fm + fext.
__global__ void __launch_bounds__(256) k_fold_mag(Dev D, int with_f) {
    const size_t n = (size_t)D.natom;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 6 * n) D.stress[t] = D.stress[t] + D.stressm[t];
    if (t < n) {
        D.vir[t] = D.vir[t] + D.virm[t];
        if (with_f) {
            const double4 f = D.f[t], g = D.fm[t];
            D.f[t] = make_double4(f.x + g.x, f.y + g.y, f.z + g.z, 0.0);
        }
    }
}
void launch_fold_mag(const Dev& D, cudaStream_t st) {
    k_fold_mag<<<div_up(6L * D.natom, 256), 256, 0, st>>>(D, D.fext ? 0 : 1);
}

// the magnetic part from the exchange rows of the list pass that ran on the
// same positions (the step graph's order); temp: also the spin terms of
// calculate_temperature into the Te-node accumulators (launch_temperature_begin
// zeroes them; the last kick's rescale adds the kinetic terms)
void launch_force_mag(const Dev& D, cudaStream_t st, bool temp) {
    const int bs = D.tune.force_block > 0 ? D.tune.force_block : 128;
    const int nb = div_up(D.natom, bs);
    if (temp) {
        const int nt = div_up(D.natom, 128);
        if (D.split) {
            if (box_ortho(D)) k_force32_temp<true><<<nt, 128, 0, st>>>(D);
            else k_force32_temp<false><<<nt, 128, 0, st>>>(D);
        }
        else if (D.analytic) k_force64_temp<true><<<nt, 128, 0, st>>>(D);
        else k_force64_temp<false><<<nt, 128, 0, st>>>(D);
        return;
    }
    if (D.split) {
        if (box_ortho(D)) k_force32<PART_MAG, true, true><<<nb, bs, 0, st>>>(D);
        else k_force32<PART_MAG, false, true><<<nb, bs, 0, st>>>(D);
    }
    else if (D.analytic) k_force64<true, PART_MAG, true><<<nb, bs, 0, st>>>(D);
    else k_force64<false, PART_MAG, true><<<nb, bs, 0, st>>>(D);
}
