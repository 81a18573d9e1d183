// Kernels of the adjoint (sld_adjoint.cu): the NVE spin-lattice step with a
// parameterised potential (forward), and the reverse of each of its parts.
//
// Forward, per step (core.cpp:55-63 without thermostats):
//   links | dp(dt/2) | ds(dt/2) | dr(dt) | neighbour lists, rho | ds(dt/2) |
//   forces | dp(dt/2)
// links, dr and the neighbour lists are the engine's own kernels (they do not
// depend on the parameters); rho, forces, the spin sweeps and the kicks are
// here, with the parameters theta.
//
// Reverse: every local term (a pair's force, density or exchange
// contribution, one spin rotation) is evaluated once more with its own
// inputs seeded as dual numbers; the partials are the rows of its Jacobian,
// contracted with the adjoints of its outputs.  Pair terms are symmetric in
// the full-shell lists, so each thread accumulates the partials for its own
// atom and half of the parameter partials; the spin sweeps are reversed visit
// by visit, colour group by colour group, in the opposite order.
#include "sld_adjpot.cuh"
#include "sld_adjoint.cuh"
#include "sld_pot32.cuh"

namespace {

__device__ __forceinline__ double3 adj_pair_vec(const Dev& D, double4 ri, int pk, double4& rj) {
    int j = pk & SLD_JMASK;
    rj = D.r[j];
    double3 d = make_double3(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z);
    if (pk & SLD_WRAP) d = find_image(D, d);
    return d;
}

// warp sum of v on every lane
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block sum of v; every thread gets the total
__device__ double block_total(double v, double* sh) {
    v = warp_sum(v);
    int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < nw; ++k) t += sh[k];
    return t;
}

// block sums of loc[lo, hi) into out[lo, hi) of this block's partial row
__device__ void block_theta(const double* loc, int lo, int hi, double* row, double* sh) {
    for (int k = lo; k < hi; ++k) {
        double t = block_total(loc[k], sh);
        if (threadIdx.x == 0) row[k] += t;
    }
}

}  // namespace

// ---------------------------------------------------------------------
// forward

// rho_i = sum_j f(r_ij) over r_ij < rcut_pot (calculate_rho_CPU.cpp:33-69);
// dF_i = F'(rho_i).  SPLIT: the pair terms in FP32, summed with compensation.
template <bool SPLIT>
__global__ void __launch_bounds__(128) k_adj_rho(Dev D, AdjDev A, AdjConst K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    ThPlain th{K.th};
    double4 ri = D.r[i];
    double rho = 0.0;
    Kahan acc;
    int nn = D.nbr_n[i];
    for (int e = 0; e < nn; ++e) {
        double4 rj;
        double3 d = adj_pair_vec(D, ri, D.nbr[(size_t)e * D.natom + i], rj);
        double r0 = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
        if (r0 < D.rcut_pot) {
            if constexpr (SPLIT) {
                float f, df;
                adj_dens32(K, (float)r0, f, df);
                acc.add(f);
            } else {
                double f, df;
                adj_dens(r0, th, f, df);
                rho += f;
            }
        }
    }
    if constexpr (SPLIT) rho = acc.value();
    double F, dF;
    adj_emb(rho, th, F, dF);
    A.rho[i] = rho;
    A.dF[i] = dF;
}

// forces, energies and the exchange field (calculate_force_energy_CPU.cpp:
// 33-216 with the Landau slopes zero, inner_spin calculate_spin_CPU.cpp:
// 201-235); per atom: f, e = pe + me + me0, H, and |f|^2 + |H|^2 into the
// block partials [E, L]
template <bool SPLIT>
__global__ void __launch_bounds__(128) k_adj_force(Dev D, AdjDev A, AdjConst K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    ThPlain th{K.th};
    double e_i = 0.0, l_i = 0.0;
    if (i < D.natom) {
        double4 ri = D.r[i], si = D.s[i];
        double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
        double rho_i = A.rho[i], dF_i = A.dF[i];
        double fx = 0, fy = 0, fz = 0, pe = 0, me = 0, me0 = 0, hx = 0, hy = 0, hz = 0;
        Kahan kfx, kfy, kfz, kpe, kme, kme0, khx, khy, khz;
        const float six = (float)si.x, siy = (float)si.y, siz = (float)si.z;
        const float si_sq32 = six * six + siy * siy + siz * siz;
        int nn = D.nbr_n[i];
        for (int e = 0; e < nn; ++e) {
            int pk = D.nbr[(size_t)e * D.natom + i];
            int j = pk & SLD_JMASK;
            double4 rj;
            double3 d = adj_pair_vec(D, ri, pk, rj);
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            double r0 = sqrt(rsq);
            if constexpr (SPLIT) {
                float rf = (float)r0, dudr = 0.f;
                if (r0 < D.rcut_pot) {
                    float f, df, phi, dphi;
                    adj_dens32(K, rf, f, df);
                    adj_pair32(K, r0, phi, dphi);
                    dudr = ((float)dF_i + (float)A.dF[j]) * df + dphi;
                    kpe.add(0.5f * phi);
                }
                if (r0 < D.rcut_mag || rsq < D.rcut_mag_sq) {
                    double4 sj = D.s[j];
                    float sjx = (float)sj.x, sjy = (float)sj.y, sjz = (float)sj.z;
                    float J, dJ;
                    adj_exch32(K, rf, J, dJ);
                    if (r0 < D.rcut_mag) {
                        float sdot = six * sjx + siy * sjy + siz * sjz;
                        float stimes = sqrtf(si_sq32 * (sjx * sjx + sjy * sjy + sjz * sjz));
                        dudr += -dJ * (sdot - stimes);
                        kme.add(-0.5f * J * sdot);
                        kme0.add(0.5f * J * stimes);
                    }
                    if (rsq < D.rcut_mag_sq) {
                        khx.add(J * sjx); khy.add(J * sjy); khz.add(J * sjz);
                    }
                }
                float force = -dudr / rf;
                kfx.add(force * (float)d.x); kfy.add(force * (float)d.y); kfz.add(force * (float)d.z);
                continue;
            }
            double dudr = 0.0;
            if (r0 < D.rcut_pot) {
                double f, df, phi, dphi;
                adj_dens(r0, th, f, df);
                adj_pair(K, r0, th, phi, dphi);
                dudr = (dF_i + A.dF[j]) * df + dphi;
                pe += 0.5 * phi;
            }
            if (r0 < D.rcut_mag) {
                double4 sj = D.s[j];
                double J, dJ;
                adj_exch(r0, th, J, dJ);
                double sdot = si.x * sj.x + si.y * sj.y + si.z * sj.z;
                double stimes = sqrt(si_sq * (sj.x * sj.x + sj.y * sj.y + sj.z * sj.z));
                dudr += -dJ * (sdot - stimes);
                me += -0.5 * J * sdot;
                me0 += 0.5 * J * stimes;
            }
            if (rsq < D.rcut_mag_sq) {
                double4 sj = D.s[j];
                double J, dJ;
                adj_exch(r0, th, J, dJ);
                hx += J * sj.x; hy += J * sj.y; hz += J * sj.z;
            }
            double force = -dudr / r0;
            fx += force * d.x; fy += force * d.y; fz += force * d.z;
        }
        if constexpr (SPLIT) {
            fx = kfx.value(); fy = kfy.value(); fz = kfz.value();
            pe = kpe.value(); me = kme.value(); me0 = kme0.value();
            hx = khx.value(); hy = khy.value(); hz = khz.value();
        }
        double F, dF;
        adj_emb(rho_i, th, F, dF);
        pe += F;
        double s4 = si_sq * si_sq;
        me += K.th[TH_LANDAU] * si_sq + K.th[TH_LANDAU + 1] * s4 + K.th[TH_LANDAU + 2] * s4 * si_sq +
              K.th[TH_LANDAU + 3] * s4 * s4;
        D.f[i] = make_double4(fx, fy, fz, 0.0);
        A.H[i] = make_double4(hx, hy, hz, 0.0);
        e_i = pe + me + me0;
        l_i = fx * fx + fy * fy + fz * fz + hx * hx + hy * hy + hz * hz;
        A.e[i] = e_i;
    }
    __shared__ double sh[32];
    double te = block_total(e_i, sh);
    double tl = block_total(l_i, sh);
    if (threadIdx.x == 0) {
        A.part[2 * blockIdx.x] = te;
        A.part[2 * blockIdx.x + 1] = tl;
    }
}

// spin_rotation (core_ds_CPU.cpp:90-127): s rotated about -Heff/hbar by
// |Heff| dt / hbar
template <class T>
__device__ __forceinline__ void adj_rot(const T H[3], const T s[3], double dt, T out[3]) {
    const double hbar = 6.58211899e-16;
    T ox = H[0] / -hbar, oy = H[1] / -hbar, oz = H[2] / -hbar;
    T o0 = dsqrt(ox * ox + oy * oy + oz * oz);
    if (val(o0) > 0.0) {
        ox = ox / o0; oy = oy / o0; oz = oz / o0;
    } else {
        ox = Num<T>::c(0.0); oy = ox; oz = ox;
    }
    T o12 = ox * oy, o23 = oy * oz, o13 = ox * oz;
    T o1sq = ox * ox, o2sq = oy * oy, o3sq = oz * oz;
    T a = dsin(o0 * dt);
    T b = 1.0 - dcos(o0 * dt);
    out[0] = s[0] + (s[0] * b * (-o2sq - o3sq) + s[1] * (b * o12 - a * oz) + s[2] * (a * oy + b * o13));
    out[1] = s[1] + (s[1] * b * (-o1sq - o3sq) + s[2] * (b * o23 - a * ox) + s[0] * (a * oz + b * o12));
    out[2] = s[2] + (s[2] * b * (-o1sq - o2sq) + s[0] * (b * o13 - a * oy) + s[1] * (a * ox + b * o23));
}

// One colour group of an NVE spin sweep (core_ds_CPU.cpp:35-83 with
// calculate_spin_CPU.cpp:43-46): a warp walks one cell, head to tail
// (forward) or tail to head (backward), rotating each spin about its
// exchange field of the current neighbour spins; the lanes share the
// neighbours of the visit.
template <bool SPLIT>
__global__ void __launch_bounds__(128) k_adj_sweep(Dev D, AdjConst K, const int* cells, int n,
                                                   double dt, int backward) {
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    ThPlain th{K.th};
    int c = cells[w];
    int st = D.cell_start[c], cnt = cell_n(D, c);
    for (int m = 0; m < cnt; ++m) {
        int i = D.cell_atoms[st + (backward ? cnt - 1 - m : m)];
        double4 ri = D.r[i];
        double hx = 0, hy = 0, hz = 0;
        int nn = D.nbr_n[i];
        for (int e = lane; e < nn; e += 32) {
            int pk = D.nbr[(size_t)e * D.natom + i];
            double4 rj;
            double3 d = adj_pair_vec(D, ri, pk, rj);
            double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
            if (rsq < D.rcut_mag_sq) {
                double4 sj = D.s[pk & SLD_JMASK];
                if constexpr (SPLIT) {
                    float J, dJ;
                    adj_exch32(K, (float)sqrt(rsq), J, dJ);
                    hx += (double)(J * (float)sj.x);
                    hy += (double)(J * (float)sj.y);
                    hz += (double)(J * (float)sj.z);
                } else {
                    double J, dJ;
                    adj_exch(sqrt(rsq), th, J, dJ);
                    hx += J * sj.x; hy += J * sj.y; hz += J * sj.z;
                }
            }
        }
        hx = warp_allsum(hx); hy = warp_allsum(hy); hz = warp_allsum(hz);
        if (lane == 0) {
            double4 si = D.s[i];
            double H[3] = {hx, hy, hz}, s[3] = {si.x, si.y, si.z}, o[3];
            adj_rot(H, s, dt, o);
            D.s[i] = make_double4(o[0], o[1], o[2], sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]));
        }
        __syncwarp();
    }
}

// core_dp_CPU.cpp:51-85 without thermostats: p += dt f, then
// rescale_momentum (core_dp_CPU.cpp:268-312): the mean momentum removed and
// the kinetic energy restored.  One block; ppre keeps p + dt f for the
// reverse pass.
__global__ void __launch_bounds__(1024) k_adj_kick(Dev D, double h, double4* ppre) {
    __shared__ double sh[32];
    const int N = D.natom;
    double sx = 0, sy = 0, sz = 0, ko = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = D.p[i], f = D.f[i];
        p = make_double4(p.x + h * f.x, p.y + h * f.y, p.z + h * f.z, 0.0);
        ppre[i] = p;
        sx += p.x; sy += p.y; sz += p.z;
        ko += (p.x * p.x + p.y * p.y + p.z * p.z) / 2e0 / D.atmass;
    }
    double mx = block_total(sx, sh) / N, my = block_total(sy, sh) / N, mz = block_total(sz, sh) / N;
    ko = block_total(ko, sh);
    double kn = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i];
        double qx = p.x - mx, qy = p.y - my, qz = p.z - mz;
        kn += (qx * qx + qy * qy + qz * qz) / 2e0 / D.atmass;
    }
    kn = block_total(kn, sh);
    double factor = sqrt(ko / kn);
    if (kn < 1e-10) factor = 1e0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i];
        D.p[i] = make_double4(factor * (p.x - mx), factor * (p.y - my), factor * (p.z - mz), 0.0);
    }
}

// dE/dtheta of one configuration: each atom's energy with every parameter
// seeded (its density as a dual number, so F(rho) carries the density
// parameters), block partials of the 36 partials in A.thb
__global__ void __launch_bounds__(128) k_adj_energy_grad(Dev D, AdjDev A, AdjConst K) {
    typedef Dual<ADJ_NTHETA> T;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    ThSeed<ADJ_NTHETA> th{K.th, 0, 0, ADJ_NTHETA};
    double loc[ADJ_NTHETA];
    for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = 0.0;
    if (i < D.natom) {
        double4 ri = D.r[i], si = D.s[i];
        double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
        T rho = dconst<ADJ_NTHETA>(0.0), e = rho;
        int nn = D.nbr_n[i];
        for (int m = 0; m < nn; ++m) {
            int pk = D.nbr[(size_t)m * D.natom + i];
            double4 rj;
            double3 d = adj_pair_vec(D, ri, pk, rj);
            double r0 = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
            T r = dconst<ADJ_NTHETA>(r0);
            if (r0 < D.rcut_pot) {
                T f, df, phi, dphi;
                adj_dens(r, th, f, df);
                adj_pair(K, r, th, phi, dphi);
                rho += f;
                e += 0.5 * phi;
            }
            if (r0 < D.rcut_mag) {
                double4 sj = D.s[pk & SLD_JMASK];
                T J, dJ;
                adj_exch(r, th, J, dJ);
                double sdot = si.x * sj.x + si.y * sj.y + si.z * sj.z;
                double stimes = sqrt(si_sq * (sj.x * sj.x + sj.y * sj.y + sj.z * sj.z));
                e += J * (0.5 * (stimes - sdot));
            }
        }
        T F, dF;
        adj_emb(rho, th, F, dF);
        e += F;
        double s4 = si_sq * si_sq;
        double pw[4] = {si_sq, s4, s4 * si_sq, s4 * s4};
        for (int k = 0; k < 4; ++k) e += th(TH_LANDAU + k) * pw[k];
        for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = e.d[k];
    }
    __shared__ double sh[32];
    block_theta(loc, 0, ADJ_NTHETA, A.thb + (size_t)blockIdx.x * ADJ_NTHETA, sh);
}

// Forward-mode Jacobians of one configuration.  d rho_i / d theta over the
// density's 12 parameters (theta 2..13): natom x 12.
__global__ void __launch_bounds__(128) k_adj_rho_tan(Dev D, AdjDev A, AdjConst K, double* drho) {
    typedef Dual<12> T;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    ThSeed<12> th{K.th, -TH_DA, TH_DA, TH_DA + 12};
    double4 ri = D.r[i];
    T rho = dconst<12>(0.0);
    int nn = D.nbr_n[i];
    for (int e = 0; e < nn; ++e) {
        double4 rj;
        double3 d = adj_pair_vec(D, ri, D.nbr[(size_t)e * D.natom + i], rj);
        double r0 = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
        if (r0 < D.rcut_pot) {
            T f, df;
            adj_dens(dconst<12>(r0), th, f, df);
            rho += f;
        }
    }
    for (int k = 0; k < 12; ++k) drho[12 * (size_t)i + k] = rho.d[k];
}

// d f_i / d theta and d Heff_H,i / d theta: natom x 3 x 36 each, slot order.
// The densities carry their parameter partials (drho), so F'(rho) takes both
// its own parameters' and the density parameters' partials.
#define ADJ_NJ TH_LANDAU
__global__ void __launch_bounds__(128) k_adj_force_tan(Dev D, AdjDev A, AdjConst K,
                                                       const double* __restrict__ drho,
                                                       double* df, double* dh) {
    typedef Dual<ADJ_NJ> T;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    ThSeed<ADJ_NJ> th{K.th, 0, 0, ADJ_NJ};
    auto rho_of = [&](int a) {
        T x = dconst<ADJ_NJ>(A.rho[a]);
        for (int k = 0; k < 12; ++k) x.d[TH_DA + k] = drho[12 * (size_t)a + k];
        return x;
    };
    double4 ri = D.r[i], si = D.s[i];
    double si_sq = si.x * si.x + si.y * si.y + si.z * si.z;
    T F_i, dF_i;
    adj_emb(rho_of(i), th, F_i, dF_i);
    T fx = dconst<ADJ_NJ>(0.0), fy = fx, fz = fx, hx = fx, hy = fx, hz = fx;
    int nn = D.nbr_n[i];
    for (int e = 0; e < nn; ++e) {
        int pk = D.nbr[(size_t)e * D.natom + i];
        int j = pk & SLD_JMASK;
        double4 rj;
        double3 d = adj_pair_vec(D, ri, pk, rj);
        double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
        double r0 = sqrt(rsq);
        T r = dconst<ADJ_NJ>(r0);
        T dudr = dconst<ADJ_NJ>(0.0);
        if (r0 < D.rcut_pot) {
            T f, dfr, phi, dphi, F_j, dF_j;
            adj_dens(r, th, f, dfr);
            adj_pair(K, r, th, phi, dphi);
            adj_emb(rho_of(j), th, F_j, dF_j);
            dudr = (dF_i + dF_j) * dfr + dphi;
        }
        T J, dJ;
        adj_exch(r, th, J, dJ);
        double4 sj = D.s[j];
        if (r0 < D.rcut_mag) {
            double sdot = si.x * sj.x + si.y * sj.y + si.z * sj.z;
            double stimes = sqrt(si_sq * (sj.x * sj.x + sj.y * sj.y + sj.z * sj.z));
            dudr = dudr - dJ * (sdot - stimes);
        }
        if (rsq < D.rcut_mag_sq) {
            hx += J * sj.x; hy += J * sj.y; hz += J * sj.z;
        }
        T force = -dudr / r0;
        fx += force * d.x; fy += force * d.y; fz += force * d.z;
    }
    const T* fv[3] = {&fx, &fy, &fz};
    const T* hv[3] = {&hx, &hy, &hz};
    for (int c = 0; c < 3; ++c) {
        double* o = df + (3 * (size_t)i + c) * ADJ_NTHETA;
        double* q = dh + (3 * (size_t)i + c) * ADJ_NTHETA;
        for (int k = 0; k < ADJ_NTHETA; ++k) {
            o[k] = k < ADJ_NJ ? fv[c]->d[k] : 0.0;   // the Landau constants move no force
            q[k] = k < ADJ_NJ ? hv[c]->d[k] : 0.0;
        }
    }
}

void adj_jacobians(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st, double* drho,
                   double* df, double* dh) {
    int nb = (D.natom + 127) / 128;
    k_adj_rho_tan<<<nb, 128, 0, st>>>(D, A, K, drho);
    k_adj_force_tan<<<nb, 128, 0, st>>>(D, A, K, drho, df, dh);
}

// ---------------------------------------------------------------------
// reverse

// Forces.  g_ij = (fbar_i - fbar_j) . f_ij is the pair's share of
// sum_i fbar_i . f_i; the partials of g_ij in r_i, rho_i, s_i go to this
// atom, half of those in theta to the block partials (atom j takes the other
// half on its own visit of the pair).
#define ADJ_NF (7 + TH_LANDAU)
__global__ void __launch_bounds__(128) k_adj_force_rev(Dev D, AdjDev A, AdjConst K) {
    typedef Dual<ADJ_NF> T;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double loc[ADJ_NTHETA];
    for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = 0.0;
    if (i < D.natom) {
        ThSeed<ADJ_NF> th{K.th, 7, 0, TH_LANDAU};
        double4 ri = D.r[i], si4 = D.s[i], fbi = A.fb[i];
        T rx = dseed<ADJ_NF>(ri.x, 0), ry = dseed<ADJ_NF>(ri.y, 1), rz = dseed<ADJ_NF>(ri.z, 2);
        T rho_i = dseed<ADJ_NF>(A.rho[i], 3);
        T six = dseed<ADJ_NF>(si4.x, 4), siy = dseed<ADJ_NF>(si4.y, 5), siz = dseed<ADJ_NF>(si4.z, 6);
        T si_sq = six * six + siy * siy + siz * siz;
        T F_i, dF_i;
        adj_emb(rho_i, th, F_i, dF_i);
        double g[7] = {0, 0, 0, 0, 0, 0, 0};
        int nn = D.nbr_n[i];
        for (int m = lane; m < nn; m += 32) {
            int pk = D.nbr[(size_t)m * D.natom + i];
            int j = pk & SLD_JMASK;
            double4 rj;
            double3 d0 = adj_pair_vec(D, ri, pk, rj);
            // the image shift is constant; the pair vector carries r_i's partials
            T dx = rx + (d0.x - ri.x), dy = ry + (d0.y - ri.y), dz = rz + (d0.z - ri.z);
            T rsq = dx * dx + dy * dy + dz * dz;
            T r = dsqrt(rsq);
            T dudr = dconst<ADJ_NF>(0.0);
            if (val(r) < D.rcut_pot) {
                T f, df, phi, dphi, F_j, dF_j;
                adj_dens(r, th, f, df);
                adj_pair(K, r, th, phi, dphi);
                adj_emb(dconst<ADJ_NF>(A.rho[j]), th, F_j, dF_j);
                dudr = (dF_i + dF_j) * df + dphi;
            }
            if (val(r) < D.rcut_mag) {
                double4 sj = D.s[j];
                T J, dJ;
                adj_exch(r, th, J, dJ);
                T sdot = six * sj.x + siy * sj.y + siz * sj.z;
                T stimes = dsqrt(si_sq * (sj.x * sj.x + sj.y * sj.y + sj.z * sj.z));
                dudr = dudr - dJ * (sdot - stimes);
            }
            T force = -dudr / r;
            double4 fbj = A.fb[j];
            double ux = fbi.x - fbj.x, uy = fbi.y - fbj.y, uz = fbi.z - fbj.z;
            T gij = force * (dx * ux + dy * uy + dz * uz);
            for (int k = 0; k < 7; ++k) g[k] += gij.d[k];
            for (int k = 0; k < TH_LANDAU; ++k) loc[k] += 0.5 * gij.d[7 + k];
        }
        for (int k = 0; k < 7; ++k) g[k] = warp_sum(g[k]);
        if (lane == 0) {
            double4 rb = A.rb[i];
            A.rb[i] = make_double4(rb.x + g[0], rb.y + g[1], rb.z + g[2], 0.0);
            A.rhob[i] += g[3];
            double4 sb = A.sb[i];
            A.sb[i] = make_double4(sb.x + g[4], sb.y + g[5], sb.z + g[6], 0.0);
        }
    }
    __shared__ double sh[32];
    block_theta(loc, 0, TH_LANDAU, A.thb + (size_t)blockIdx.x * ADJ_NTHETA, sh);
}

// Exchange field of the loss: Q_ij = J(r_ij) (hbar_i . s_j + hbar_j . s_i)
// is the pair's share of sum_i hbar_i . H_i.
__global__ void __launch_bounds__(128) k_adj_field_rev(Dev D, AdjDev A, AdjConst K) {
    typedef Dual<8> T;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double loc[ADJ_NTHETA];
    for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = 0.0;
    if (i < D.natom) {
        ThSeed<8> th{K.th, 6 - TH_JA, TH_JA, TH_JA + 2};
        double4 ri = D.r[i], si4 = D.s[i], hbi = A.hb[i];
        T rx = dseed<8>(ri.x, 0), ry = dseed<8>(ri.y, 1), rz = dseed<8>(ri.z, 2);
        T six = dseed<8>(si4.x, 3), siy = dseed<8>(si4.y, 4), siz = dseed<8>(si4.z, 5);
        double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int nn = D.nbr_n[i];
        for (int m = 0; m < nn; ++m) {
            int pk = D.nbr[(size_t)m * D.natom + i];
            int j = pk & SLD_JMASK;
            double4 rj;
            double3 d0 = adj_pair_vec(D, ri, pk, rj);
            if (d0.x * d0.x + d0.y * d0.y + d0.z * d0.z >= D.rcut_mag_sq) continue;
            T dx = rx + (d0.x - ri.x), dy = ry + (d0.y - ri.y), dz = rz + (d0.z - ri.z);
            T r = dsqrt(dx * dx + dy * dy + dz * dz);
            T J, dJ;
            adj_exch(r, th, J, dJ);
            double4 sj = D.s[j], hbj = A.hb[j];
            T q = J * ((hbi.x * sj.x + hbi.y * sj.y + hbi.z * sj.z) +
                       (six * hbj.x + siy * hbj.y + siz * hbj.z));
            for (int k = 0; k < 8; ++k) g[k] += q.d[k];
        }
        double4 rb = A.rb[i];
        A.rb[i] = make_double4(rb.x + g[0], rb.y + g[1], rb.z + g[2], 0.0);
        double4 sb = A.sb[i];
        A.sb[i] = make_double4(sb.x + g[3], sb.y + g[4], sb.z + g[5], 0.0);
        loc[TH_JA] = 0.5 * g[6];
        loc[TH_JRC] = 0.5 * g[7];
    }
    __shared__ double sh[32];
    block_theta(loc, TH_JA, TH_JA + 2, A.thb + (size_t)blockIdx.x * ADJ_NTHETA, sh);
}

// Densities: R_ij = (rhobar_i + rhobar_j) f(r_ij) is the pair's share of
// sum_i rhobar_i rho_i.  rhobar is cleared after use.
__global__ void __launch_bounds__(128) k_adj_rho_rev(Dev D, AdjDev A, AdjConst K) {
    const int NR = 3 + 12;
    typedef Dual<NR> T;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double loc[ADJ_NTHETA];
    for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = 0.0;
    double g[NR];
    for (int k = 0; k < NR; ++k) g[k] = 0.0;
    if (i < D.natom) {
        ThSeed<NR> th{K.th, 3 - TH_DA, TH_DA, TH_DA + 12};
        double4 ri = D.r[i];
        double rbi = A.rhob[i];
        T rx = dseed<NR>(ri.x, 0), ry = dseed<NR>(ri.y, 1), rz = dseed<NR>(ri.z, 2);
        int nn = D.nbr_n[i];
        for (int m = 0; m < nn; ++m) {
            int pk = D.nbr[(size_t)m * D.natom + i];
            int j = pk & SLD_JMASK;
            double4 rj;
            double3 d0 = adj_pair_vec(D, ri, pk, rj);
            if (sqrt(d0.x * d0.x + d0.y * d0.y + d0.z * d0.z) >= D.rcut_pot) continue;
            T dx = rx + (d0.x - ri.x), dy = ry + (d0.y - ri.y), dz = rz + (d0.z - ri.z);
            T r = dsqrt(dx * dx + dy * dy + dz * dz);
            T f, df;
            adj_dens(r, th, f, df);
            T q = f * (rbi + A.rhob[j]);
            for (int k = 0; k < NR; ++k) g[k] += q.d[k];
        }
        for (int k = 0; k < 12; ++k) loc[TH_DA + k] = 0.5 * g[3 + k];
    }
    __shared__ double sh[32];
    block_theta(loc, TH_DA, TH_DA + 12, A.thb + (size_t)blockIdx.x * ADJ_NTHETA, sh);
    // every block has read the densities' adjoints of its pairs before any
    // is cleared: the clearing runs in k_adj_rho_rev_done
    if (i < D.natom) {
        double4 rb = A.rb[i];
        A.rb[i] = make_double4(rb.x + g[0], rb.y + g[1], rb.z + g[2], 0.0);
    }
}

__global__ void k_adj_clear_rhob(AdjDev A, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) A.rhob[i] = 0.0;
}

// One colour group of a spin sweep, reversed.  s0 / s1 hold every spin
// before / after the sweep; a neighbour's spin at the time of a visit is its
// s1 if the forward sweep visited it earlier, else its s0.  sbar holds the
// adjoint of each spin's latest version in reverse order: a visit turns its
// atom's entry from the rotated spin's adjoint into the input spin's and
// adds the field's adjoint to the neighbours' entries.  A warp takes one
// cell, its lanes the neighbours of a visit.
__device__ __forceinline__ bool adj_visited_before(const Dev& D, const AdjDev& A, int c, int i,
                                                   int j, int backward, int group, bool& same) {
    int cj = D.cell_of[j];
    same = cj == c;
    if (same) return backward ? D.cell_slot[j] > D.cell_slot[i] : D.cell_slot[j] < D.cell_slot[i];
    return backward ? A.cell_group[cj] > group : A.cell_group[cj] < group;
}

__global__ void __launch_bounds__(128) k_adj_sweep_rev(Dev D, AdjDev A, AdjConst K,
                                                       const int* cells, int n, double dt,
                                                       int backward, int group,
                                                       const double4* __restrict__ s0,
                                                       const double4* __restrict__ s1) {
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double lj[2] = {0.0, 0.0};
    if (w < n) {
        int c = cells[w];
        int st = D.cell_start[c], cnt = cell_n(D, c);
        const double A0 = K.th[TH_JA], rc = K.th[TH_JRC];
        for (int m = cnt - 1; m >= 0; --m) {
            int pos = backward ? cnt - 1 - m : m;   // the forward walk's m-th visit
            int i = D.cell_atoms[st + pos];
            double4 ri = D.r[i];
            int nn = D.nbr_n[i];
            // the field of the visit
            double hx = 0, hy = 0, hz = 0;
            for (int e = lane; e < nn; e += 32) {
                int pk = D.nbr[(size_t)e * D.natom + i];
                int j = pk & SLD_JMASK;
                double4 rj;
                double3 d = adj_pair_vec(D, ri, pk, rj);
                double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
                if (rsq >= D.rcut_mag_sq) continue;
                double r = sqrt(rsq);
                if (r >= rc) continue;
                bool same;
                double4 sj = adj_visited_before(D, A, c, i, j, backward, group, same) ? s1[j] : s0[j];
                double u = 1.0 - r / rc;
                double J = A0 * u * u * u;
                hx += J * sj.x; hy += J * sj.y; hz += J * sj.z;
            }
            hx = warp_allsum(hx); hy = warp_allsum(hy); hz = warp_allsum(hz);
            // Jacobian of the rotation in (H, s), on every lane
            typedef Dual<6> T;
            double4 sp = s0[i];
            T H[3] = {dseed<6>(hx, 0), dseed<6>(hy, 1), dseed<6>(hz, 2)};
            T s[3] = {dseed<6>(sp.x, 3), dseed<6>(sp.y, 4), dseed<6>(sp.z, 5)};
            T o[3];
            adj_rot(H, s, dt, o);
            double4 sb = A.sb[i];
            double ob[3] = {sb.x, sb.y, sb.z};
            double hb[3], sin_[3];
            for (int k = 0; k < 3; ++k) {
                hb[k] = ob[0] * o[0].d[k] + ob[1] * o[1].d[k] + ob[2] * o[2].d[k];
                sin_[k] = ob[0] * o[0].d[3 + k] + ob[1] * o[1].d[3 + k] + ob[2] * o[2].d[3 + k];
            }
            __syncwarp();
            if (lane == 0) A.sb[i] = make_double4(sin_[0], sin_[1], sin_[2], 0.0);
            // the field's adjoint to the neighbours' spins, the positions and J
            double rbx = 0, rby = 0, rbz = 0;
            for (int e = lane; e < nn; e += 32) {
                int pk = D.nbr[(size_t)e * D.natom + i];
                int j = pk & SLD_JMASK;
                double4 rj;
                double3 d = adj_pair_vec(D, ri, pk, rj);
                double rsq = d.x * d.x + d.y * d.y + d.z * d.z;
                if (rsq >= D.rcut_mag_sq) continue;
                double r = sqrt(rsq);
                if (r >= rc) continue;
                bool same;
                double4 sj = adj_visited_before(D, A, c, i, j, backward, group, same) ? s1[j] : s0[j];
                double u = 1.0 - r / rc;
                double J = A0 * u * u * u;
                double dJ = -3.0 * A0 * u * u / rc;
                double hs = hb[0] * sj.x + hb[1] * sj.y + hb[2] * sj.z;
                double gx = hs * dJ * d.x / r, gy = hs * dJ * d.y / r, gz = hs * dJ * d.z / r;
                rbx += gx; rby += gy; rbz += gz;
                lj[0] += hs * u * u * u;
                lj[1] += hs * 3.0 * A0 * u * u * r / (rc * rc);
                double* sbj = reinterpret_cast<double*>(A.sb + j);
                double* rbj = reinterpret_cast<double*>(A.rb + j);
                if (same) {
                    // only this warp touches the atoms of its cell
                    sbj[0] += J * hb[0]; sbj[1] += J * hb[1]; sbj[2] += J * hb[2];
                    rbj[0] -= gx; rbj[1] -= gy; rbj[2] -= gz;
                } else {
                    atomicAdd(sbj, J * hb[0]); atomicAdd(sbj + 1, J * hb[1]);
                    atomicAdd(sbj + 2, J * hb[2]);
                    atomicAdd(rbj, -gx); atomicAdd(rbj + 1, -gy); atomicAdd(rbj + 2, -gz);
                }
            }
            rbx = warp_sum(rbx); rby = warp_sum(rby); rbz = warp_sum(rbz);
            if (lane == 0) {
                double4 rb = A.rb[i];
                A.rb[i] = make_double4(rb.x + rbx, rb.y + rby, rb.z + rbz, 0.0);
            }
            __syncwarp();
        }
    }
    double loc[ADJ_NTHETA];
    for (int k = 0; k < ADJ_NTHETA; ++k) loc[k] = 0.0;
    loc[TH_JA] = lj[0];
    loc[TH_JRC] = lj[1];
    __shared__ double sh[32];
    block_theta(loc, TH_JA, TH_JA + 2, A.thb + (size_t)blockIdx.x * ADJ_NTHETA, sh);
}

// Kick and momentum rescaling reversed.  p' = c q, q = ppre - <ppre>,
// c = sqrt(K_old / K_new): pbar' -> pbar of ppre; then fbar += h pbar and
// the momentum before the kick keeps pbar.  One block.
__global__ void __launch_bounds__(1024) k_adj_kick_rev(Dev D, AdjDev A, double h,
                                                       const double4* __restrict__ ppre) {
    __shared__ double sh[32];
    const int N = D.natom;
    double sx = 0, sy = 0, sz = 0, ko = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i];
        sx += p.x; sy += p.y; sz += p.z;
        ko += p.x * p.x + p.y * p.y + p.z * p.z;
    }
    double mx = block_total(sx, sh) / N, my = block_total(sy, sh) / N, mz = block_total(sz, sh) / N;
    ko = block_total(ko, sh);
    double kn = 0, sg = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i], b = A.pb[i];
        double qx = p.x - mx, qy = p.y - my, qz = p.z - mz;
        kn += qx * qx + qy * qy + qz * qz;
        sg += b.x * qx + b.y * qy + b.z * qz;
    }
    kn = block_total(kn, sh);
    sg = block_total(sg, sh);
    bool fixed = kn / 2e0 / D.atmass < 1e-10;
    double c = fixed ? 1.0 : sqrt(ko / kn);
    double kq = fixed ? 0.0 : c * sg / kn, kp = fixed ? 0.0 : c * sg / ko;
    // qbar = c pbar' - kq q; pbar = qbar - <qbar> + kp ppre
    double ax = 0, ay = 0, az = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i], b = A.pb[i];
        ax += c * b.x - kq * (p.x - mx);
        ay += c * b.y - kq * (p.y - my);
        az += c * b.z - kq * (p.z - mz);
    }
    ax = block_total(ax, sh) / N; ay = block_total(ay, sh) / N; az = block_total(az, sh) / N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double4 p = ppre[i], b = A.pb[i];
        double bx = c * b.x - kq * (p.x - mx) - ax + kp * p.x;
        double by = c * b.y - kq * (p.y - my) - ay + kp * p.y;
        double bz = c * b.z - kq * (p.z - mz) - az + kp * p.z;
        A.pb[i] = make_double4(bx, by, bz, 0.0);
        double4 fb = A.fb[i];
        A.fb[i] = make_double4(fb.x + h * bx, fb.y + h * by, fb.z + h * bz, 0.0);
    }
}

// the drift r += dt p / m reversed: pbar += dt/m rbar
__global__ void k_adj_drift_rev(Dev D, AdjDev A, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double k = dt / D.atmass;
    double4 rb = A.rb[i], pb = A.pb[i];
    A.pb[i] = make_double4(pb.x + k * rb.x, pb.y + k * rb.y, pb.z + k * rb.z, 0.0);
}

// the block partials of theta's adjoint added to the running total, in a
// fixed order, and cleared
__global__ void k_adj_theta_acc(AdjDev A, int nb) {
    int k = threadIdx.x;
    if (k >= ADJ_NTHETA) return;
    double t = 0.0;
    for (int b = 0; b < nb; ++b) {
        t += A.thb[(size_t)b * ADJ_NTHETA + k];
        A.thb[(size_t)b * ADJ_NTHETA + k] = 0.0;
    }
    A.theta_bar[k] += t;
}

// the block partials [E, L] of the forward force pass
__global__ void k_adj_el(AdjDev A, int nb, double* out2) {
    if (threadIdx.x != 0) return;
    double e = 0, l = 0;
    for (int b = 0; b < nb; ++b) { e += A.part[2 * b]; l += A.part[2 * b + 1]; }
    out2[0] = e;
    out2[1] = l;
}

// adjoint seeds of the loss L = sum |f|^2 + |H|^2: fbar = 2 f, hbar = 2 H
__global__ void k_adj_seed_loss(Dev D, AdjDev A) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double4 f = D.f[i], h = A.H[i], fb = A.fb[i];
    A.fb[i] = make_double4(fb.x + 2.0 * f.x, fb.y + 2.0 * f.y, fb.z + 2.0 * f.z, 0.0);
    A.hb[i] = make_double4(2.0 * h.x, 2.0 * h.y, 2.0 * h.z, 0.0);
}

// ---------------------------------------------------------------------
// launchers

static int adj_blocks(int n, int b) { return (n + b - 1) / b; }

void adj_rho(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st) {
    if (D.split)
        k_adj_rho<true><<<adj_blocks(D.natom, 128), 128, 0, st>>>(D, A, K);
    else
        k_adj_rho<false><<<adj_blocks(D.natom, 128), 128, 0, st>>>(D, A, K);
}
void adj_force(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st, double* el2) {
    int nb = adj_blocks(D.natom, 128);
    if (D.split)
        k_adj_force<true><<<nb, 128, 0, st>>>(D, A, K);
    else
        k_adj_force<false><<<nb, 128, 0, st>>>(D, A, K);
    if (el2) k_adj_el<<<1, 32, 0, st>>>(A, nb, el2);
}
void adj_sweep(const Dev& D, const AdjConst& K, cudaStream_t st, const int* cells, int n, double dt,
               bool backward) {
    if (n <= 0) return;
    int nb = adj_blocks(n, 4);   // a warp per cell
    if (D.split)
        k_adj_sweep<true><<<nb, 128, 0, st>>>(D, K, cells, n, dt, backward);
    else
        k_adj_sweep<false><<<nb, 128, 0, st>>>(D, K, cells, n, dt, backward);
}
void adj_kick(const Dev& D, cudaStream_t st, double h, double4* ppre) {
    k_adj_kick<<<1, 1024, 0, st>>>(D, h, ppre);
}
void adj_energy_grad(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st) {
    int nb = adj_blocks(D.natom, 128);
    k_adj_energy_grad<<<nb, 128, 0, st>>>(D, A, K);
    k_adj_theta_acc<<<1, 64, 0, st>>>(A, nb);
}
void adj_force_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st) {
    int nb = adj_blocks(D.natom, 4);   // a warp per atom
    k_adj_force_rev<<<nb, 128, 0, st>>>(D, A, K);
    k_adj_theta_acc<<<1, 64, 0, st>>>(A, nb);
}
void adj_field_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st) {
    int nb = adj_blocks(D.natom, 128);
    k_adj_field_rev<<<nb, 128, 0, st>>>(D, A, K);
    k_adj_theta_acc<<<1, 64, 0, st>>>(A, nb);
}
void adj_rho_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st) {
    int nb = adj_blocks(D.natom, 128);
    k_adj_rho_rev<<<nb, 128, 0, st>>>(D, A, K);
    k_adj_theta_acc<<<1, 64, 0, st>>>(A, nb);
    k_adj_clear_rhob<<<adj_blocks(D.natom, 256), 256, 0, st>>>(A, D.natom);
}
// the block partials of theta's adjoint stay in A.thb (rows < nb) until
// adj_theta_flush
void adj_sweep_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st,
                   const int* cells, int n, double dt, bool backward, int group, const double4* s0,
                   const double4* s1) {
    if (n <= 0) return;
    int nb = adj_blocks(n, 4);   // a warp per cell
    k_adj_sweep_rev<<<nb, 128, 0, st>>>(D, A, K, cells, n, dt, backward, group, s0, s1);
}
void adj_theta_flush(const AdjDev& A, cudaStream_t st, int nb) {
    k_adj_theta_acc<<<1, 64, 0, st>>>(A, nb);
}
void adj_kick_rev(const Dev& D, const AdjDev& A, cudaStream_t st, double h, const double4* ppre) {
    k_adj_kick_rev<<<1, 1024, 0, st>>>(D, A, h, ppre);
}
void adj_drift_rev(const Dev& D, const AdjDev& A, cudaStream_t st, double dt) {
    k_adj_drift_rev<<<adj_blocks(D.natom, 256), 256, 0, st>>>(D, A, dt);
}
void adj_seed_loss(const Dev& D, const AdjDev& A, cudaStream_t st) {
    k_adj_seed_loss<<<adj_blocks(D.natom, 256), 256, 0, st>>>(D, A);
}
