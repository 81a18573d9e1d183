// Lattice updates: core_dp (core_dp_CPU.cpp:51-312) and core_dr
// (core_dr_CPU.cpp:33-44).
//
// With the lattice thermostat, core_dp is C1(dt/2) B(dt/2) A(dt) B(dt/2)
// C2(dt/2).  Every one of those touches only the atoms of one link cell (C1
// and C2 mix the momenta inside a cell, A subtracts the cell mean of the
// noise, B is per atom), so one thread per cell runs the whole sequence on
// its atoms in the reference's list order: the momenta are read and written
// once per core_dp.  rescale_momentum (:268-312) then needs two global sums
// (total momentum, kinetic energy before/after removing it); they are formed
// by per-block partials and one finishing block, in a fixed order, so every
// run gives the same bits.
#include "sld_common.cuh"

// per-block sums of a kick for rescale_momentum: the momentum and the
// kinetic energy |p|^2 / 2 / m, each atom's rounded as the reference rounds
// its ke (core_dp_CPU.cpp:292)
__device__ __forceinline__ void block_partials4(const Dev& D, double a, double b, double c,
                                                double k) {
    __shared__ double sh[32];
    double ta = block_sum(a, sh);
    double tb = block_sum(b, sh);
    double tc = block_sum(c, sh);
    double tk = block_sum(k, sh);
    if (threadIdx.x == 0) {
        double* o = D.red + 4 * (size_t)blockIdx.x;
        o[0] = ta; o[1] = tb; o[2] = tc; o[3] = tk;
    }
}
__device__ __forceinline__ double ke_of(const Dev& D, double px, double py, double pz) {
    return (px * px + py * py + pz * pz) / 2.0 / D.atmass;
}

__global__ void __launch_bounds__(256) k_dp_nve(Dev D, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double px = 0, py = 0, pz = 0, kk = 0;
    if (i < D.natom) {
        double4 p = D.p[i], f = D.f[i];
        if (D.fm) {   // the magnetic part, kept apart
            const double4 g = D.fm[i];
            f.x = f.x + g.x; f.y = f.y + g.y; f.z = f.z + g.z;
        }
        if (D.fext) {
            // core_dp_CPU.cpp:68-71: the external force is added into f itself
            double4 e = D.fext[i];
            f.x = f.x + e.x; f.y = f.y + e.y; f.z = f.z + e.z;
            D.f[i] = f;
        }
        p.x = p.x + dt * f.x; p.y = p.y + dt * f.y; p.z = p.z + dt * f.z;
        D.p[i] = p;
        px = p.x; py = p.y; pz = p.z;
        kk = ke_of(D, p.x, p.y, p.z);
    }
    block_partials4(D, px, py, pz, kk);
}

__device__ __forceinline__ void add3(double4& a, double k, double x, double y, double z) {
    a.x = a.x + k * x; a.y = a.y + k * y; a.z = a.z + k * z;
}

// The momenta of one cell's atoms, m = 0..n-1 in list order: in the block's
// shared memory (cells of up to KDP_MAXA atoms: the kick's six passes then
// read and write shared memory, and global memory once each way) or in
// global memory.  The arithmetic is the same code for both.
#define KDP_BLOCK 128
#define KDP_MAXA 12
struct PGlobal {
    const Dev& D;
    const int* a;
    __device__ double3 get(int m) const {
        const double4 p = D.p[a[m]];
        return make_double3(p.x, p.y, p.z);
    }
    __device__ void set(int m, double3 v) const { D.p[a[m]] = make_double4(v.x, v.y, v.z, 0.0); }
};
struct PShared {
    double* s;   // s[(3 m + k) KDP_BLOCK]: component k of atom m of this thread's cell
    __device__ double3 get(int m) const {
        return make_double3(s[(3 * m) * KDP_BLOCK], s[(3 * m + 1) * KDP_BLOCK],
                            s[(3 * m + 2) * KDP_BLOCK]);
    }
    __device__ void set(int m, double3 v) const {
        s[(3 * m) * KDP_BLOCK] = v.x;
        s[(3 * m + 1) * KDP_BLOCK] = v.y;
        s[(3 * m + 2) * KDP_BLOCK] = v.z;
    }
};

// C1 / C2: p_i += gamma/m dt / n (sum_cell p - p_i), Gauss-Seidel in list
// order.  The reference re-adds the cell's momenta for every atom; here the
// cell sum is carried along and corrected by each update (the same sum up to
// rounding), so the pass is linear in the cell's size.
template <class P>
__device__ __forceinline__ void cell_mix(const Dev& D, const P& P_, int n, double dt, bool backward) {
    double factor = D.gamma_L / D.atmass * dt / n;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int m = 0; m < n; ++m) {
        double3 pm = P_.get(m);
        sx = sx + pm.x; sy = sy + pm.y; sz = sz + pm.z;
    }
    for (int q = 0; q < n; ++q) {
        const int m = backward ? n - 1 - q : q;
        double3 p = P_.get(m);
        double nx = p.x + factor * (sx - p.x);
        double ny = p.y + factor * (sy - p.y);
        double nz = p.z + factor * (sz - p.z);
        sx += nx - p.x; sy += ny - p.y; sz += nz - p.z;
        P_.set(m, make_double3(nx, ny, nz));
    }
}

template <class P>
__device__ __forceinline__ void friction(const Dev& D, const P& P_, int n, double dt) {
    double e = D.localcolmot ? exp(-D.gamma_L / D.atmass * dt * (1.0 - 1.0 / n))
                             : exp(-D.gamma_L / D.atmass * dt);
    for (int m = 0; m < n; ++m) {
        double3 p = P_.get(m);
        p.x = e * p.x; p.y = e * p.y; p.z = e * p.z;
        P_.set(m, p);
    }
}

// core_dp_CPU.cpp:51-85 for one cell: C1(dt/2) B(dt/2) A(dt) B(dt/2) C2(dt/2);
// returns the cell's momentum and kinetic-energy sums for rescale_momentum
template <class P>
__device__ __forceinline__ double4 dp_cell(const Dev& D, const P& P_, const int* a, int n, double dt,
                                           unsigned long long epoch) {
    if (D.localcolmot) cell_mix(D, P_, n, dt / 2.0, false);
    friction(D, P_, n, dt / 2.0);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int m = 0; m < n; ++m) {            // A: force + noise
        int i = a[m];
        double fx, fy, fz;
        if (D.quantum) {
            // core_dp_CPU.cpp:137-147: sqrt(2 gamma_L / h) times the coloured noise
            double amp = sqrt(2.0 * D.gamma_L / (dt * D.qM));
            double4 q = D.qnoise[i];
            fx = amp * q.x; fy = amp * q.y; fz = amp * q.z;
        } else {
            double T = D.eltemp ? D.Te[D.node[i]] : D.temperature;
            double amp = sqrt(2.0 * T * D.gamma_L / dt);
            double3 xi = D.split ? normals3_f32(D.seed, D.replica, (unsigned)D.id[i], epoch)
                                 : normals3(D.seed, D.replica, (unsigned)D.id[i], epoch);
            fx = amp * xi.x; fy = amp * xi.y; fz = amp * xi.z;
        }
        double4 f = D.f[i];
        if (D.fm) {   // the magnetic part, kept apart
            const double4 g = D.fm[i];
            f.x = f.x + g.x; f.y = f.y + g.y; f.z = f.z + g.z;
        }
        if (D.fext) {   // core_dp_CPU.cpp:129-132
            double4 e = D.fext[i];
            f.x = f.x + e.x; f.y = f.y + e.y; f.z = f.z + e.z;
            D.f[i] = f;
        }
        double3 p = P_.get(m);
        p.x = p.x + dt * (f.x + fx); p.y = p.y + dt * (f.y + fy); p.z = p.z + dt * (f.z + fz);
        P_.set(m, p);
        ax = ax + fx; ay = ay + fy; az = az + fz;
    }
    if (D.localcolmot) {
        ax = ax / n; ay = ay / n; az = az / n;
        for (int m = 0; m < n; ++m) {
            double3 p = P_.get(m);
            p.x = p.x - dt * ax; p.y = p.y - dt * ay; p.z = p.z - dt * az;
            P_.set(m, p);
        }
    }
    friction(D, P_, n, dt / 2.0);
    if (D.localcolmot) cell_mix(D, P_, n, dt / 2.0, true);
    double px = 0, py = 0, pz = 0, kk = 0;
    for (int m = 0; m < n; ++m) {
        double3 p = P_.get(m);
        px += p.x; py += p.y; pz += p.z;
        kk += ke_of(D, p.x, p.y, p.z);
    }
    return make_double4(px, py, pz, kk);
}

__global__ void __launch_bounds__(KDP_BLOCK) k_dp_lang(Dev D, double dt, int epoch_off) {
    __shared__ double sp[3 * KDP_MAXA * KDP_BLOCK];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double4 ps = make_double4(0.0, 0.0, 0.0, 0.0);
    if (c < D.ncells) {
        const int n = cell_n(D, c);
        const int* a = D.cell_atoms + D.cell_start[c];
        const unsigned long long epoch = D.ctl->epoch + (unsigned long long)epoch_off;
        if (n > 0 && n <= KDP_MAXA) {
            const PShared P_{sp + threadIdx.x};
            // all of the cell's loads in flight at once: the indices, then the momenta
            int idx[KDP_MAXA];
#pragma unroll
            for (int m = 0; m < KDP_MAXA; ++m) idx[m] = m < n ? __ldg(a + m) : 0;
#pragma unroll
            for (int m = 0; m < KDP_MAXA; ++m)
                if (m < n) {
                    const double4 p = D.p[idx[m]];
                    P_.set(m, make_double3(p.x, p.y, p.z));
                }
            ps = dp_cell(D, P_, a, n, dt, epoch);
#pragma unroll
            for (int m = 0; m < KDP_MAXA; ++m)
                if (m < n) {
                    const double3 p = P_.get(m);
                    D.p[idx[m]] = make_double4(p.x, p.y, p.z, 0.0);
                }
        } else if (n > 0) {
            ps = dp_cell(D, PGlobal{D, a}, a, n, dt, epoch);
        }
    }
    block_partials4(D, ps.x, ps.y, ps.z, ps.w);
}

// rescale_momentum (core_dp_CPU.cpp:268-311) from the kick's block sums: the
// mean momentum a, the kinetic energy before (sum of |p|^2 / 2m) and after
// removing a, which is the same sum less N |a|^2 / 2m (the reference sums
// |p - a|^2 / 2m atom by atom; the two agree to rounding), and the factor
// sqrt(ke_old / ke_new) that k_scale applies.
__global__ void __launch_bounds__(1024) k_rescale(Dev D, int nb) {
    __shared__ double sh[32];
    double a = 0, b = 0, c = 0, k = 0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
        a += D.red[4 * q]; b += D.red[4 * q + 1]; c += D.red[4 * q + 2]; k += D.red[4 * q + 3];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    k = block_sum(k, sh);
    if (threadIdx.x == 0) {
        const double n = (double)D.natom;
        const double ax = a / n, ay = b / n, az = c / n;
        D.ctl->avep[0] = ax;
        D.ctl->avep[1] = ay;
        D.ctl->avep[2] = az;
        const double ke_new = k - n * (ax * ax + ay * ay + az * az) / 2.0 / D.atmass;
        double factor = sqrt(k / ke_new);
        if (ke_new < 1e-10) factor = 1.0;
        D.ctl->ke_factor = factor;
    }
}

// TEMP: also the kinetic terms of calculate_temperature (the kinetic energy
// and the momentum) into the Te-node accumulators
template <bool TEMP>
__global__ void __launch_bounds__(256) k_scale(Dev D) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double k = D.ctl->ke_factor;
    double4 p = D.p[i];
    p.x = k * (p.x - D.ctl->avep[0]);
    p.y = k * (p.y - D.ctl->avep[1]);
    p.z = k * (p.z - D.ctl->avep[2]);
    D.p[i] = p;
    const double ke = (p.x * p.x + p.y * p.y + p.z * p.z) / 2.0 / D.atmass;
    D.ke[i] = ke;
    if constexpr (TEMP) {
        double v[4] = {ke, p.x, p.y, p.z};
        node_add<4>(D, D.node[i], v, 0);
    }
}

// SCALE: first finish the kick's rescale_momentum for this atom (as
// k_scale<false> does), for a step that defers it to the drift
template <bool SCALE>
__global__ void __launch_bounds__(256) k_dr(Dev D, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double k = dt / D.atmass;
    double4 r = D.r[i], p = D.p[i];
    if constexpr (SCALE) {
        const double f = D.ctl->ke_factor;
        p.x = f * (p.x - D.ctl->avep[0]);
        p.y = f * (p.y - D.ctl->avep[1]);
        p.z = f * (p.z - D.ctl->avep[2]);
        D.p[i] = p;
        D.ke[i] = (p.x * p.x + p.y * p.y + p.z * p.z) / 2.0 / D.atmass;
    }
    const double3 u = make_double3(r.x + k * p.x, r.y + k * p.y, r.z + k * p.z);
    double3 x = periodic(D, u);
    if (!isfinite(x.x + x.y + x.z)) atomicOr(&D.ctl->err, SLD_FLAG_NAN);
    D.r[i] = make_double4(x.x, x.y, x.z, 0.0);
    // the FP32 copy keeps the unwrapped position, relative to the cell the
    // atom is linked in until the next links
    const int4 q = cell_fix(D, D.cell_of[i], u.x, u.y, u.z);
    D.fxs[D.cell_slot[i]] = q;
    if (D.fxa) D.fxa[i] = q;
}

// quantum_noise_CPU.cpp:56-72 for every degree of freedom at once (their
// counters advance together): every M kicks, each atom's coloured noise is
// the filter over its history of normals, newest first.  With counter-based
// normals the history of update u is the draws t = u - Nf2 .. u - 1; the
// reference's initial history is the draws before update 0.
__global__ void __launch_bounds__(256) k_quantum_update(Dev D) {
    const long long c = D.ctl->qcount;
    if (c % D.qM != 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    const long long u = c / D.qM;
    double qx = 0.0, qy = 0.0, qz = 0.0;
    for (int k = 0; k < D.qNf2; ++k) {
        const double h = __ldg(D.qH + k);
        double3 x = normals3(D.seed, D.replica, (unsigned)D.id[i],
                             SLD_QEPOCH + (unsigned long long)(u - 1 - k + D.qNf2));
        qx += h * x.x; qy += h * x.y; qz += h * x.z;
    }
    D.qnoise[i] = make_double4(qx, qy, qz, 0.0);
}

__global__ void k_quantum_tick(Dev D) {
    if (threadIdx.x == 0) ++D.ctl->qcount;
}

void launch_dp(const Dev& D, cudaStream_t st, double dt, int epoch_off, bool temp,
               bool defer_scale) {
    int nb;
    if (D.lattlang) {
        if (D.quantum) k_quantum_update<<<div_up(D.natom, 256), 256, 0, st>>>(D);
        nb = div_up(D.ncells, KDP_BLOCK);
        k_dp_lang<<<nb, KDP_BLOCK, 0, st>>>(D, dt, epoch_off);
        if (D.quantum) k_quantum_tick<<<1, 32, 0, st>>>(D);
    } else {
        nb = div_up(D.natom, 256);
        k_dp_nve<<<nb, 256, 0, st>>>(D, dt);
    }
    k_rescale<<<1, 1024, 0, st>>>(D, nb);
    if (defer_scale) return;
    int na = div_up(D.natom, 256);
    if (temp) k_scale<true><<<na, 256, 0, st>>>(D);
    else k_scale<false><<<na, 256, 0, st>>>(D);
}

void launch_dr(const Dev& D, cudaStream_t st, double dt, bool scale) {
    if (scale) k_dr<true><<<div_up(D.natom, 256), 256, 0, st>>>(D, dt);
    else k_dr<false><<<div_up(D.natom, 256), 256, 0, st>>>(D, dt);
}

// sld_set_state on the device: the caller's r, p, s ([atom][3], caller order)
// to slot order, with the periodic wrap (periodic_CPU.cpp:31-50), |s| and the
// kinetic energy.  Products and sums are rounded one by one in the order the
// host expressions evaluate them, so the values are those of a plain C++ loop.
__device__ __forceinline__ double add3_rn(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(a, b), c);
}

__global__ void __launch_bounds__(256) k_load_state(Dev D, const double* __restrict__ r,
                                                    const double* __restrict__ p,
                                                    const double* __restrict__ s) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.natom) return;
    const size_t i = (size_t)D.id[k];
    double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
    const double* I = D.inv;
    const double* d = D.d;
    double qx = add3_rn(__dmul_rn(I[0], x), __dmul_rn(I[1], y), __dmul_rn(I[3], z));
    double qy = __dadd_rn(__dmul_rn(I[2], y), __dmul_rn(I[4], z));
    double qz = __dmul_rn(I[5], z);
    int idx = 0;
    if (qx < 0.0 || qx >= 1.0) { qx = __dsub_rn(qx, (double)(int)qx); ++idx; }
    if (qy < 0.0 || qy >= 1.0) { qy = __dsub_rn(qy, (double)(int)qy); ++idx; }
    if (qz < 0.0 || qz >= 1.0) { qz = __dsub_rn(qz, (double)(int)qz); ++idx; }
    if (idx > 0) {
        x = add3_rn(__dmul_rn(d[0], qx), __dmul_rn(d[1], qy), __dmul_rn(d[3], qz));
        y = __dadd_rn(__dmul_rn(d[2], qy), __dmul_rn(d[4], qz));
        z = __dmul_rn(d[5], qz);
    }
    D.r[k] = make_double4(x, y, z, 0.0);
    const double px = p[3 * i], py = p[3 * i + 1], pz = p[3 * i + 2];
    D.p[k] = make_double4(px, py, pz, 0.0);
    const double sx = s[3 * i], sy = s[3 * i + 1], sz = s[3 * i + 2];
    const double s0 = sqrt(add3_rn(__dmul_rn(sx, sx), __dmul_rn(sy, sy), __dmul_rn(sz, sz)));
    D.s[k] = make_double4(sx, sy, sz, s0);
    if (D.split) D.s32[k] = make_float4((float)sx, (float)sy, (float)sz, (float)s0);
    D.ke[k] = __ddiv_rn(__ddiv_rn(add3_rn(__dmul_rn(px, px), __dmul_rn(py, py),
                                          __dmul_rn(pz, pz)), 2.0), D.atmass);
}

void launch_load_state(const Dev& D, cudaStream_t st, const double* r, const double* p,
                       const double* s) {
    k_load_state<<<div_up(D.natom, 256), 256, 0, st>>>(D, r, p, s);
}

// ---------------------------------------------------------------------
// Box rescaling of the barostats (scale.cpp:31-44).  D carries the new box.
// Products and sums are rounded one by one, as the reference's expressions.

// scale_pressure_CPU.cpp:57-59: r = factor r
__global__ void __launch_bounds__(256) k_scale_positions(Dev D, double factor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double4 r = D.r[i];
    double x = __dmul_rn(factor, r.x), y = __dmul_rn(factor, r.y), z = __dmul_rn(factor, r.z);
    D.r[i] = make_double4(x, y, z, 0.0);
    const int4 q = cell_fix(D, D.cell_of[i], x, y, z);
    D.fxs[D.cell_slot[i]] = q;
    if (D.fxa) D.fxa[i] = q;
}

// scale_stress_CPU.cpp:66-80: fractional coordinates from the old inverse
// box, back to positions with the new box
struct InvBox { double v[6]; };
__global__ void __launch_bounds__(256) k_reshape_positions(Dev D, InvBox old) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.natom) return;
    double4 r = D.r[i];
    const double* I = old.v;
    const double* d = D.d;
    double qx = add3_rn(__dmul_rn(I[0], r.x), __dmul_rn(I[1], r.y), __dmul_rn(I[3], r.z));
    double qy = __dadd_rn(__dmul_rn(I[2], r.y), __dmul_rn(I[4], r.z));
    double qz = __dmul_rn(I[5], r.z);
    double x = add3_rn(__dmul_rn(d[0], qx), __dmul_rn(d[1], qy), __dmul_rn(d[3], qz));
    double y = __dadd_rn(__dmul_rn(d[2], qy), __dmul_rn(d[4], qz));
    double z = __dmul_rn(d[5], qz);
    D.r[i] = make_double4(x, y, z, 0.0);
    const int4 q = cell_fix(D, D.cell_of[i], x, y, z);
    D.fxs[D.cell_slot[i]] = q;
    if (D.fxa) D.fxa[i] = q;
}

void launch_scale_positions(const Dev& D, cudaStream_t st, double factor) {
    k_scale_positions<<<div_up(D.natom, 256), 256, 0, st>>>(D, factor);
}

void launch_reshape_positions(const Dev& D, cudaStream_t st, const double old_inv[6]) {
    InvBox b;
    for (int k = 0; k < 6; ++k) b.v[k] = old_inv[k];
    k_reshape_positions<<<div_up(D.natom, 256), 256, 0, st>>>(D, b);
}

// scale_step_CPU.cpp:39-73: the largest |p|^2 and |Heff_H|^2 over the atoms
__global__ void __launch_bounds__(256) k_max_partials(Dev D, double* part) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0, b = 0.0;
    if (i < D.natom) {
        double4 p = D.p[i], h = D.H[i];
        a = add3_rn(__dmul_rn(p.x, p.x), __dmul_rn(p.y, p.y), __dmul_rn(p.z, p.z));
        b = add3_rn(__dmul_rn(h.x, h.x), __dmul_rn(h.y, h.y), __dmul_rn(h.z, h.z));
    }
    __shared__ double sa[8], sb[8];
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { a = fmax(a, sa[k]); b = fmax(b, sb[k]); }
        part[2 * (size_t)blockIdx.x] = a;
        part[2 * (size_t)blockIdx.x + 1] = b;
    }
}

__global__ void __launch_bounds__(1024) k_max_final(const double* part, int nb, double* out) {
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a = fmax(a, part[2 * (size_t)k]);
        b = fmax(b, part[2 * (size_t)k + 1]);
    }
    __shared__ double sa[32], sb[32];
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { a = fmax(a, sa[k]); b = fmax(b, sb[k]); }
        out[0] = a;
        out[1] = b;
    }
}

// part: 2 doubles per 256 atoms; out: 2 doubles (max |p|^2, max |Heff_H|^2)
void launch_max_p_h(const Dev& D, cudaStream_t st, double* part, double* out) {
    int nb = div_up(D.natom, 256);
    k_max_partials<<<nb, 256, 0, st>>>(D, part);
    k_max_final<<<1, 1024, 0, st>>>(part, nb, out);
}
