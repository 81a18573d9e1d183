// Device state and helpers shared by the engine's kernels.
//
// Layout in HBM (one system; atoms stored in "slots" sorted by link cell at
// load time, the caller's atom index kept in `id`):
//   r, p, f, s, H, HL : double4 per atom (s.w = |s|, the reference's s0)
//   rho, pe, ke, me, me0, vir, sumJ : double per atom; stress: 6 per atom
//   cell_of, id, node : int per atom; stamp : int64 insertion key per atom
//   cell_start/count/atoms : CSR cell member lists in the reference's
//     linked-list order (head -> tail), rebuilt by links each step
//   Te ... Ges : double per Te cell (link cell, or a decoupled mesh node)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SLD_NINPUT 1000000
#define SLD_BOLTZ 8.617343e-5
#define SLD_HBAR 6.58211899e-16
#define SLD_EVTOJ 1.602176487e-19
#define SLD_MAXC 64   // == SLD_MAX_CELL_ATOMS in sld.h
#define SLD_MAXNB 48  // neighbours within rcut_max per atom (bcc Fe: 26)
#define SLD_MAXJ 32   // exchange neighbours within rcut_mag (bcc Fe: 14)
#define SLD_WRAP (1 << 30)
#define SLD_JMASK ((1 << 30) - 1)

// error flag bits in Ctl::err
#define SLD_FLAG_CAPACITY 1u
#define SLD_FLAG_TABLE 2u
#define SLD_FLAG_NAN 4u
#define SLD_FLAG_WAIT 8u         // a bounded device-side wait ran out

struct Ctl {
    unsigned long long epoch;     // Philox counter: one per noise-drawing sweep
    long long links_calls;        // stamps of relinked atoms
    long long steps;              // main-loop steps done
    unsigned int err;
    int pad;
    double initial_ave_energy;
    double total_time;
    double avep[3];
    double ke_factor;
    double virial;
    double avg[8];                // last energy averages
    // averages check_energy formed before its last renormalisation (pe, ke,
    // me, me0, Ee per atom) and the step it ran at, as step + 2 (0: none)
    double chk[5];
    long long chk_tag;
    long long qcount;             // kicks of the quantum thermostat so far
};

// data of the quintic that joins the ZBL core to the cubic knots of the
// DD05 pair term between 1.8 and 2.0 A (split form)
struct Pot32 {
    float zbl_y1, zbl_d1, zbl_c1, knot_y2, knot_d2, knot_c2;
    float zbl_as;   // ZBL screening length
};

// launch shapes chosen by sld_autotune (0: the built-in default)
struct Tune {
    int sweep_block;   // cells per block of the pipelined spin sweep (a thread a cell)
    int pair_block;    // atoms per block of the pair and list pass
    int force_block;   // atoms per block of the force passes
    int temp_block;    // atoms per block of the cell-temperature pass on a Te mesh
    int dte_mode;      // core_dTe kernel: 0 one CTA, 1 cluster, 2 hub by colour
                       // phases, 3 hub by levels; -1 default
    int dte_threads;   // threads per CTA of the hub core_dTe kernel
    int sweep_cap;     // CTAs per SM of a spin-sweep launch (0: one thread per cell),
                       // leaving room for the other graph branch's kernels
    int pair_cap;      // CTAs per SM of the pair/list pass (0: one thread per atom)
    int force_cap;     // CTAs per SM of the EAM force pass (0: one thread per atom)
    int graph_prio;    // 1: the step graph keeps its streams' priorities (the spin
                       // sweeps' branch first), 0: every node at the launch priority
};

struct Dev {
    // box (struct.h box_vector order: xx yx yy zx zy zz) and inverse
    double d[6], inv[6];
    double box_len[3], box_volume;
    double rcut_pot, rcut_mag, rcut_max, rcut_pot_sq, rcut_mag_sq, rcut_max_sq;
    double atmass, temperature, gamma_L, gamma_S_HL, step;
    double inv_r, inv_rho;
    double landau[4];             // A B C D (the reference's tables are constant)
    double kappa_e;
    int natom, nx, ny, nz, ncells;
    int tx, ty, tz, nte, te_mesh;
    unsigned seed;
    unsigned replica;             // second word of the Philox key
    int spinlang, lattlang, eltemp, localcolmot, renormalize, print_every;
    // the Hamiltonian (sld_hamiltonian) and what it has: lattice degrees of
    // freedom, spins, the Landau terms, the exchange correction of the Landau
    // field (SLDHL only), the Heisenberg Langevin scheme (SDH, SLDH)
    int ham, latt, spin, landau_on, hc, hint;
    double gamma_S_H;
    // quantum thermostat: the filter (qNf2 values), the coloured noise of each
    // atom, its update interval in kicks
    int quantum, qM, qNf2;
    const double* qH;
    double4* qnoise;
    int te_nloop;
    int small_grid;               // a link-cell axis of 3: every pair gets the minimum image
    Tune tune;
    int split;                    // 1: split-precision form (FP32 pair terms)
    int analytic;                 // 1: the split form's kernels in FP64
    Pot32 pot32;
    const float* cubic;           // piecewise-cubic pair and density coefficients
    const double* cubic64;        // the same in FP64 (analytic FP64 form)
    // tables (potential_CPU.cpp:61-157): F, F', f, f', phi, phi', J, J'
    const double *tF, *tdF, *tf, *tdf, *tphi, *tdphi, *tJ, *tdJ;
    // atoms
    double4 *r, *p, *f, *s, *H, *HL;
    double4* hext;                // external field per atom (eV), or null (extfield)
    double4* fext;                // external force per atom (eV/A), or null (extforce)
    float4* s32;                  // split form: s rounded to FP32, written with s by every
                                  // spin writer; the FP32 exchange sums gather it
    int4* fxs;                    // positions in fixed point, relative to the atom's link
                                  // cell: (fractional coordinate x n - cell index) x 2^29
                                  // per axis, in cell-list order (slot order); written by
                                  // links and by every drift (with the drift's unwrapped
                                  // position, so that an atom the drift wraps across the
                                  // box stays next to its cell until the next links)
    int4* fxa;                    // split form: the same in atom order
    unsigned char* nbk;           // split form: [SLD_MAXNB][natom] the neighbour cell
                                  // (0..26, map_cells order) of each nbr entry
    int* cell_slot;               // index of each atom in cell_atoms (its slot)
    float pair_loose;             // margin of the FP32 pair pre-test (A^2), k_pair.cu
                                  // (FP64 form; the split form's FP32 test is its own)
    double *rho, *pe, *ke, *me, *me0, *vir, *sumJ, *stress;
    int *cell_of, *id, *node;
    long long* stamp;
    // cells
    int *cell_start, *cell_count, *cell_atoms, *cell_fill, *scan_tmp;
    // Te cells
    double *Te, *Ee, *Tl, *TsR, *TsL, *Gel, *Ges, *acc;   // acc: 9 per Te cell
    double* trl;   // per Te cell: sum_R_up, sum_R_dn, sum_L_up, sum_L_dn
    int* te_count;
    const int *te_gcells, *te_gstart;
    const unsigned char* te_color;   // colour group of each Te cell
    int te_ngroups;
    // the diffusion sweep as levels of independent tasks, the cells named by
    // their position in te_gcells (position | 0x8000 for two updates in a
    // row), te_lstart[l]..te_lstart[l+1] for level l; te_lnb: per position,
    // the positions of the six face neighbours (+x -x +y -y +z -z, then two
    // zeros); 0 levels when the mesh is too large for them
    const unsigned short* te_ltasks;
    const int* te_lstart;
    const uint4* te_lnb;
    int te_nlevels;
    // per-step neighbour lists (built after every drift by k_pairs):
    //   nbr  [SLD_MAXNB][natom]  j | (1<<30 when the pair crosses the box)
    //        for r_ij < rcut_max, in the reference's traversal order; entry
    //        major, as its readers take atoms in storage order
    //   jl/jv [natom][SLD_MAXJ]  j and J(r_ij) for r_ij < rcut_mag; atom
    //        major, as the spin sweeps visit atoms of cells scattered over
    //        the box and each visit should read one contiguous row
    int *nbr, *nbr_n, *jl, *jl_n;
    double* jv;                   // FP64 form
    float* jvf;                   // split form
    unsigned char* jlk;           // split form: [natom][SLD_MAXJ] the neighbour cell
                                  // (0..26) of each exchange entry, as nbk
    double* dF;                   // F'(rho) per atom, refreshed after each rho pass
    double4* vrec;                // [natom][2 sweeps] visit records of one core_ds: rho and
                                  // the noise increment dS of the atom's visit in that sweep
    // The magnetic part of the forces, virial and stress, kept apart while
    // the EAM part is formed beside it (set in the spin-lattice step only,
    // null elsewhere): the magnetic pass writes them here instead of adding
    // them to f, vir and stress; the last kick adds fm to f for its own use,
    // and launch_fold_mag adds all three in
    double4* fm;
    double* virm;
    double* stressm;
    // control and reduction scratch
    Ctl* ctl;
    double* red;                  // partial sums
    int red_blocks;
};

// ---------------------------------------------------------------------
// geometry: periodic_CPU.cpp:31-50, find_image_CPU.cpp:31-53

__device__ __forceinline__ double3 to_frac(const Dev& D, double x, double y, double z) {
    return make_double3(D.inv[0] * x + D.inv[1] * y + D.inv[3] * z,
                        D.inv[2] * y + D.inv[4] * z, D.inv[5] * z);
}
__device__ __forceinline__ double3 to_cart(const Dev& D, double3 q) {
    return make_double3(D.d[0] * q.x + D.d[1] * q.y + D.d[3] * q.z,
                        D.d[2] * q.y + D.d[4] * q.z, D.d[5] * q.z);
}
// The reference truncates toward zero, so slightly negative fractional
// coordinates stay negative; kept as is.
__device__ __forceinline__ double3 periodic(const Dev& D, double3 r) {
    double3 q = to_frac(D, r.x, r.y, r.z);
    int idx = 0;
    if (q.x < 0.0 || q.x >= 1.0) { q.x -= (double)(int)q.x; ++idx; }
    if (q.y < 0.0 || q.y >= 1.0) { q.y -= (double)(int)q.y; ++idx; }
    if (q.z < 0.0 || q.z >= 1.0) { q.z -= (double)(int)q.z; ++idx; }
    return idx ? to_cart(D, q) : r;
}
__device__ __forceinline__ double3 find_image(const Dev& D, double3 rij) {
    double3 q = to_frac(D, rij.x, rij.y, rij.z);
    int idx = 0;
    if (q.x < -0.5) { q.x += 1.0; ++idx; }
    if (q.x >= 0.5) { q.x -= 1.0; ++idx; }
    if (q.y < -0.5) { q.y += 1.0; ++idx; }
    if (q.y >= 0.5) { q.y -= 1.0; ++idx; }
    if (q.z < -0.5) { q.z += 1.0; ++idx; }
    if (q.z >= 0.5) { q.z -= 1.0; ++idx; }
    return idx ? to_cart(D, q) : rij;
}

// The 26 neighbour cells in the order of map_cells.cpp:96-121 (offsets in
// x, y, z), then the cell itself.
static __constant__ signed char kNbr[27][3] = {
    {1, 0, 0},  {1, 1, 0},   {0, 1, 0},  {-1, 1, 0},  {1, 0, -1},  {1, 1, -1},  {0, 1, -1},
    {-1, 1, -1}, {1, 0, 1},  {1, 1, 1},  {0, 1, 1},   {-1, 1, 1},  {0, 0, 1},   {-1, 0, 0},
    {0, -1, 0}, {0, 0, -1},  {1, -1, 0}, {-1, -1, 0}, {-1, 0, 1},  {-1, 0, -1}, {0, -1, 1},
    {0, -1, -1}, {1, -1, 1}, {1, -1, -1}, {-1, -1, 1}, {-1, -1, -1}, {0, 0, 0}};

__device__ __forceinline__ int nbr_cell(const Dev& D, int cx, int cy, int cz, int k) {
    int x = cx + kNbr[k][0], y = cy + kNbr[k][1], z = cz + kNbr[k][2];
    x = x < 0 ? x + D.nx : (x >= D.nx ? x - D.nx : x);
    y = y < 0 ? y + D.ny : (y >= D.ny ? y - D.ny : y);
    z = z < 0 ? z + D.nz : (z >= D.nz ? z - D.nz : z);
    return x + (y + z * D.ny) * D.nx;
}
// the same, also telling whether the neighbour lies across the periodic
// boundary (only such pairs can need the minimum-image shift)
__device__ __forceinline__ int nbr_cell_w(const Dev& D, int cx, int cy, int cz, int k, bool& wrap) {
    int x = cx + kNbr[k][0], y = cy + kNbr[k][1], z = cz + kNbr[k][2];
    wrap = D.small_grid || x < 0 || x >= D.nx || y < 0 || y >= D.ny || z < 0 || z >= D.nz;
    x = x < 0 ? x + D.nx : (x >= D.nx ? x - D.nx : x);
    y = y < 0 ? y + D.ny : (y >= D.ny ? y - D.ny : y);
    z = z < 0 ? z + D.nz : (z >= D.nz ? z - D.nz : z);
    return x + (y + z * D.ny) * D.nx;
}
// the same, with the periodic image of the neighbour cell: s* = -1 / +1 when
// it lies across the low / high face of the box along that axis
__device__ __forceinline__ int nbr_cell_s(const Dev& D, int cx, int cy, int cz, int k, int& sx,
                                          int& sy, int& sz) {
    int x = cx + kNbr[k][0], y = cy + kNbr[k][1], z = cz + kNbr[k][2];
    sx = x < 0 ? -1 : (x >= D.nx ? 1 : 0);
    sy = y < 0 ? -1 : (y >= D.ny ? 1 : 0);
    sz = z < 0 ? -1 : (z >= D.nz ? 1 : 0);
    x -= sx * D.nx;
    y -= sy * D.ny;
    z -= sz * D.nz;
    return x + (y + z * D.ny) * D.nx;
}
// The atoms of link cell c that a kernel walks: at most SLD_MAXC.  A fuller
// cell (a system that has blown up, or an input far outside the reference's
// densities) has set SLD_FLAG_CAPACITY in links, so the step is reported as
// failed; the bound keeps every per-cell walk short in the meantime instead of
// letting one thread walk millions of atoms.
__device__ __forceinline__ int cell_n(const Dev& D, int c) {
    const int n = D.cell_count[c];
    return n < SLD_MAXC ? n : SLD_MAXC;
}

__device__ __forceinline__ void cell_xyz(const Dev& D, int c, int& cx, int& cy, int& cz) {
    cx = c % D.nx;
    int t = c / D.nx;
    cy = t % D.ny;
    cz = t / D.ny;
}

// Fixed-point positions relative to a link cell.  A component is the
// fractional coordinate times the cells per axis, less the cell's index
// (within [0, 1) for an atom inside its cell), in units of 2^-29, clamped to
// [-0.75, 1.75] (an atom never drifts that far between two links): the pair
// vector r_i - r_j of two atoms whose cells are k apart is
// M (f_i - f_j - delta_k 2^29), exact in integers, with one rounding to FP32
// per product of the cell matrix M (the box vectors over the cells per axis
// and 2^29).
#define SLD_FX_ONE (1 << 29)
// kNbr[k] * SLD_FX_ONE (k = 0..26) into a block's shared table: a pass over
// list entries takes a different neighbour cell k in every lane, and constant
// memory serves the lanes' distinct addresses one at a time.  Every thread of
// the block must call it (it ends with a barrier).
__device__ __forceinline__ void fx_offsets_load(int4* koff) {
    if (threadIdx.x < 27)
        koff[threadIdx.x] = make_int4(kNbr[threadIdx.x][0] * SLD_FX_ONE,
                                      kNbr[threadIdx.x][1] * SLD_FX_ONE,
                                      kNbr[threadIdx.x][2] * SLD_FX_ONE, 0);
    __syncthreads();
}

__device__ __forceinline__ int4 cell_fix(const Dev& D, int c, double x, double y, double z) {
    int cx, cy, cz;
    cell_xyz(D, c, cx, cy, cz);
    const double3 q = to_frac(D, x, y, z);
    auto f = [](double v) {
        v = fmin(fmax(v, -0.75), 1.75);
        return __double2int_rn(v * (double)SLD_FX_ONE);
    };
    return make_int4(f(q.x * D.nx - cx), f(q.y * D.ny - cy), f(q.z * D.nz - cz), 0);
}
struct FxMat {
    float xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ FxMat fx_mat(const Dev& D) {
    const double u = 1.0 / SLD_FX_ONE;
    return FxMat{(float)(D.d[0] / D.nx * u), (float)(D.d[1] / D.ny * u), (float)(D.d[3] / D.nz * u),
                 (float)(D.d[2] / D.ny * u), (float)(D.d[4] / D.nz * u), (float)(D.d[5] / D.nz * u)};
}
// the Cartesian vector (FP32) of a fixed-point difference; ORTHO: a box whose
// off-diagonal components are zero (the same values: fmaf(0, y, x) is x)
template <bool ORTHO = false>
__device__ __forceinline__ float3 fx_vec(const FxMat& M, int dx, int dy, int dz) {
    const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
    if constexpr (ORTHO) return make_float3(M.xx * fx, M.yy * fy, M.zz * fz);
    return make_float3(fmaf(M.xz, fz, fmaf(M.xy, fy, M.xx * fx)), fmaf(M.yz, fz, M.yy * fy),
                       M.zz * fz);
}
__host__ __device__ inline bool box_ortho(const Dev& D) {
    return D.d[1] == 0.0 && D.d[3] == 0.0 && D.d[4] == 0.0;
}

// potential_CPU.cpp:172-179: linear interpolation between entries n-1 and n
// of a 10^6-point table at x_n = (n+1) max / 10^6.  Out-of-range indices are
// clamped and flagged (the reference reads out of bounds).
__device__ __forceinline__ double interp(const double* __restrict__ t, double x, double inv,
                                         unsigned* err) {
    double fn = x * inv;
    int n = (int)fn;
    if (n < 1 || n >= SLD_NINPUT) {
        atomicOr(err, SLD_FLAG_TABLE);
        n = n < 1 ? 1 : SLD_NINPUT - 1;
    }
    double ratio = (double)(n + 1) - fn;
    return __ldg(t + n - 1) * ratio + __ldg(t + n) * (1.0 - ratio);
}
// the same for a table whose every entry is c
__device__ __forceinline__ double interp_const(double c, double x, double inv) {
    double fn = x * inv;
    int n = (int)fn;
    double ratio = (double)(n + 1) - fn;
    return c * ratio + c * (1.0 - ratio);
}

// ---------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Counter (atom id,
// epoch lo, epoch hi, tag), key (seed, replica).  One call gives 4 uniforms
// u = (x + 0.5) 2^-32 and two Box-Muller pairs; three normals are used.

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ double3 normals3(unsigned seed, unsigned replica, unsigned atom,
                                            unsigned long long epoch) {
    uint32_t c[4] = {atom, (uint32_t)epoch, (uint32_t)(epoch >> 32), 0x53504e53u};
    philox4x32_10(c, seed, replica);
    const double s = 2.3283064365386963e-10;
    double u0 = ((double)c[0] + 0.5) * s, u1 = ((double)c[1] + 0.5) * s;
    double u2 = ((double)c[2] + 0.5) * s, u3 = ((double)c[3] + 0.5) * s;
    double ra = sqrt(-2.0 * log(u0)), rb = sqrt(-2.0 * log(u2));
    double sa, ca, sb, cb;
    sincos(6.283185307179586 * u1, &sa, &ca);
    sincos(6.283185307179586 * u3, &sb, &cb);
    (void)sb;
    return make_double3(ra * ca, ra * sa, rb * cb);
}

// The same three normals from the same counter, with the Box-Muller transform
// in FP32 (the split form's thermostats).  The uniforms are (k + 1/2) 2^-32
// rounded to FP32, which keeps their relative precision (2^-24) down to the
// smallest, so each normal differs from the FP64 transform's by about 1e-7
// relative, in the tails too.  The noise is a stochastic force and field;
// what the split form keeps in FP64 is the integration it enters.
__device__ __forceinline__ double3 normals3_f32(unsigned seed, unsigned replica, unsigned atom,
                                                unsigned long long epoch) {
    uint32_t c[4] = {atom, (uint32_t)epoch, (uint32_t)(epoch >> 32), 0x53504e53u};
    philox4x32_10(c, seed, replica);
    const float s = 2.3283064365386963e-10f;   // 2^-32; u <= 1, so -2 log u >= 0
    const float u0 = ((float)c[0] + 0.5f) * s, u1 = ((float)c[1] + 0.5f) * s;
    const float u2 = ((float)c[2] + 0.5f) * s, u3 = ((float)c[3] + 0.5f) * s;
    const float ra = sqrtf(-2.f * logf(u0)), rb = sqrtf(-2.f * logf(u2));
    float sa, ca;
    sincospif(2.f * u1, &sa, &ca);
    const float cb = cospif(2.f * u3);
    return make_double3((double)(ra * ca), (double)(ra * sa), (double)(rb * cb));
}

// ---------------------------------------------------------------------
// heat capacity of the electrons: heatcapacity_CPU.cpp:34-57
__device__ __forceinline__ double te_Ce(double Te) {
    const double a = 3.0, b = 2e-4 / SLD_BOLTZ;
    return a * tanh(b * Te);
}
__device__ __forceinline__ double te_to_Ee(double Te) {
    const double a = 3.0, b = 2e-4 / SLD_BOLTZ;
    return a / b * log(cosh(b * Te));
}
__device__ __forceinline__ double Ee_to_te(double Ee) {
    const double a = 3.0, b = 2e-4 / SLD_BOLTZ;
    return acosh(exp(b / a * Ee)) / b;
}

// ---------------------------------------------------------------------
// reductions (deterministic: fixed shuffle tree, fixed block order)
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// sums v over the block; result valid in thread 0.  `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        t = lane < nw ? sh[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

// block_sum for a caller that has passed a block-wide barrier since the last
// read of `sh`
__device__ __forceinline__ double block_sum_after_barrier(double v, double* sh) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        t = lane < nw ? sh[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

static inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

// 32-byte global accesses: one instruction on sm_100 where a double4 or two
// 16-byte vectors take two, so a warp's scattered rows and spins cost half
// the load requests.  The address must be 32-byte aligned.  ld32_d4 and
// st32_d4 are coherent and volatile (kept in program order with each other),
// for spins that a thread reads after writing them; ld32cg_d4 reads through
// L2 only, for spins other blocks write during the kernel.  The *_once
// variants below are for streamed data; ldg32_*_once read data no thread
// writes during the kernel (the non-coherent path).
__device__ __forceinline__ double4 ld32_d4(const double4* p) {
    double4 v;
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ double4 ld32cg_d4(const double4* p) {
    double4 v;
    asm volatile("ld.global.cg.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ void st32_d4(double4* p, double4 v) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
                 :: "l"(p), "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w) : "memory");
}

// Streamed data: a sweep reads each visit's row, couplings and record once,
// while the neighbour spins it gathers (the FP32 copy: 16 B per atom) are read
// by many visits.  The *_once accesses take L2's evict-first priority and skip
// L1, so that the streamed bytes leave the caches before the gathered spins.
__device__ __forceinline__ void ldg32_i8_once(const int* p, int4& a, int4& b) {
    asm("ld.global.nc.L1::no_allocate.L2::evict_first.v8.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
}
__device__ __forceinline__ void ldg32_f8_once(const float* p, float4& a, float4& b) {
    asm("ld.global.nc.L1::no_allocate.L2::evict_first.v8.f32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}
__device__ __forceinline__ double4 ldg32_d4_once(const void* p) {
    double4 v;
    asm("ld.global.nc.L1::no_allocate.L2::evict_first.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ double4 ld32_d4_once(const double4* p) {
    double4 v;
    asm volatile("ld.global.L1::no_allocate.L2::evict_first.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ void st32_d4_once(double4* p, double4 v) {
    asm volatile("st.global.L1::no_allocate.L2::evict_first.v4.f64 [%0], {%1, %2, %3, %4};"
                 :: "l"(p), "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w) : "memory");
}

// One exchange term of H = sum_j J s_j and sum_j J |s_j|, with every product
// and sum rounded on its own (no fused multiply-add): the FP64 form then adds
// exactly as the reference's separate multiply and add do, and every kernel
// that sums the same list gets the same bits whatever its control flow (the
// compiler fuses a multiply into an add only within one basic block).
__device__ __forceinline__ void exch_add64(double& hx, double& hy, double& hz, double& hj,
                                           double J, const double4& s) {
    hx = __dadd_rn(hx, __dmul_rn(J, s.x));
    hy = __dadd_rn(hy, __dmul_rn(J, s.y));
    hz = __dadd_rn(hz, __dmul_rn(J, s.z));
    hj = __dadd_rn(hj, __dmul_rn(J, s.w));
}
// the same in FP32 with Kahan compensation (split form)
__device__ __forceinline__ void exch_add32(float ks[4], float kc[4], float J, const float4& s) {
    const float w[4] = {__fmul_rn(J, s.x), __fmul_rn(J, s.y), __fmul_rn(J, s.z),
                        __fmul_rn(J, s.w)};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float y = __fsub_rn(w[q], kc[q]);
        float t = __fadd_rn(ks[q], y);
        kc[q] = __fsub_rn(__fsub_rn(t, ks[q]), y);
        ks[q] = t;
    }
}

// Exchange field of atom i from its J list: H = sum J_ij s_j and
// sumJ = sum J_ij |s_j| in list order.  The list is read in batches of 8
// (indices and J first, then the 8 spins) so that a batch costs two memory
// latencies instead of two per neighbour; the additions stay in list order.
// Entries whose neighbour satisfies skip(j) are left out (and reported to
// on_skip(j, J)).  FP64 form: FP64 products and sums; split form: FP32
// products with compensated FP32 sums.
#define SLD_GB 8
// The same terms taken only when `on`: computed unconditionally and kept by
// selects, so an unrolled sum over a fixed number of slots needs no branch
// per slot (the kept values are those of the plain sum).
__device__ __forceinline__ void exch_add64_if(bool on, double& hx, double& hy, double& hz,
                                              double& hj, double J, const double4& s) {
    const double ax = __dadd_rn(hx, __dmul_rn(J, s.x));
    const double ay = __dadd_rn(hy, __dmul_rn(J, s.y));
    const double az = __dadd_rn(hz, __dmul_rn(J, s.z));
    const double aj = __dadd_rn(hj, __dmul_rn(J, s.w));
    hx = on ? ax : hx;
    hy = on ? ay : hy;
    hz = on ? az : hz;
    hj = on ? aj : hj;
}
__device__ __forceinline__ void exch_add32_if(bool on, float ks[4], float kc[4], float J,
                                              const float4& s) {
    const float w[4] = {__fmul_rn(J, s.x), __fmul_rn(J, s.y), __fmul_rn(J, s.z),
                        __fmul_rn(J, s.w)};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float y = __fsub_rn(w[q], kc[q]);
        const float t = __fadd_rn(ks[q], y);
        const float c = __fsub_rn(__fsub_rn(t, ks[q]), y);
        ks[q] = on ? t : ks[q];
        kc[q] = on ? c : kc[q];
    }
}

template <class Skip, class OnSkip>
__device__ __forceinline__ void exchange_field(const Dev& D, int i, double3& H, double& sumJ,
                                               Skip skip, OnSkip on_skip) {
    const int nj = D.jl_n[i];
    double hx = 0, hy = 0, hz = 0, hj = 0;
    // the reference starts the field at the external one (calculate_spin_CPU.cpp:35-40)
    if (D.hext && !D.split) {
        double4 h = D.hext[i];
        hx = h.x; hy = h.y; hz = h.z;
    }
    float ks[4] = {0, 0, 0, 0}, kc[4] = {0, 0, 0, 0};   // Kahan sums (split form)
    for (int e0 = 0; e0 < nj; e0 += SLD_GB) {
        int jj[SLD_GB];
        double Jv[SLD_GB];
#pragma unroll
        for (int u = 0; u < SLD_GB; ++u) {
            int e = e0 + u;
            size_t at = (size_t)i * SLD_MAXJ + e;
            jj[u] = e < nj ? D.jl[at] : -1;
            Jv[u] = e < nj ? (D.split ? (double)D.jvf[at] : D.jv[at])
                           : 0.0;
        }
        if (!D.split) {
            double4 sj[SLD_GB];
#pragma unroll
            for (int u = 0; u < SLD_GB; ++u)
                sj[u] = jj[u] >= 0 ? D.s[jj[u]] : make_double4(0, 0, 0, 0);
#pragma unroll
            for (int u = 0; u < SLD_GB; ++u) {
                if (jj[u] < 0) continue;
                if (skip(jj[u])) {
                    on_skip(jj[u], Jv[u]);
                    continue;
                }
                exch_add64(hx, hy, hz, hj, Jv[u], sj[u]);
            }
        } else {
            // the FP32 copy of the spins: the values the FP32 sums use
            float4 sj[SLD_GB];
#pragma unroll
            for (int u = 0; u < SLD_GB; ++u)
                sj[u] = jj[u] >= 0 ? D.s32[jj[u]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int u = 0; u < SLD_GB; ++u) {
                if (jj[u] < 0) continue;
                if (skip(jj[u])) {
                    on_skip(jj[u], Jv[u]);
                    continue;
                }
                exch_add32(ks, kc, (float)Jv[u], sj[u]);
            }
        }
    }
    if (D.split) {
        hx = (double)ks[0] - (double)kc[0];
        hy = (double)ks[1] - (double)kc[1];
        hz = (double)ks[2] - (double)kc[2];
        hj = (double)ks[3] - (double)kc[3];
        if (D.hext) {   // the external field added in FP64
            double4 h = D.hext[i];
            hx = h.x + hx; hy = h.y + hy; hz = h.z + hz;
        }
    }
    H = make_double3(hx, hy, hz);
    sumJ = hj;
}

// The per-atom spin terms of calculate_temperature
// (calculate_temperature_CPU.cpp:72-114) from the atom's exchange field H and
// sum_j J |s_j|: R_up = |s x H|^2, R_dn = s.H and, for the Heisenberg-Landau
// Hamiltonians, L_up and L_dn of the Landau field; writes H, HL and sum J.
__device__ __forceinline__ void temp_spin_terms(const Dev& D, int i, double3 H, double sumJ,
                                                double& Rup, double& Rdn, double& Lup,
                                                double& Ldn) {
    Lup = Ldn = 0.0;
    double4 s4 = D.s[i];
    double3 s = make_double3(s4.x, s4.y, s4.z);
    double cx_ = s.y * H.z - H.y * s.z, cy_ = s.z * H.x - H.z * s.x, cz_ = s.x * H.y - H.x * s.y;
    Rup = cx_ * cx_ + cy_ * cy_ + cz_ * cz_;
    Rdn = s.x * H.x + s.y * H.y + s.z * H.z;
    D.H[i] = make_double4(H.x, H.y, H.z, 0.0);
    if (!D.landau_on) return;   // the Heisenberg Hamiltonians: no Landau field
    if (!D.hc) sumJ = 0.0;      // the exchange correction is SLDHL's
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
    D.HL[i] = make_double4(HL.x, HL.y, HL.z, 0.0);
    if (D.hc) D.sumJ[i] = sumJ;
}

// Adds v[0..NV) into the Te-node accumulators acc[9 node + at + q].  Atoms
// are stored cell by cell, so neighbouring lanes mostly share a node: a
// segmented warp scan (segments = runs of equal node, marked by head flags)
// sums each run, and the run's last lane does the atomics.  The calling
// lanes must be a prefix of the warp (lanes past natom have returned).
template <int NV>
__device__ __forceinline__ void node_add(const Dev& D, int node, double (&v)[NV], int at) {
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    int prev = __shfl_up_sync(act, node, 1);
    int head = (lane == 0 || prev != node) ? 1 : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int th = __shfl_up_sync(act, head, o);
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) t[q] = __shfl_up_sync(act, v[q], o);
        if (lane >= o) {
            if (!head) {
#pragma unroll
                for (int q = 0; q < NV; ++q) v[q] += t[q];
            }
            head |= th;
        }
    }
    int nxt = __shfl_down_sync(act, node, 1);
    bool last = lane == 31 || !((act >> (lane + 1)) & 1u) || nxt != node;
    if (last) {
        double* acc = D.acc + 9 * (size_t)node + at;
#pragma unroll
        for (int q = 0; q < NV; ++q) atomicAdd(acc + q, v[q]);
    }
}

// ---------------------------------------------------------------------
// launch wrappers (host), one file per kernel family
void launch_links(const Dev& D, cudaStream_t st, bool initial, int scan_blocks);
void launch_pairs(const Dev& D, cudaStream_t st, bool write_rho);
void sweep_init();
void launch_force(const Dev& D, cudaStream_t st);
void launch_embed(const Dev& D, cudaStream_t st);
void launch_force_eam(const Dev& D, cudaStream_t st);   // lattice terms (no spins)
void launch_force_mag(const Dev& D, cudaStream_t st, bool temp);   // adds the magnetic terms
void launch_fold_mag(const Dev& D, cudaStream_t st);   // f, vir, stress += fm, virm, stressm
void launch_sweep(const Dev& D, cudaStream_t st, const int* gcells, int ncell_g, double dt,
                  bool backward, bool fields);
void launch_spin_noise(const Dev& D, cudaStream_t st, int epoch_off, double dt);
void launch_load_state(const Dev& D, cudaStream_t st, const double* r, const double* p,
                       const double* s);
// data-flow schedule of both sweeps of one core_ds call (k_spin.cu)
struct SweepFlow {
    const int4* tasks;                // (backward, first, count, group), sweep order
    int ntasks;
    const int* gcells;                // cells by colour group
    const unsigned char* cell_group;  // colour group of each link cell
    int* cell_flag;                   // tag of each cell's last finished sweep
    int* sync;                        // [0] tag base of the next call, [1] next task
    int polls;                        // bound on the polls of one cell's waits
    int stall;                        // added to every tag a wait needs (0; a test
                                      // sets it to make the waits run out)
};
bool sweep_uses_flow();
void launch_sweep_flow(const Dev& D, cudaStream_t st, const SweepFlow& F, double dt,
                       bool fields);
// temp: the last kick of a step whose calculate_temperature is split over the
// magnetic force pass and this kick (launch_force_mag)
// defer_scale: leave rescale_momentum's scaling of the momenta to the next
// drift (launch_dr with scale), for a step in which nothing reads them before
void launch_dp(const Dev& D, cudaStream_t st, double dt, int epoch_off, bool temp = false,
               bool defer_scale = false);
// the quantum thermostat's normals: Philox epoch SLD_QEPOCH + t, t >= -Nf2 the
// index of the draw in each atom's history
#define SLD_QEPOCH (1ULL << 62)
void launch_dr(const Dev& D, cudaStream_t st, double dt, bool scale = false);
// barostat position rescaling (D holds the new box) and the adaptive time
// step's maxima (k_lattice.cu)
void launch_scale_positions(const Dev& D, cudaStream_t st, double factor);
void launch_reshape_positions(const Dev& D, cudaStream_t st, const double old_inv[6]);
void launch_max_p_h(const Dev& D, cudaStream_t st, double* part, double* out);
void launch_temperature(const Dev& D, cudaStream_t st);
// calculate_temperature on a Te mesh in three parts: zero the node sums; the
// per-atom terms (launch_force_mag and launch_dp with temp); the nodes
void launch_temperature_begin(const Dev& D, cudaStream_t st);
void launch_temperature_end(const Dev& D, cudaStream_t st);
void launch_dte(const Dev& D, cudaStream_t st, double dt);
int dte_init(int device);
void launch_energy_check(const Dev& D, cudaStream_t st, int mode);
void launch_advance(const Dev& D, cudaStream_t st, int epochs, int steps);
void launch_averages(const Dev& D, cudaStream_t st, double* out_dev);
void launch_virial(const Dev& D, cudaStream_t st);
// slots of the check() sums (launch_check_sums): per-atom sums first
enum {
    SLD_CHK_PE, SLD_CHK_KE, SLD_CHK_ME, SLD_CHK_ME0, SLD_CHK_SX, SLD_CHK_SY, SLD_CHK_SZ,
    SLD_CHK_VIR, SLD_CHK_STRESS,                       // 6: 11 22 33 12 23 31
    SLD_CHK_RUP = SLD_CHK_STRESS + 6, SLD_CHK_RDN, SLD_CHK_LUP, SLD_CHK_LDN,
    SLD_CHK_ATOM,                                      // per-atom sums end here
    SLD_CHK_TE = SLD_CHK_ATOM, SLD_CHK_EE, SLD_CHK_N
};
void launch_check_sums(const Dev& D, cudaStream_t st, double* part, double* out);
