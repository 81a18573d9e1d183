/*
 * Test infrastructure only (the checker, never the product).
 *
 * Plain C restatement of the reference CPU step of SPILADY 1.0 built with
 * -DSLDHL, for one system on one thread.  Each function names the reference
 * code it follows (file:line in the reference tree).  The arithmetic keeps
 * the reference's operation order so that, with the reference's own random
 * number stream (ORC_RNG_MWC) and one OpenMP thread, results agree with the
 * reference binary (oracle/_ref) to the last bits; tests/test_oracle_pin.py
 * checks that.  The runtime switches stand for the reference's control.h
 * #defines (spinlang, lattlang, eltemp, localcolmot, renormalizeEnergy).
 *
 * Additions that have no reference counterpart, marked where they occur:
 *   - ORC_RNG_PHILOX: the CUDA engine's counter-based noise, so that Langevin
 *     runs of the engine can be compared with this code number for number;
 *   - te_mesh > 0: electron temperature on an n^3 mesh decoupled from the
 *     link cells (the reference keeps Te per link cell, map_cells.cpp:128).
 */
#include "sld_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BOLTZ 8.617343e-5                       /* spilady.h:54 */
#define C_LIGHT 299792458e0
#define UTOEV (931.494028e6 / C_LIGHT / C_LIGHT)
#define LENGTH_SCALE 1e-10
#define HBAR 6.58211899e-16
#define PI_NUM 3.141592653589793238462e0            /* spilady.h:61 */
#define EVTOJ 1.602176487e-19
#define NINPUT 1000000                          /* global.h:67 */

typedef struct { double x, y, z; } v3;

/* vec_utils_CPU.cpp:31-133 */
static v3 vinit(double x, double y, double z) { v3 c = {x, y, z}; return c; }
static v3 vzero(void) { return vinit(0e0, 0e0, 0e0); }
static v3 vadd(v3 a, v3 b) { return vinit(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return vinit(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vmul(double a, v3 b) { return vinit(a * b.x, a * b.y, a * b.z); }
static v3 vdiv(v3 a, double b) { return vinit(a.x / b, a.y / b, a.z / b); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double vsq(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static double vlen(v3 a) { return sqrt(vsq(a)); }
static v3 vcross(v3 a, v3 b) {
    return vinit(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

static v3 ld(const double* a, int i) { return vinit(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static void st(double* a, int i, v3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

/* ------------------------------------------------------------------ */
/* Potential: DD05 EAM for Fe and the Fe exchange / Landau terms.      */
/* Functional forms and published constants as DD05.cpp:6-164 and     */
/* JijFe.cpp:5-43 define them.                                         */

static double emb_F(double rho) {                 /* DD05.cpp:6-18 */
    const double a = 4.100199340884814, b = 1.565647547483517;
    double F = 0e0;
    if (rho >= 1e0) F = -a * sqrt(rho);
    else F = -a * sqrt(rho) - b / log(2e0) * (1e0 - sqrt(rho)) * log(2e0 - rho);
    return F;
}

static double dens_f(double r) {                  /* DD05.cpp:20-43 */
    static const double a[6] = {0.9332056681088162, -1.162558782567700,
                                -0.3502026949249225, 0.4287820835430028,
                                4.907925057809273, -5.307049068415304};
    static const double k[6] = {3.0, 2.8666666666666666, 2.7333333333333333,
                                2.6, 2.4, 2.3};
    double f = 0e0;
    for (int i = 0; i < 6; ++i)
        if (r < k[i]) f += a[i] * pow(k[i] - r, 3);
    return f;
}

static double zbl(double r) {                     /* DD05.cpp:45-62 */
    const double z = 26e0, abohr = 0.52917720859e0;
    double as = 0.88535e0 * abohr / (2e0 * pow(z, 0.23));
    double x = r / as;
    double v = 0.1818e0 * exp(-3.2 * x) + 0.5099e0 * exp(-0.9423 * x) +
               0.2802e0 * exp(-0.4029 * x) + 0.02817e0 * exp(-0.2016 * x);
    return z * z * 14.3992 * v / r;
}

static const double PV[8] = {-0.1960674387419232, 0.3687525935422963,
                             -1.505333614924853, 4.948907078156191,
                             -4.894613262753399, 3.468897724782442,
                             -1.792218099820337, 80.22069592246987};
static const double PK[8] = {4.1, 3.8, 3.5, 3.2, 2.9, 2.6, 2.4, 2.3};

static double pair_knots(double r, int deriv) {
    double v = 0e0;
    for (int i = 0; i < 8; ++i) {
        if (r < PK[i]) {
            double u = PK[i] - r;
            if (deriv == 0) v += PV[i] * pow(u, 3);
            else if (deriv == 1) v -= 3e0 * PV[i] * u * u;
            else v += 6e0 * PV[i] * u;
        }
    }
    return v;
}

/* Pair term (DD05.cpp:64-164): ZBL below 1.8 A, the knot cubics above
   2.0 A, and between them the quintic that matches value, slope and
   curvature at both ends.  The quintic is written here in Hermite form; it
   is the same polynomial as the reference's monomial coefficients. */
static double pair_phi(double r) {
    const double x1 = 1.8, x2 = 2.0;
    if (r <= x1) return zbl(r);
    if (r <= x2) {
        double h = 1e-7;
        double y1 = zbl(x1);
        double d1 = (zbl(x1 + h) - zbl(x1 - h)) / 2e-7;
        double c1 = (zbl(x1 + h) + zbl(x1 - h) - 2e0 * zbl(x1)) / pow(h, 2);
        double y2 = pair_knots(x2, 0), d2 = pair_knots(x2, 1), c2 = pair_knots(x2, 2);
        double w = x2 - x1, t = (r - x1) / w;
        double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
        double h00 = 1 - 10 * t3 + 15 * t4 - 6 * t5, h01 = 10 * t3 - 15 * t4 + 6 * t5;
        double h10 = t - 6 * t3 + 8 * t4 - 3 * t5, h11 = -4 * t3 + 7 * t4 - 3 * t5;
        double h20 = 0.5 * t2 - 1.5 * t3 + 1.5 * t4 - 0.5 * t5;
        double h21 = 0.5 * t3 - t4 + 0.5 * t5;
        return h00 * y1 + h01 * y2 + w * (h10 * d1 + h11 * d2) +
               w * w * (h20 * c1 + h21 * c2);
    }
    return pair_knots(r, 0);
}

static double exch_J(double r) {                  /* JijFe.cpp:5-14 */
    const double A = 0.870, rc = 3.75;
    double J = 0e0;
    if (r < rc) J = A * pow(1.0 - r / rc, 3);
    return J;
}
static double landau_A(double rho) { (void)rho; return -0.744824; }   /* JijFe.cpp:18-43 */
static double landau_B(double rho) { (void)rho; return 0.345295; }
static double landau_C(double rho) { (void)rho; return -0.00790205; }
static double landau_D(double rho) { (void)rho; return 0e0; }

/* potential_CPU.cpp:159-170: seven-point central difference, dx = x/1000 */
static double deriv7(double (*fn)(double), double x) {
    double dx = x / 1000e0;
    double p1 = fn(x + dx), m1 = fn(x - dx);
    double p2 = fn(x + 2 * dx), m2 = fn(x - 2 * dx);
    double p3 = fn(x + 3 * dx), m3 = fn(x - 3 * dx);
    return (45e0 * (p1 - m1) - 9e0 * (p2 - m2) + (p3 - m3)) / (60e0 * dx);
}

enum { T_F, T_dF, T_f, T_df, T_phi, T_dphi, T_J, T_dJ, T_LA, T_LB, T_LC, T_LD,
       T_dLA, T_dLB, T_dLC, T_dLD, T_COUNT };

typedef struct {
    double* t[T_COUNT];
    double inv_r, inv_rho;   /* finput/rmax, finput/rhomax */
} tables;

/* potential_CPU.cpp:61-157 */
static void build_tables(tables* T, double rmax) {
    double rhomax = 2e0 * dens_f(1e0);
    if (rhomax < 1000e0) rhomax = 1000e0;
    double finput = (double)NINPUT;
    T->inv_r = finput / rmax;
    T->inv_rho = finput / rhomax;
    for (int k = 0; k < T_COUNT; ++k) T->t[k] = (double*)malloc(sizeof(double) * NINPUT);
    for (int n = 0; n < NINPUT; ++n) {
        double r = rmax / (double)NINPUT * (double)(n + 1);
        double rho = rhomax / (double)NINPUT * (double)(n + 1);
        T->t[T_F][n] = emb_F(rho);
        T->t[T_dF][n] = deriv7(emb_F, rho);
        T->t[T_f][n] = dens_f(r);
        T->t[T_df][n] = deriv7(dens_f, r);
        T->t[T_phi][n] = pair_phi(r);
        T->t[T_dphi][n] = deriv7(pair_phi, r);
        T->t[T_J][n] = exch_J(r);
        T->t[T_dJ][n] = deriv7(exch_J, r);
        T->t[T_LA][n] = landau_A(rho);
        T->t[T_LB][n] = landau_B(rho);
        T->t[T_LC][n] = landau_C(rho);
        T->t[T_LD][n] = landau_D(rho);
        T->t[T_dLA][n] = deriv7(landau_A, rho);
        T->t[T_dLB][n] = deriv7(landau_B, rho);
        T->t[T_dLC][n] = deriv7(landau_C, rho);
        T->t[T_dLD][n] = deriv7(landau_D, rho);
    }
}

/* potential_CPU.cpp:172-179: linear interpolation between entries n-1, n */
static double interp(double x, double inv, const double* t) {
    double fn = x * inv;
    int n = (int)fn;
    double ratio = (double)(n + 1) - fn;
    return t[n - 1] * ratio + t[n] * (1e0 - ratio);
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the engine's      */
/* noise source; no reference counterpart.                             */

static void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_philox4x32(const unsigned* ctr, const unsigned* key, unsigned* out) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]}, k[2] = {key[0], key[1]}, o[4];
    philox4x32_10(c, k, o);
    for (int i = 0; i < 4; ++i) out[i] = o[i];
}

/* Three standard normals for (seed, replica, atom, epoch): one Philox call,
   four 32-bit uniforms u = (x + 0.5) 2^-32, two Box-Muller pairs, the fourth
   normal unused. */
void orc_philox_normals(unsigned seed, unsigned replica, unsigned atom,
                        unsigned long long epoch, double* out3) {
    uint32_t ctr[4] = {atom, (uint32_t)epoch, (uint32_t)(epoch >> 32), 0x53504e53u};
    uint32_t key[2] = {seed, replica};
    uint32_t x[4];
    philox4x32_10(ctr, key, x);
    const double s = 2.3283064365386963e-10;   /* 2^-32 */
    double u0 = ((double)x[0] + 0.5) * s, u1 = ((double)x[1] + 0.5) * s;
    double u2 = ((double)x[2] + 0.5) * s, u3 = ((double)x[3] + 0.5) * s;
    double ra = sqrt(-2e0 * log(u0)), ta = 6.283185307179586 * u1;
    double rb = sqrt(-2e0 * log(u2)), tb = 6.283185307179586 * u3;
    out3[0] = ra * cos(ta);
    out3[1] = ra * sin(ta);
    out3[2] = rb * cos(tb);
}

/* ------------------------------------------------------------------ */

struct orc_sys {
    orc_params P;
    int n;
    double d[6], inv[6];         /* xx yx yy zx zy zz */
    double box_len[3], box_volume;
    double atmass, temperature, gamma_L, gamma_S_HL;
    double rcut_pot, rcut_mag, rcut_max;
    double rcut_pot_sq, rcut_mag_sq, rcut_max_sq, min_len;
    tables T;
    int dLandau_zero;
    /* atoms */
    double *r, *p, *f, *s, *s0, *H, *HL, *HC, *rho, *pe, *ke, *me, *me0, *vir, *stress,
        *sumJ, *lv;
    int *cell, *old_cell, *next, *prev, *node;
    /* link cells */
    int nx, ny, nz, ncells;
    int *head, *tail, *count, *neigh;
    int ngroups, *gstart, *gcells;
    double* ave_ff;              /* localcolmot noise mean per link cell */
    /* Te cells (link cells, or the decoupled mesh) */
    int tx, ty, tz, nte;
    int *te_neigh, te_ngroups, *te_gstart, *te_gcells, *te_count;
    double *Te, *Ee, *Tl, *TsR, *TsL, *Gel, *Ges, *sRup, *sRdn, *sLup, *sLdn, *ave_p;
    double initial_ave_energy, total_time;
    long steps_done;
    /* random numbers */
    uint32_t m_w, m_z;
    int spare;
    double rand1, rand2;
    unsigned long long epoch;
    /* quantum thermostat */
    double* qH;                  /* the filter, 2 Nfrequency_quantum values */
    int qNf2;
    double* qnoise;              /* current coloured noise per degree of freedom */
    long long qcount;            /* calls of the kick's A part so far */
};

/* the quantum thermostat's normals: epoch QEPOCH + t, with t >= -Nf2 the
   index of the draw in each degree of freedom's history */
#define QEPOCH (1ULL << 62)

/* ---- geometry: periodic_CPU.cpp:31-50, find_image_CPU.cpp:31-53 ---- */
static v3 to_frac(const orc_sys* S, v3 r) {
    const double* I = S->inv;
    return vinit(I[0] * r.x + I[1] * r.y + I[3] * r.z, I[2] * r.y + I[4] * r.z, I[5] * r.z);
}
static v3 to_cart(const orc_sys* S, v3 q) {
    const double* d = S->d;
    return vinit(d[0] * q.x + d[1] * q.y + d[3] * q.z, d[2] * q.y + d[4] * q.z, d[5] * q.z);
}
static v3 periodic(const orc_sys* S, v3 r) {
    v3 q = to_frac(S, r);
    int idx = 0;
    if (q.x < 0e0 || q.x >= 1e0) { q.x -= (int)q.x; ++idx; }
    if (q.y < 0e0 || q.y >= 1e0) { q.y -= (int)q.y; ++idx; }
    if (q.z < 0e0 || q.z >= 1e0) { q.z -= (int)q.z; ++idx; }
    return idx > 0 ? to_cart(S, q) : r;
}
static v3 find_image(const orc_sys* S, v3 rij) {
    v3 q = to_frac(S, rij);
    int idx = 0;
    if (q.x < -0.5e0) { q.x += 1e0; ++idx; }
    if (q.x >= 0.5e0) { q.x -= 1e0; ++idx; }
    if (q.y < -0.5e0) { q.y += 1e0; ++idx; }
    if (q.y >= 0.5e0) { q.y -= 1e0; ++idx; }
    if (q.z < -0.5e0) { q.z += 1e0; ++idx; }
    if (q.z >= 0.5e0) { q.z -= 1e0; ++idx; }
    return idx > 0 ? to_cart(S, q) : rij;
}

/* map_cells.cpp:77-125: the 26 neighbours in the reference's fixed order */
static void neighbour_table(int nx, int ny, int nz, int* neigh) {
    int nd = nx, nh = nx * ny;
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int iz = 0; iz < nz; ++iz) {
                int* c = neigh + 26 * (ix + iy * nd + iz * nh);
                int xp = (ix + 1) % nx, yp = (iy + 1) % ny, zp = (iz + 1) % nz;
                int xm = (ix - 1 + nx) % nx, ym = (iy - 1 + ny) % ny, zm = (iz - 1 + nz) % nz;
                int X[26] = {xp, xp, ix, xm, xp, xp, ix, xm, xp, xp, ix, xm, ix,
                             xm, ix, ix, xp, xm, xm, xm, ix, ix, xp, xp, xm, xm};
                int Y[26] = {iy, yp, yp, yp, iy, yp, yp, yp, iy, yp, yp, yp, iy,
                             iy, ym, iy, ym, ym, iy, iy, ym, ym, ym, ym, ym, ym};
                int Z[26] = {iz, iz, iz, iz, zm, zm, zm, zm, zp, zp, zp, zp, zp,
                             iz, iz, zm, iz, iz, zp, zm, zp, zm, zp, zm, zp, zm};
                for (int k = 0; k < 26; ++k) c[k] = X[k] + Y[k] * nd + Z[k] * nh;
            }
}

/* allocate_cells_CPU.cpp:33-125: greedy colouring in cell-index order */
static int colour(int nc, const int* neigh, int** gstart_out, int** gcells_out) {
    int* type = (int*)calloc(nc, sizeof(int));
    int* gcells = (int*)malloc(sizeof(int) * nc);
    int* gstart = (int*)malloc(sizeof(int) * (nc + 1));
    int ng = 0, left = nc, k = 0;
    gstart[0] = 0;
    while (left > 0) {
        for (int i = 0; i < nc; ++i) {
            if (type[i] == 0) {
                gcells[k++] = i;
                type[i] = 1;
                --left;
                for (int j = 0; j < 26; ++j)
                    if (type[neigh[26 * i + j]] != 1) type[neigh[26 * i + j]] = -1;
            }
        }
        ++ng;
        gstart[ng] = k;
        for (int i = 0; i < nc; ++i)
            if (type[i] == -1) type[i] = 0;
    }
    free(type);
    *gstart_out = gstart;
    *gcells_out = gcells;
    return ng;
}

/* ---- Te heat capacity: heatcapacity_CPU.cpp:34-57 ---- */
static double Ce(double Te) { double a = 3e0, b = 2e-4 / BOLTZ; return a * tanh(b * Te); }
static double Te_to_Ee(double Te) { double a = 3e0, b = 2e-4 / BOLTZ; return a / b * log(cosh(b * Te)); }
static double Ee_to_Te(double Ee) { double a = 3e0, b = 2e-4 / BOLTZ; return acosh(exp(b / a * Ee)) / b; }

/* ---- random numbers: random_number_CPU.cpp:38-104 (one thread) ---- */
static double mwc_uniform(orc_sys* S) {
    uint32_t m_z = S->m_z, m_w = S->m_w;
    m_z = 36969 * (m_z & 65535) + (m_z >> 16);
    m_w = 18000 * (m_w & 65535) + (m_w >> 16);
    uint32_t un = (m_z << 16) + m_w;
    S->m_z = m_z;
    S->m_w = m_w;
    return (un + 1.0) * 2.328306435454494e-10;
}
static double mwc_normal(orc_sys* S) {
    if (S->spare == 1) {
        S->spare = 0;
        return sqrt(S->rand1) * sin(S->rand2);
    }
    S->spare = 1;
    S->rand1 = mwc_uniform(S);
    S->rand1 = -2e0 * log(S->rand1);
    S->rand2 = mwc_uniform(S) * 6.283185307179586;
    return sqrt(S->rand1) * cos(S->rand2);
}
/* three normals for atom i, drawn from the active source */
static v3 normals3(orc_sys* S, int i) {
    if (S->P.rng == ORC_RNG_MWC) {
        double a = mwc_normal(S), b = mwc_normal(S), c = mwc_normal(S);
        return vinit(a, b, c);
    }
    double o[3];
    orc_philox_normals((unsigned)S->P.random_seed, 0u, (unsigned)i, S->epoch, o);
    return vinit(o[0], o[1], o[2]);
}

/* ---- links: links_CPU.cpp:33-177 ---- */
static void list_push_front(orc_sys* S, int c, int i) {
    S->prev[i] = -1;
    S->next[i] = S->head[c];
    S->head[c] = i;
    ++S->count[c];
    if (S->next[i] < 0) S->tail[c] = i;
    else S->prev[S->next[i]] = i;
}

static int te_node_of(const orc_sys* S, v3 r) {
    if (S->P.te_mesh <= 0) return -1;
    v3 q = to_frac(S, r);
    int a = (int)(q.x * S->tx), b = (int)(q.y * S->ty), c = (int)(q.z * S->tz);
    if (a < 0) a = 0;
    if (b < 0) b = 0;
    if (c < 0) c = 0;
    if (a >= S->tx) a = S->tx - 1;
    if (b >= S->ty) b = S->ty - 1;
    if (c >= S->tz) c = S->tz - 1;
    return a + b * S->tx + c * S->tx * S->ty;
}

static void update_te_nodes(orc_sys* S) {
    if (S->P.te_mesh <= 0) {
        for (int i = 0; i < S->n; ++i) S->node[i] = S->cell[i];
        return;
    }
    for (int k = 0; k < S->nte; ++k) S->te_count[k] = 0;
    for (int i = 0; i < S->n; ++i) {
        S->node[i] = te_node_of(S, ld(S->r, i));
        ++S->te_count[S->node[i]];
    }
}

static void initial_links(orc_sys* S) {
    for (int i = 0; i < S->n; ++i) {
        S->next[i] = S->prev[i] = -1;
        S->old_cell[i] = -1;
        S->cell[i] = -2;
        st(S->r, i, periodic(S, ld(S->r, i)));
    }
    for (int c = 0; c < S->ncells; ++c) { S->head[c] = S->tail[c] = -1; S->count[c] = 0; }
    for (int i = 0; i < S->n; ++i) {
        v3 q = to_frac(S, ld(S->r, i));
        int c = (int)(q.x * S->nx) + (int)(q.y * S->ny) * S->nx +
                (int)(q.z * S->nz) * S->nx * S->ny;
        S->cell[i] = c;
        list_push_front(S, c, i);
    }
    update_te_nodes(S);
}

void orc_links(orc_sys* S) {
    int moved = 0;
    for (int i = 0; i < S->n; ++i) {
        S->old_cell[i] = S->cell[i];
        v3 q = to_frac(S, ld(S->r, i));
        int lx = (int)(q.x * S->nx), ly = (int)(q.y * S->ny), lz = (int)(q.z * S->nz);
        if (lx < 0) lx = 0;
        if (ly < 0) ly = 0;
        if (lz < 0) lz = 0;
        if (lx >= S->nx) lx = S->nx - 1;
        if (ly >= S->ny) ly = S->ny - 1;
        if (lz >= S->nz) lz = S->nz - 1;
        int c = lx + ly * S->nx + lz * S->nx * S->ny;
        S->cell[i] = c;
        if (c != S->old_cell[i]) ++moved;
    }
    if (moved) {
        for (int i = 0; i < S->n; ++i) {      /* ascending atom index */
            if (S->cell[i] == S->old_cell[i]) continue;
            int oc = S->old_cell[i], nc = S->cell[i];
            if (S->prev[i] < 0) S->head[oc] = S->next[i];
            else S->next[S->prev[i]] = S->next[i];
            if (S->next[i] < 0) S->tail[oc] = S->prev[i];
            else S->prev[S->next[i]] = S->prev[i];
            --S->count[oc];
            list_push_front(S, nc, i);
        }
    }
    update_te_nodes(S);
}

/* ---- rho: calculate_rho_CPU.cpp:33-92 (half shell, colour order) ---- */
void orc_rho(orc_sys* S) {
    for (int i = 0; i < S->n; ++i) S->rho[i] = 0e0;
    for (int g = 0; g < S->ngroups; ++g)
        for (int k = S->gstart[g]; k < S->gstart[g + 1]; ++k)
            for (int i = S->head[S->gcells[k]]; i >= 0; i = S->next[i]) {
                int c0 = S->cell[i];
                v3 ri = ld(S->r, i);
                for (int w = 0; w <= 13; ++w) {
                    int wc = (w == 13) ? c0 : S->neigh[26 * c0 + w];
                    for (int j = S->head[wc]; j >= 0; j = S->next[j]) {
                        if (j == i && w == 13) break;
                        v3 rij = find_image(S, vsub(ri, ld(S->r, j)));
                        double r0 = vlen(rij);
                        if (r0 < S->rcut_pot && j != i) {
                            double fv = interp(r0, S->T.inv_r, S->T.t[T_f]);
                            S->rho[i] += fv;
                            S->rho[j] += fv;
                        }
                    }
                }
            }
}

/* ---- force/energy: calculate_force_energy_CPU.cpp:33-301 ---- */
static void force_inner(orc_sys* S, int i) {
    const tables* T = &S->T;
    v3 si = ld(S->s, i);
    double si_sq = vsq(si);
    int c0 = S->cell[i];
    v3 ri = ld(S->r, i);
    for (int w = 0; w <= 13; ++w) {
        int wc = (w == 13) ? c0 : S->neigh[26 * c0 + w];
        for (int j = S->head[wc]; j >= 0; j = S->next[j]) {
            if (j == i && w == 13) break;
            v3 rij = find_image(S, vsub(ri, ld(S->r, j)));
            double rsq = vsq(rij);
            double pair_enr = 0e0, dudr = 0e0, dudr_spin = 0e0;
            v3 sj = ld(S->s, j);
            double sj_sq = vsq(sj);
            if (rsq < S->rcut_max_sq && i != j) {
                double r0 = sqrt(rsq);
                if (r0 < S->rcut_pot) {
                    double df = interp(r0, T->inv_r, T->t[T_df]);
                    dudr = (interp(S->rho[i], T->inv_rho, T->t[T_dF]) +
                            interp(S->rho[j], T->inv_rho, T->t[T_dF])) * df +
                           interp(r0, T->inv_r, T->t[T_dphi]);
                    double ri_ = S->rho[i], rj_ = S->rho[j];
                    dudr += (interp(ri_, T->inv_rho, T->t[T_dLA]) * si_sq +
                             interp(ri_, T->inv_rho, T->t[T_dLB]) * pow(si_sq, 2) +
                             interp(ri_, T->inv_rho, T->t[T_dLC]) * pow(si_sq, 3) +
                             interp(ri_, T->inv_rho, T->t[T_dLD]) * pow(si_sq, 4)) * df;
                    dudr += (interp(rj_, T->inv_rho, T->t[T_dLA]) * sj_sq +
                             interp(rj_, T->inv_rho, T->t[T_dLB]) * pow(sj_sq, 2) +
                             interp(rj_, T->inv_rho, T->t[T_dLC]) * pow(sj_sq, 3) +
                             interp(rj_, T->inv_rho, T->t[T_dLD]) * pow(sj_sq, 4)) * df;
                    pair_enr = interp(r0, T->inv_r, T->t[T_phi]);
                    S->pe[i] += 0.5e0 * pair_enr;
                    S->pe[j] += 0.5e0 * pair_enr;
                }
                if (r0 < S->rcut_mag) {
                    double dot = vdot(si, sj);
                    double times = sqrt(si_sq * sj_sq);
                    dudr_spin = -interp(r0, T->inv_r, T->t[T_dJ]) * (dot - times);
                    double Jh = interp(r0, T->inv_r, T->t[T_J]) / 2e0;
                    double Jt = Jh * times, Jd = -Jh * dot;
                    S->me0[i] += Jt;
                    S->me[i] += Jd;
                    S->me0[j] += Jt;
                    S->me[j] += Jd;
                }
                dudr += dudr_spin;
                double force = -dudr / r0;
                v3 fij = vmul(force, rij);
                S->f[3 * i] += fij.x; S->f[3 * i + 1] += fij.y; S->f[3 * i + 2] += fij.z;
                S->f[3 * j] -= fij.x; S->f[3 * j + 1] -= fij.y; S->f[3 * j + 2] -= fij.z;
                double* a = S->stress + 6 * i;
                double* b = S->stress + 6 * j;
                a[0] += fij.x * rij.x; a[1] += fij.y * rij.y; a[2] += fij.z * rij.z;
                a[3] += fij.x * rij.y; a[4] += fij.y * rij.z; a[5] += fij.z * rij.x;
                b[0] += fij.x * rij.x; b[1] += fij.y * rij.y; b[2] += fij.z * rij.z;
                b[3] += fij.x * rij.y; b[4] += fij.y * rij.z; b[5] += fij.z * rij.x;
                S->vir[i] += -force * rsq;
            }
        }
    }
    double rho = S->rho[i];
    S->pe[i] += interp(rho, T->inv_rho, T->t[T_F]);
    S->me[i] += interp(rho, T->inv_rho, T->t[T_LA]) * si_sq +
                interp(rho, T->inv_rho, T->t[T_LB]) * pow(si_sq, 2) +
                interp(rho, T->inv_rho, T->t[T_LC]) * pow(si_sq, 3) +
                interp(rho, T->inv_rho, T->t[T_LD]) * pow(si_sq, 4);
}

void orc_force(orc_sys* S) {
    for (int i = 0; i < S->n; ++i) {
        S->f[3 * i] = S->f[3 * i + 1] = S->f[3 * i + 2] = 0e0;
        S->pe[i] = S->vir[i] = 0e0;
        for (int k = 0; k < 6; ++k) S->stress[6 * i + k] = 0e0;
        S->me[i] = S->me0[i] = 0e0;
    }
    for (int g = 0; g < S->ngroups; ++g)
        for (int k = S->gstart[g]; k < S->gstart[g + 1]; ++k)
            for (int i = S->head[S->gcells[k]]; i >= 0; i = S->next[i]) force_inner(S, i);
    for (int i = 0; i < S->n; ++i) S->lv[i] = S->box_volume / S->n;
    for (int i = 0; i < S->n; ++i) {
        v3 p = ld(S->p, i);
        double* a = S->stress + 6 * i;
        double m = S->atmass, V = S->lv[i];
        a[0] = (pow(p.x, 2) / m + a[0] / 2e0) / V;
        a[1] = (pow(p.y, 2) / m + a[1] / 2e0) / V;
        a[2] = (pow(p.z, 2) / m + a[2] / 2e0) / V;
        a[3] = ((p.x * p.y) / m + a[3] / 2e0) / V;
        a[4] = ((p.y * p.z) / m + a[4] / 2e0) / V;
        a[5] = ((p.z * p.x) / m + a[5] / 2e0) / V;
    }
}

/* ---- spin: calculate_spin_CPU.cpp:33-274, core_ds_CPU.cpp:90-127 ---- */
static v3 spin_rotation(v3 Heff, v3 s, double dt) {
    v3 w = vdiv(Heff, -HBAR);
    double w0 = vlen(w);
    if (w0 > 0e0) w = vdiv(w, w0);
    else w = vzero();
    double w12 = w.x * w.y, w23 = w.y * w.z, w13 = w.x * w.z;
    double w1s = w.x * w.x, w2s = w.y * w.y, w3s = w.z * w.z;
    double A = sin(w0 * dt);
    double B = 1e0 - cos(w0 * dt);
    v3 o;
    o.x = s.x + (s.x * B * (-w2s - w3s) + s.y * (B * w12 - A * w.z) + s.z * (A * w.y + B * w13));
    o.y = s.y + (s.y * B * (-w1s - w3s) + s.z * (B * w23 - A * w.x) + s.x * (A * w.z + B * w12));
    o.z = s.z + (s.z * B * (-w1s - w2s) + s.x * (B * w13 - A * w.y) + s.y * (A * w.x + B * w23));
    return o;
}

/* inner_spin (:201-235) and inner_sum_Jij_sj (:238-274): 26 neighbour
   cells in table order, then the atom's own cell, each head -> tail */
static v3 heff_H(const orc_sys* S, int i) {
    v3 H = vzero();
    int c0 = S->cell[i];
    v3 ri = ld(S->r, i);
    for (int w = 0; w <= 26; ++w) {
        int wc = (w == 26) ? c0 : S->neigh[26 * c0 + w];
        for (int j = S->head[wc]; j >= 0; j = S->next[j]) {
            v3 rij = find_image(S, vsub(ri, ld(S->r, j)));
            double rsq = vsq(rij);
            if (rsq < S->rcut_mag_sq && i != j) {
                double J = interp(sqrt(rsq), S->T.inv_r, S->T.t[T_J]);
                H = vadd(H, vmul(J, ld(S->s, j)));
            }
        }
    }
    return H;
}
static double sum_J_sj(const orc_sys* S, int i) {
    double acc = 0e0;
    int c0 = S->cell[i];
    v3 ri = ld(S->r, i);
    for (int w = 0; w <= 26; ++w) {
        int wc = (w == 26) ? c0 : S->neigh[26 * c0 + w];
        for (int j = S->head[wc]; j >= 0; j = S->next[j]) {
            v3 rij = find_image(S, vsub(ri, ld(S->r, j)));
            double rsq = vsq(rij);
            if (rsq < S->rcut_mag_sq && i != j) {
                double J = interp(sqrt(rsq), S->T.inv_r, S->T.t[T_J]);
                acc += J * vlen(ld(S->s, j));
            }
        }
    }
    return acc;
}

static double landau_poly(double A, double B, double C, double D, double s_sq) {
    return 2e0 * A + 4e0 * B * s_sq + 6e0 * C * pow(s_sq, 2) + 8e0 * D * pow(s_sq, 3);
}

/* Landau + exchange-correction field for spin x (calculate_spin_CPU.cpp:127-136) */
static v3 landau_field(double A, double B, double C, double D, double sumJ, v3 x) {
    double s_sq = vsq(x);
    v3 HL = vmul(-landau_poly(A, B, C, D, s_sq), x);
    double s0 = sqrt(s_sq);
    v3 HC = vzero();
    if (s0 > 0e0) HC = vmul(-sumJ / s0, x);
    return vadd(HL, HC);
}

static double atom_T(const orc_sys* S, int i) {
    return S->P.eltemp ? S->Te[S->node[i]] : S->temperature;
}

static void spin_visit(orc_sys* S, int i, double dt) {
    v3 H = heff_H(S, i);
    v3 s = ld(S->s, i);
    v3 HL = vzero();
    if (!S->P.spinlang) {
        s = spin_rotation(H, s, dt);
    } else {
        double dt_half = dt / 2e0, dt_quad = dt / 4e0;
        double g = S->gamma_S_HL;
        const tables* T = &S->T;
        double rho = S->rho[i];
        double A = interp(rho, T->inv_rho, T->t[T_LA]);
        double B = interp(rho, T->inv_rho, T->t[T_LB]);
        double C = interp(rho, T->inv_rho, T->t[T_LC]);
        double D = interp(rho, T->inv_rho, T->t[T_LD]);
        s = spin_rotation(H, s, dt_half);                            /* part 1 */
        double sumJ = sum_J_sj(S, i);
        S->sumJ[i] = sumJ;
        HL = landau_field(A, B, C, D, sumJ, s);                      /* part 2 */
        v3 s_tmp = vadd(s, vmul(g * dt_quad, vadd(H, HL)));
        HL = landau_field(A, B, C, D, sumJ, s_tmp);
        s = vadd(s, vmul(g * dt_half, vadd(H, HL)));
        double amp = sqrt(2e0 * atom_T(S, i) * g / dt);              /* part 3 */
        v3 xi = normals3(S, i);
        v3 dS = vinit(amp * xi.x, amp * xi.y, amp * xi.z);
        s = vadd(s, vmul(dt, dS));
        HL = landau_field(A, B, C, D, sumJ, s);                      /* part 4 */
        s_tmp = vadd(s, vmul(g * dt_quad, vadd(H, HL)));
        HL = landau_field(A, B, C, D, sumJ, s_tmp);
        s = vadd(s, vmul(g * dt_half, vadd(H, HL)));
        s = spin_rotation(H, s, dt_half);                            /* part 5 */
    }
    st(S->H, i, H);
    st(S->HL, i, HL);
    st(S->s, i, s);
    S->s0[i] = vlen(s);
}

/* core_ds_CPU.cpp:35-83: forward sweep over colour groups (head -> tail),
   then the backward sweep (tail -> head), each visit with dt/2 */
void orc_core_ds(orc_sys* S, double dt) {
    double dt_half = dt / 2e0;
    for (int g = 0; g < S->ngroups; ++g)
        for (int k = S->gstart[g]; k < S->gstart[g + 1]; ++k)
            for (int i = S->head[S->gcells[k]]; i >= 0; i = S->next[i]) spin_visit(S, i, dt_half);
    if (S->P.spinlang) ++S->epoch;
    for (int g = S->ngroups - 1; g >= 0; --g)
        for (int k = S->gstart[g]; k < S->gstart[g + 1]; ++k)
            for (int i = S->tail[S->gcells[k]]; i >= 0; i = S->prev[i]) spin_visit(S, i, dt_half);
    if (S->P.spinlang) ++S->epoch;
}

/* ---- lattice: core_dp_CPU.cpp:51-312, core_dr_CPU.cpp:33-44 ---- */
static void kick_atom(orc_sys* S, int i, double dt, v3* noise_out) {
    v3 ff;
    if (S->P.quantum) {
        /* core_dp_CPU.cpp:137-147: sqrt(2 gamma_L / h) times the coloured noise */
        double h = dt * S->P.msteps_quantum;
        ff = vmul(sqrt(2e0 * S->gamma_L / h), ld(S->qnoise, i));
    } else {
        double amp = sqrt(2e0 * atom_T(S, i) * S->gamma_L / dt);
        ff = vmul(amp, normals3(S, i));
    }
    st(S->p, i, vadd(ld(S->p, i), vmul(dt, vadd(ld(S->f, i), ff))));
    *noise_out = ff;
}

/* quantum_noise_CPU.cpp:56-72 for every degree of freedom at once (their
   counters advance together): every Msteps_quantum calls, the filter over
   the history of normals, newest first, then one new normal.  With
   counter-based normals the history is the draws t = u - Nf2 .. u - 1 of
   update u; the reference's initial history is the draws before update 0. */
static void quantum_update(orc_sys* S) {
    if (S->qcount % S->P.msteps_quantum == 0) {
        long long u = S->qcount / S->P.msteps_quantum;
        int Nf2 = S->qNf2;
        for (int i = 0; i < S->n; ++i) {
            double q[3] = {0e0, 0e0, 0e0};
            for (int k = 0; k < Nf2; ++k) {
                double o[3];
                orc_philox_normals((unsigned)S->P.random_seed, 0u, (unsigned)i,
                                   QEPOCH + (unsigned long long)(u - 1 - k + Nf2), o);
                for (int c = 0; c < 3; ++c) q[c] += S->qH[k] * o[c];
            }
            st(S->qnoise, i, vinit(q[0], q[1], q[2]));
        }
    }
    ++S->qcount;
}

static void dp_A(orc_sys* S, double dt) {                 /* :94-188 */
    if (S->P.quantum) quantum_update(S);
    if (S->P.localcolmot) {
        for (int g = 0; g < S->ngroups; ++g)
            for (int k = S->gstart[g]; k < S->gstart[g + 1]; ++k) {
                int c = S->gcells[k];
                if (S->head[c] < 0) continue;
                v3 acc = vzero();
                for (int i = S->head[c]; i >= 0; i = S->next[i]) {
                    v3 ff;
                    kick_atom(S, i, dt, &ff);
                    acc = vadd(acc, ff);
                }
                st(S->ave_ff, c, vdiv(acc, S->count[c]));
            }
        for (int i = 0; i < S->n; ++i)
            st(S->p, i, vsub(ld(S->p, i), vmul(dt, ld(S->ave_ff, S->cell[i]))));
    } else {
        for (int i = 0; i < S->n; ++i) {
            v3 ff;
            kick_atom(S, i, dt, &ff);
        }
    }
    ++S->epoch;
}

static void dp_B(orc_sys* S, double dt) {                 /* :190-207 */
    for (int i = 0; i < S->n; ++i) {
        double e;
        if (S->P.localcolmot)
            e = exp(-S->gamma_L / S->atmass * dt * (1e0 - 1e0 / S->count[S->cell[i]]));
        else
            e = exp(-S->gamma_L / S->atmass * dt);
        st(S->p, i, vmul(e, ld(S->p, i)));
    }
}

/* :211-264; the colour order does not change the result (each cell only
   touches its own atoms), the in-cell order does */
static void dp_C(orc_sys* S, double dt, int backward) {
    for (int c = 0; c < S->ncells; ++c) {
        if (S->head[c] < 0) continue;
        double factor = S->gamma_L / S->atmass * dt / S->count[c];
        for (int i = backward ? S->tail[c] : S->head[c]; i >= 0;
             i = backward ? S->prev[i] : S->next[i]) {
            v3 sum_p = vzero();
            for (int j = S->head[c]; j >= 0; j = S->next[j]) sum_p = vadd(sum_p, ld(S->p, j));
            v3 pi = ld(S->p, i);
            st(S->p, i, vadd(pi, vmul(factor, vsub(sum_p, pi))));
        }
    }
}

static void rescale_momentum(orc_sys* S) {                /* :268-312 */
    double ax = 0e0, ay = 0e0, az = 0e0;
    for (int i = 0; i < S->n; ++i) { ax += S->p[3 * i]; ay += S->p[3 * i + 1]; az += S->p[3 * i + 2]; }
    ax /= S->n; ay /= S->n; az /= S->n;
    double old_ke = 0e0, new_ke = 0e0;
    for (int i = 0; i < S->n; ++i) {
        S->ke[i] = vsq(ld(S->p, i)) / 2e0 / S->atmass;
        old_ke += S->ke[i];
        S->p[3 * i] -= ax; S->p[3 * i + 1] -= ay; S->p[3 * i + 2] -= az;
        S->ke[i] = vsq(ld(S->p, i)) / 2e0 / S->atmass;
        new_ke += S->ke[i];
    }
    double factor = sqrt(old_ke / new_ke);
    if (new_ke < 1e-10) factor = 1e0;
    for (int i = 0; i < S->n; ++i) st(S->p, i, vmul(factor, ld(S->p, i)));
}

void orc_core_dp(orc_sys* S, double dt) {
    if (S->P.lattlang) {
        if (S->P.localcolmot) dp_C(S, dt / 2e0, 0);
        dp_B(S, dt / 2e0);
        dp_A(S, dt);
        dp_B(S, dt / 2e0);
        if (S->P.localcolmot) dp_C(S, dt / 2e0, 1);
    } else {
        for (int i = 0; i < S->n; ++i) st(S->p, i, vadd(ld(S->p, i), vmul(dt, ld(S->f, i))));
    }
    rescale_momentum(S);
    for (int i = 0; i < S->n; ++i) S->ke[i] = vsq(ld(S->p, i)) / 2e0 / S->atmass;
}

void orc_core_dr(orc_sys* S, double dt) {
    double k = dt / S->atmass;
    for (int i = 0; i < S->n; ++i) st(S->r, i, periodic(S, vadd(ld(S->r, i), vmul(k, ld(S->p, i)))));
}

/* ---- electron temperature: calculate_temperature_CPU.cpp:35-148,
        core_dTe_CPU.cpp:47-217 ---- */
static void te_cell_sums(orc_sys* S, int i, int k) {
    double rho = S->rho[i];
    const tables* T = &S->T;
    if (S->P.lattlang) {
        S->Tl[k] += S->ke[i];                      /* sum_ke, finished below */
        if (S->P.localcolmot) st(S->ave_p, k, vadd(ld(S->ave_p, k), ld(S->p, i)));
    }
    v3 H = heff_H(S, i);
    v3 s = ld(S->s, i);
    st(S->H, i, H);
    S->sRup[k] += vsq(vcross(s, H));
    S->sRdn[k] += vdot(s, H);
    double A = interp(rho, T->inv_rho, T->t[T_LA]), B = interp(rho, T->inv_rho, T->t[T_LB]);
    double C = interp(rho, T->inv_rho, T->t[T_LC]), D = interp(rho, T->inv_rho, T->t[T_LD]);
    double s_sq = vsq(s);
    S->s0[i] = vlen(s);
    v3 HL = vmul(-landau_poly(A, B, C, D, s_sq), s);
    double sumJ = sum_J_sj(S, i);
    S->sumJ[i] = sumJ;
    v3 HC = vmul(-sumJ / S->s0[i], s);
    HL = vadd(HL, HC);
    st(S->HL, i, HL);
    S->sLup[k] += vsq(vadd(H, HL));
    S->sLdn[k] += 6e0 * A + 20e0 * B * s_sq + 42e0 * C * pow(s_sq, 2) + 72e0 * D * pow(s_sq, 3);
    S->sLdn[k] += 2e0 * sumJ / S->s0[i];
}

void orc_temperature(orc_sys* S) {
    if (!S->P.eltemp) return;
    for (int k = 0; k < S->nte; ++k) {
        S->Tl[k] = 0e0;
        st(S->ave_p, k, vzero());
        S->sRup[k] = S->sRdn[k] = S->sLup[k] = S->sLdn[k] = 0e0;
    }
    if (S->P.te_mesh <= 0) {
        for (int c = 0; c < S->ncells; ++c)
            for (int i = S->head[c]; i >= 0; i = S->next[i]) te_cell_sums(S, i, c);
    } else {
        for (int i = 0; i < S->n; ++i) te_cell_sums(S, i, S->node[i]);
    }
    double per = (double)S->n / (double)S->nte;
    for (int k = 0; k < S->nte; ++k) {
        double n = S->te_count[k];
        double sum_ke = S->Tl[k];
        if (S->P.lattlang) {
            if (S->P.localcolmot) {
                st(S->ave_p, k, vdiv(ld(S->ave_p, k), n));
                sum_ke -= n * vsq(ld(S->ave_p, k)) / 2e0 / S->atmass;
                S->Tl[k] = 2e0 / 3e0 * sum_ke / (n - 1e0) / BOLTZ;
                S->Gel[k] = 3e0 * (n - 1e0) * BOLTZ * S->gamma_L / S->atmass / per;
            } else {
                S->Tl[k] = sum_ke * 2e0 / 3e0 / n / BOLTZ;
                S->Gel[k] = 3e0 * n * BOLTZ * S->gamma_L / S->atmass / per;
            }
        } else {
            S->Tl[k] = 0e0;
            S->Gel[k] = 0e0;
        }
        S->TsR[k] = S->sRup[k] / S->sRdn[k] / 2e0 / BOLTZ;
        S->TsL[k] = S->sLup[k] / S->sLdn[k] / BOLTZ;
        S->Ges[k] = BOLTZ * S->gamma_S_HL * S->sLdn[k] / per;
    }
}

static void dte_A(orc_sys* S, double dt) {
    for (int k = 0; k < S->nte; ++k) {
        S->Ee[k] = Te_to_Ee(S->Te[k]);
        double dE = 0e0;
        if (S->P.lattlang) dE += S->Gel[k] * S->Tl[k];
        if (S->P.spinlang) dE += S->Ges[k] * S->TsL[k];
        S->Ee[k] += dt * dE;
        S->Te[k] = Ee_to_Te(S->Ee[k]);
    }
}

static void dte_B(orc_sys* S, double dt) {
    for (int k = 0; k < S->nte; ++k) {
        double g = 0e0;
        if (S->P.lattlang) g += S->Gel[k];
        if (S->P.spinlang) g += S->Ges[k];
        g *= dt / BOLTZ;
        double T0 = S->Te[k];
        double k1 = T0 * (exp(-g / Ce(T0)) - 1e0) / dt;
        double T1 = T0 + k1 * dt / 2e0;
        double k2 = T1 * (exp(-g / Ce(T1)) - 1e0) / dt;
        double T2 = T0 + k2 * dt / 2e0;
        double k3 = T2 * (exp(-g / Ce(T2)) - 1e0) / dt;
        double T3 = T0 + k3 * dt;
        double k4 = T3 * (exp(-g / Ce(T3)) - 1e0) / dt;
        S->Te[k] += dt / 6e0 * (k1 + 2e0 * k2 + 2e0 * k3 + k4);
    }
}

static void dte_C(orc_sys* S, double dt) {
    double start = 0e0;
    for (int k = 0; k < S->nte; ++k) { S->Ee[k] = Te_to_Ee(S->Te[k]); start += S->Ee[k]; }
    double cond = S->P.kappa_e / EVTOJ / 1e10;
    double dx2 = pow(S->box_len[0] / S->tx, 2);
    double dy2 = pow(S->box_len[1] / S->ty, 2);
    double dz2 = pow(S->box_len[2] / S->tz, 2);
    double atomic_volume = S->box_volume / (double)S->n;
    double volume_factor = atomic_volume / ((double)S->n / (double)S->nte);
    double pre = dt / 2e0 * cond * volume_factor / BOLTZ;
    for (int pass = 0; pass < 2; ++pass)
        for (int gg = 0; gg < S->te_ngroups; ++gg) {
            int g = pass == 0 ? gg : S->te_ngroups - 1 - gg;
            for (int m = S->te_gstart[g]; m < S->te_gstart[g + 1]; ++m) {
                int k = S->te_gcells[m];
                const int* nb = S->te_neigh + 26 * k;
                double* Te = S->Te;
                S->Ee[k] = Te_to_Ee(Te[k]);
                S->Ee[k] += pre * ((Te[nb[0]] + Te[nb[13]] - 2e0 * Te[k]) / dx2 +
                                   (Te[nb[2]] + Te[nb[14]] - 2e0 * Te[k]) / dy2 +
                                   (Te[nb[12]] + Te[nb[15]] - 2e0 * Te[k]) / dz2);
                Te[k] = Ee_to_Te(S->Ee[k]);
            }
        }
    double end = 0e0;
    for (int k = 0; k < S->nte; ++k) { S->Ee[k] = Te_to_Ee(S->Te[k]); end += S->Ee[k]; }
    double fac = start / end;
    for (int k = 0; k < S->nte; ++k) { S->Ee[k] *= fac; S->Te[k] = Ee_to_Te(S->Ee[k]); }
}

void orc_core_dte(orc_sys* S, double dt) {
    if (!S->P.eltemp) return;
    int nloop = S->P.te_nloop > 0 ? S->P.te_nloop : 50;
    double h = dt / nloop;
    for (int i = 0; i < nloop; ++i) {
        dte_A(S, h / 2e0);
        dte_B(S, h / 2e0);
        dte_C(S, h);
        dte_B(S, h / 2e0);
        dte_A(S, h / 2e0);
    }
}

/* check_energy_CPU.cpp:33-111: averages, and with renormalizeEnergy the
   energy error moved into the electrons */
static void check_energy(orc_sys* S, int step, double* av) {
    double pe = 0e0, ke = 0e0, me = 0e0, me0 = 0e0;
    for (int i = 0; i < S->n; ++i) { pe += S->pe[i]; ke += S->ke[i]; }
    pe /= S->n; ke /= S->n;
    for (int i = 0; i < S->n; ++i) { me += S->me[i]; me0 += S->me0[i]; }
    me /= S->n; me0 /= S->n;
    double Ee = 0e0;
    if (S->P.eltemp) {
        for (int k = 0; k < S->nte; ++k) {
            S->Ee[k] = Te_to_Ee(S->Te[k]);
            Ee += ((double)S->n / (double)S->nte) * S->Ee[k];
        }
        Ee /= S->n;
        if (S->P.renormalize) {
            double err = 0e0;
            if (step == -1) {
                S->initial_ave_energy = 0e0;
                S->initial_ave_energy += pe;
                S->initial_ave_energy += ke;
                S->initial_ave_energy += me;
                S->initial_ave_energy += me0;
                S->initial_ave_energy += Ee;
            } else {
                double cur = 0e0;
                cur += pe; cur += ke; cur += me; cur += me0; cur += Ee;
                err = cur - S->initial_ave_energy;
            }
            for (int k = 0; k < S->nte; ++k) {
                S->Ee[k] -= err;
                S->Te[k] = Ee_to_Te(S->Ee[k]);
            }
        }
    }
    if (av) { av[0] = pe; av[1] = ke; av[2] = me; av[3] = me0; av[4] = Ee; }
}

/* core.cpp:31-76, spin-lattice branch */
static void core(orc_sys* S) {
    double dt = S->P.step;
    orc_links(S);
    if (S->P.eltemp) orc_core_dte(S, dt / 2e0);
    orc_core_dp(S, dt / 2e0);
    orc_core_ds(S, dt / 2e0);
    orc_core_dr(S, dt);
    orc_rho(S);
    orc_core_ds(S, dt / 2e0);
    orc_force(S);
    orc_core_dp(S, dt / 2e0);
    if (S->P.eltemp) {
        orc_temperature(S);
        orc_core_dte(S, dt / 2e0);
    }
}

void orc_run(orc_sys* S, int nsteps) {
    int every = S->P.interval_of_print_out > 0 ? S->P.interval_of_print_out : 1;
    for (int k = 0; k < nsteps; ++k) {
        int cur = (int)S->steps_done;
        core(S);
        S->total_time += S->P.step;
        if (S->P.eltemp && S->P.renormalize && (cur + 1) % every == 0) check_energy(S, cur, NULL);
        ++S->steps_done;
    }
}

void orc_averages(orc_sys* S, double* out) {
    double saved = S->initial_ave_energy;
    double av[5];
    /* reading the averages must not renormalise: evaluate as step -1 on a
       copy of the Te state */
    double* te = (double*)malloc(sizeof(double) * (S->nte > 0 ? S->nte : 1));
    double* ee = (double*)malloc(sizeof(double) * (S->nte > 0 ? S->nte : 1));
    if (S->nte > 0) { memcpy(te, S->Te, sizeof(double) * S->nte); memcpy(ee, S->Ee, sizeof(double) * S->nte); }
    int ren = S->P.renormalize;
    S->P.renormalize = 0;
    check_energy(S, 0, av);
    S->P.renormalize = ren;
    if (S->nte > 0) { memcpy(S->Te, te, sizeof(double) * S->nte); memcpy(S->Ee, ee, sizeof(double) * S->nte); }
    free(te);
    free(ee);
    S->initial_ave_energy = saved;
    double ke = 0e0;
    for (int i = 0; i < S->n; ++i) ke += S->ke[i];
    double Te = 0e0;
    for (int k = 0; k < S->nte; ++k) Te += S->Te[k];
    double sx = 0e0, sy = 0e0, sz = 0e0;
    for (int i = 0; i < S->n; ++i) { sx += S->s[3 * i]; sy += S->s[3 * i + 1]; sz += S->s[3 * i + 2]; }
    out[0] = av[0]; out[1] = av[1]; out[2] = av[2]; out[3] = av[3]; out[4] = av[4];
    out[5] = ke * 2e0 / 3e0 / S->n / BOLTZ;                 /* check_temperature_CPU.cpp:38 */
    out[6] = S->nte > 0 ? Te / S->nte / BOLTZ : 0e0;
    out[7] = sx / S->n; out[8] = sy / S->n; out[9] = sz / S->n;
}

/* ---- set-up: initial.cpp:31-106 with the state given in memory ---- */
/* initial_quantum_noise (quantum_noise_CPU.cpp:75-104): the filter of the
   coloured noise, from the quantum spectrum hbar w (1/2 + n(w)) at Nf2
   frequencies up to pi/h, h = Msteps_quantum step/2 */
static void quantum_filter(orc_sys* S) {
    int Nf = S->P.nfrequency_quantum, Nf2 = 2 * Nf;
    double h = S->P.msteps_quantum * S->P.step / 2e0;
    double wmax = PI_NUM / h, dw = wmax / (double)Nf, T = S->temperature;
    double* Ht = (double*)malloc(sizeof(double) * Nf2);
    for (int i = 0; i < Nf2; ++i) {
        int k = i - Nf;
        double w = dw * (double)k;
        Ht[i] = sqrt(HBAR * fabs(w) * (0.5e0 + 1e0 / expm1(HBAR * fabs(w) / T)));
        Ht[i] *= (w * h / 2e0) / sin(w * h / 2e0);
        if (k == 0) Ht[i] = sqrt(T);
    }
    S->qNf2 = Nf2;
    S->qH = (double*)malloc(sizeof(double) * Nf2);
    for (int i = 0; i < Nf2; ++i) {
        S->qH[i] = 0e0;
        for (int j = 0; j < Nf2; ++j) {
            int k = j - Nf;
            S->qH[i] += Ht[j] * cos(PI_NUM / (double)Nf * (double)k * (double)(i - Nf));
        }
        S->qH[i] /= (double)Nf2;
    }
    free(Ht);
    S->qnoise = (double*)calloc(3 * (size_t)S->n, sizeof(double));
}

int orc_quantum_filter(orc_sys* S, double* out, int n) {
    if (!S->qH || n < S->qNf2) return -1;
    memcpy(out, S->qH, sizeof(double) * S->qNf2);
    return S->qNf2;
}

orc_sys* orc_create(const orc_params* prm, int natom, const double* r,
                    const double* p, const double* s, const double* te_K) {
    if (natom <= 0) return NULL;
    if (prm->quantum && (!prm->lattlang || prm->msteps_quantum < 1 || prm->nfrequency_quantum < 1))
        return NULL;
    if (prm->eltemp && !(prm->lattlang && prm->spinlang)) return NULL;
    orc_sys* S = (orc_sys*)calloc(1, sizeof(orc_sys));
    S->P = *prm;
    S->n = natom;
    memcpy(S->d, prm->box, sizeof(S->d));
    /* vec_utils_CPU.cpp:135-148 */
    double* d = S->d;
    S->inv[0] = 1e0 / d[0];
    S->inv[1] = -d[1] / (d[0] * d[2]);
    S->inv[2] = 1e0 / d[2];
    S->inv[3] = (d[1] * d[4] - d[2] * d[3]) / (d[0] * d[2] * d[5]);
    S->inv[4] = -d[4] / (d[2] * d[5]);
    S->inv[5] = 1e0 / d[5];
    S->box_len[0] = fabs(d[0]);
    S->box_len[1] = sqrt(d[1] * d[1] + d[2] * d[2]);
    S->box_len[2] = sqrt(d[3] * d[3] + d[4] * d[4] + d[5] * d[5]);
    S->box_volume = d[0] * d[2] * d[5];
    /* read_variables.cpp:191-276 unit conversions */
    S->atmass = prm->atmass * UTOEV * pow(LENGTH_SCALE, 2);
    S->temperature = prm->temperature * BOLTZ;
    S->gamma_L = prm->gamma_L_over_mass * S->atmass;
    S->gamma_S_HL = prm->gamma_S_HL;
    if (prm->quantum) quantum_filter(S);
    S->rcut_pot = prm->rcut_pot;
    S->rcut_mag = prm->rcut_mag;
    S->rcut_max = prm->rcut_max;
    S->min_len = prm->min_length_link_cell;
    if (S->rcut_max > S->min_len) S->min_len = S->rcut_max + 0.001;
    S->rcut_pot_sq = pow(S->rcut_pot, 2);
    S->rcut_mag_sq = pow(S->rcut_mag, 2);
    S->rcut_max_sq = pow(S->rcut_max, 2);

    build_tables(&S->T, S->rcut_max);

    int n = natom;
#define AL(ptr, cnt, T) ptr = (T*)calloc((size_t)(cnt), sizeof(T))
    AL(S->r, 3 * n, double); AL(S->p, 3 * n, double); AL(S->f, 3 * n, double);
    AL(S->s, 3 * n, double); AL(S->s0, n, double); AL(S->H, 3 * n, double);
    AL(S->HL, 3 * n, double); AL(S->HC, 3 * n, double); AL(S->rho, n, double);
    AL(S->pe, n, double); AL(S->ke, n, double); AL(S->me, n, double);
    AL(S->me0, n, double); AL(S->vir, n, double); AL(S->stress, 6 * n, double);
    AL(S->sumJ, n, double); AL(S->lv, n, double);
    AL(S->cell, n, int); AL(S->old_cell, n, int); AL(S->next, n, int);
    AL(S->prev, n, int); AL(S->node, n, int);
    memcpy(S->r, r, sizeof(double) * 3 * n);
    memcpy(S->p, p, sizeof(double) * 3 * n);
    memcpy(S->s, s, sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i) {
        S->s0[i] = vlen(ld(S->s, i));
        S->ke[i] = vsq(ld(S->p, i)) / 2e0 / S->atmass;
    }

    /* map_cells.cpp:41-61 */
    double a1 = sin(atan2(d[2], d[1])), a2 = sin(atan2(d[5], d[3])), a3 = sin(atan2(d[5], d[4]));
    double ex = fmax(S->min_len / a1, S->min_len / a2);
    double ey = fmax(S->min_len, S->min_len / a3);
    double ez = S->min_len;
    S->nx = (int)(d[0] / ex);
    S->ny = (int)(d[2] / ey);
    S->nz = (int)(d[5] / ez);
    if (S->nx < 3 || S->ny < 3 || S->nz < 3) { orc_destroy(S); return NULL; }
    S->ncells = S->nx * S->ny * S->nz;
    int nc = S->ncells;
    AL(S->head, nc, int); AL(S->tail, nc, int); AL(S->count, nc, int);
    AL(S->neigh, 26 * nc, int); AL(S->ave_ff, 3 * nc, double);
    neighbour_table(S->nx, S->ny, S->nz, S->neigh);

    if (prm->te_mesh > 0) {
        S->tx = S->ty = S->tz = prm->te_mesh;
        if (S->tx < 3) { orc_destroy(S); return NULL; }
        S->nte = S->tx * S->ty * S->tz;
        AL(S->te_neigh, 26 * S->nte, int);
        AL(S->te_count, S->nte, int);
        neighbour_table(S->tx, S->ty, S->tz, S->te_neigh);
    } else {
        S->tx = S->nx; S->ty = S->ny; S->tz = S->nz;
        S->nte = nc;
        S->te_neigh = S->neigh;
        S->te_count = S->count;
    }
    int nt = S->nte;
    AL(S->Te, nt, double); AL(S->Ee, nt, double); AL(S->Tl, nt, double);
    AL(S->TsR, nt, double); AL(S->TsL, nt, double); AL(S->Gel, nt, double);
    AL(S->Ges, nt, double); AL(S->sRup, nt, double); AL(S->sRdn, nt, double);
    AL(S->sLup, nt, double); AL(S->sLdn, nt, double); AL(S->ave_p, 3 * nt, double);
#undef AL
    for (int k = 0; k < nt; ++k) {         /* map_cells.cpp:128-158 */
        S->Te[k] = te_K ? te_K[k] * BOLTZ : S->temperature;
        S->Ee[k] = Te_to_Ee(S->Te[k]);
    }

    initial_links(S);
    S->ngroups = colour(nc, S->neigh, &S->gstart, &S->gcells);
    if (prm->te_mesh > 0)
        S->te_ngroups = colour(S->nte, S->te_neigh, &S->te_gstart, &S->te_gcells);
    else {
        S->te_ngroups = S->ngroups;
        S->te_gstart = S->gstart;
        S->te_gcells = S->gcells;
    }
    orc_rho(S);
    orc_force(S);
    if (prm->eltemp) orc_temperature(S);
    S->total_time = 0e0;
    /* random_number_CPU.cpp:38-50, thread 0 */
    S->m_w = 0 + (uint32_t)prm->random_seed;
    S->m_z = 0 * 3 + (uint32_t)prm->random_seed * 2;
    S->spare = 0;
    S->epoch = 0;
    if (prm->eltemp && prm->renormalize) check_energy(S, -1, NULL);
    return S;
}

void orc_destroy(orc_sys* S) {
    if (!S) return;
    for (int k = 0; k < T_COUNT; ++k) free(S->T.t[k]);
    double* dp[] = {S->r, S->p, S->f, S->s, S->s0, S->H, S->HL, S->HC, S->rho, S->pe,
                    S->ke, S->me, S->me0, S->vir, S->stress, S->sumJ, S->lv, S->ave_ff,
                    S->Te, S->Ee, S->Tl, S->TsR, S->TsL, S->Gel, S->Ges, S->sRup,
                    S->sRdn, S->sLup, S->sLdn, S->ave_p, S->qH, S->qnoise};
    for (size_t k = 0; k < sizeof(dp) / sizeof(dp[0]); ++k) free(dp[k]);
    int* ip[] = {S->cell, S->old_cell, S->next, S->prev, S->node, S->head, S->tail,
                 S->count, S->neigh, S->gstart, S->gcells};
    for (size_t k = 0; k < sizeof(ip) / sizeof(ip[0]); ++k) free(ip[k]);
    if (S->P.te_mesh > 0) {
        free(S->te_neigh);
        free(S->te_count);
        free(S->te_gstart);
        free(S->te_gcells);
    }
    free(S);
}

int orc_natom(const orc_sys* S) { return S->n; }
int orc_ncells(const orc_sys* S) { return S->ncells; }
int orc_nte(const orc_sys* S) { return S->nte; }
int orc_ngroups(const orc_sys* S) { return S->ngroups; }
double orc_total_time(const orc_sys* S) { return S->total_time; }

int orc_get(const orc_sys* S, const char* name, double* out) {
    int n = S->n, nt = S->nte;
    struct { const char* k; const double* a; int m; int per_te; } F[] = {
        {"r", S->r, 3, 0}, {"p", S->p, 3, 0}, {"f", S->f, 3, 0}, {"s", S->s, 3, 0},
        {"s0", S->s0, 1, 0}, {"H", S->H, 3, 0}, {"HL", S->HL, 3, 0}, {"rho", S->rho, 1, 0},
        {"pe", S->pe, 1, 0}, {"ke", S->ke, 1, 0}, {"me", S->me, 1, 0}, {"me0", S->me0, 1, 0},
        {"vir", S->vir, 1, 0}, {"sumJ", S->sumJ, 1, 0}, {"stress", S->stress, 6, 0},
        {"Te", S->Te, 1, 1}, {"Ee", S->Ee, 1, 1}, {"Tl", S->Tl, 1, 1}, {"Ts_R", S->TsR, 1, 1},
        {"Ts_L", S->TsL, 1, 1}, {"Gel", S->Gel, 1, 1}, {"Ges", S->Ges, 1, 1}};
    for (size_t k = 0; k < sizeof(F) / sizeof(F[0]); ++k) {
        if (strcmp(F[k].k, name) == 0) {
            int cnt = (F[k].per_te ? nt : n) * F[k].m;
            memcpy(out, F[k].a, sizeof(double) * cnt);
            if (strcmp(name, "Te") == 0)
                for (int i = 0; i < cnt; ++i) out[i] /= BOLTZ;
            return cnt;
        }
    }
    if (strcmp(name, "cell") == 0) { for (int i = 0; i < n; ++i) out[i] = S->cell[i]; return n; }
    if (strcmp(name, "node") == 0) { for (int i = 0; i < n; ++i) out[i] = S->node[i]; return n; }
    if (strcmp(name, "count") == 0) { for (int k = 0; k < nt; ++k) out[k] = S->te_count[k]; return nt; }
    return -1;
}

void orc_lists(const orc_sys* S, int* out) {
    int m = 0;
    for (int c = 0; c < S->ncells; ++c)
        for (int i = S->head[c]; i >= 0; i = S->next[i]) out[m++] = i;
}
