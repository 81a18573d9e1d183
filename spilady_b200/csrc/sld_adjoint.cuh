// Device buffers and kernel launchers of the adjoint (k_adjoint.cu), used by
// the entry points in sld_adjoint.cu.
#pragma once
#include "sld_adjpot.cuh"

struct AdjDev {
    double* rho;        // densities of the parameterised potential
    double* dF;         // F'(rho)
    double* e;          // per-atom energy pe + me + me0
    double4* H;         // exchange field (the loss's field)
    double* part;       // block partials [E, L]
    // adjoints (x, y, z; w unused)
    double4 *rb, *pb, *sb, *fb, *hb;
    double* rhob;
    double* thb;        // block partials of theta's adjoint [blocks][36]
    double* theta_bar;  // running total [36]
    const int* cell_group;   // colour group of each link cell
};

void adj_rho(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st);
void adj_force(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st, double* el2);
void adj_sweep(const Dev& D, const AdjConst& K, cudaStream_t st, const int* cells, int n, double dt,
               bool backward);
void adj_kick(const Dev& D, cudaStream_t st, double h, double4* ppre);
void adj_jacobians(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st, double* drho,
                   double* df, double* dh);
void adj_energy_grad(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st);
void adj_force_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st);
void adj_field_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st);
void adj_rho_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st);
void adj_sweep_rev(const Dev& D, const AdjDev& A, const AdjConst& K, cudaStream_t st,
                   const int* cells, int n, double dt, bool backward, int group, const double4* s0,
                   const double4* s1);
void adj_theta_flush(const AdjDev& A, cudaStream_t st, int nb);
void adj_kick_rev(const Dev& D, const AdjDev& A, cudaStream_t st, double h, const double4* ppre);
void adj_drift_rev(const Dev& D, const AdjDev& A, cudaStream_t st, double dt);
void adj_seed_loss(const Dev& D, const AdjDev& A, cudaStream_t st);
