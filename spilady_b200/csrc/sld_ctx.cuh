// The context behind the C ABI's opaque sld_ctx: parameters, host
// geometry, the device state and the captured step graphs.  Shared by the
// files that implement entry points (sld_api.cu, sld_adjoint.cu).
#pragma once
#include <vector>

#include "../../include/sld.h"
#include "sld_common.cuh"
#include "sld_host.h"

struct sld_ctx {
    sld_params P{};
    sld::HostGeom G;
    std::vector<int> id_of_slot, slot_of_id;
    Dev D{};
    std::vector<void*> allocs;
    std::vector<size_t> alloc_bytes;   // size of each allocation (a whole-state snapshot)
    int* d_gcells = nullptr;
    // the spin-lattice step's magnetic forces, virial and stress, kept apart
    // from the EAM part formed beside them (Dev::fm)
    double4* fm = nullptr;
    double* virm = nullptr;
    double* stressm = nullptr;
    double* d_stage = nullptr;     // sld_get's device staging (6 doubles per atom), made
                                   // at its first use
    SweepFlow flow{};                  // data-flow schedule of the spin sweeps
    int* d_te_gcells = nullptr;
    int* d_te_gstart = nullptr;
    unsigned char* d_te_color = nullptr;
    unsigned short* d_te_ltasks = nullptr;
    uint4* d_te_lnb = nullptr;
    int* d_te_lstart = nullptr;
    double* d_avg = nullptr;
    double* d_chk = nullptr;           // check() sums: per-block partials, then totals
    double4* hext_buf = nullptr;       // external field / force per atom, slot order;
    double4* fext_buf = nullptr;       // D.hext / D.fext point here while set
    // what the last sld_check printed and the barostats read (check_pressure,
    // check_stress), and the barostats' clocks (initial.cpp:92-97)
    double pressure0 = 0.0, ave_stress[6] = {0, 0, 0, 0, 0, 0};
    double last_t_pressure = 0.0, last_t_stress = 0.0;
    // box volume of the last force pass: its local volume V/N per atom
    // (calculate_force_energy_CPU.cpp:276) stays until the next force pass
    double force_volume = 0.0;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;        // second branch of the step graph
    cudaEvent_t fork_ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t step_graph = nullptr;
    cudaGraphExec_t step_graphs[2] = {nullptr, nullptr};   // by current buffer set
    // exchange lists and rho are double buffered: the list pass of a step
    // writes the other set while the first spin sweep still reads this one
    int cur = 0;
    int* jl_set[2] = {nullptr, nullptr};
    int* jln_set[2] = {nullptr, nullptr};
    double* jv_set[2] = {nullptr, nullptr};
    float* jvf_set[2] = {nullptr, nullptr};
    unsigned char* jlk_set[2] = {nullptr, nullptr};
    double* rho_set[2] = {nullptr, nullptr};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int scan_blocks = 1;
    int red_cap = 0;
    bool lists_stale = false;   // positions moved since the neighbour lists were built
    bool groups_ordered = false;   // colour groups ordered by cell counts (first set_state)

    template <class T>
    int alloc(T** p, size_t n) {
        void* q = nullptr;
        if (n == 0) n = 1;
        if (cudaMalloc(&q, n * sizeof(T)) != cudaSuccess) return SLD_ERR_NOMEM;
        // cleared on the default stream, which does not order against the
        // engine's non-blocking streams: finished before any use of it there
        if (cudaMemset(q, 0, n * sizeof(T)) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
            cudaFree(q);
            return SLD_ERR_CUDA;
        }
        allocs.push_back(q);
        alloc_bytes.push_back(n * sizeof(T));
        *p = static_cast<T*>(q);
        return SLD_OK;
    }
};

// Makes the context's device current for the duration of an entry point and
// gives the caller's current device back afterwards: a context's buffers,
// streams and graphs belong to the device it was created on, whatever device
// the calling thread has made current since.
struct DevGuard {
    int prev = -1;
    bool ok = true;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
        else prev = -1;   // already current: nothing to give back
    }
    ~DevGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DevGuard(const DevGuard&) = delete;
    DevGuard& operator=(const DevGuard&) = delete;
};
#define SLD_DEVICE_OF(c)                 \
    DevGuard sld_dev_guard_((c)->P.device); \
    if (!sld_dev_guard_.ok) return SLD_ERR_CUDA

// the device state with buffer set k of the exchange lists and rho
inline Dev dev_set(const sld_ctx* c, int k) {
    Dev D = c->D;
    D.jl = c->jl_set[k];
    D.jl_n = c->jln_set[k];
    D.jv = c->jv_set[k];
    D.jvf = c->jvf_set[k];
    D.jlk = c->jlk_set[k];
    D.rho = c->rho_set[k];
    return D;
}
