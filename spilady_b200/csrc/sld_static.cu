// Allocation-free averages over caller-owned device arrays.
//
// The same averages as sld_averages (check_energy_CPU.cpp:33-60,
// check_temperature_CPU.cpp:33-39, check_spin_CPU.cpp:33-53), for callers
// that cannot let this library allocate device memory:
//   - a code whose device memory all comes from its own pool (a caching
//     allocator, or a job that reserves the GPU's memory up front) and so has
//     no room, or no wish, for a library's private cudaMalloc;
//   - a code that cannot afford cudaFree, which waits for all work on the
//     device, in the middle of its own stream-ordered work.
// Its only scratch is the array of per-block partial sums below: a fixed
// file-scope device array, sized for SLD_AVERAGES_STATIC_MAX_ATOMS atoms
// (2 MiB), whose device address is looked up once per device.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "../../include/sld.h"
#include "sld_common.cuh"

#define SLD_STATIC_BLOCK 256
#define SLD_STATIC_MAX_PARTIALS (SLD_AVERAGES_STATIC_MAX_ATOMS / SLD_STATIC_BLOCK)

static_assert(SLD_AVERAGES_STATIC_MAX_ATOMS % SLD_STATIC_BLOCK == 0,
              "the atom limit must be a whole number of blocks");

// 8 slots per block: pe, ke, me, me0, sx, sy, sz, one spare.  Every slot a
// call reads is written earlier in the same call (block b writes slots
// 8b..8b+6 for every b < nb, and the final kernel reads only those), so
// nothing has to start at zero and nothing is cleared.
static __device__ __align__(256) double g_static_partials[SLD_STATIC_MAX_PARTIALS * 8];

namespace {

const int kMaxDevices = 64;
std::atomic<double*> g_scratch[kMaxDevices];

__global__ void __launch_bounds__(SLD_STATIC_BLOCK)
k_avg_static_partials(const double* __restrict__ pe, const double* __restrict__ ke,
                      const double* __restrict__ me, const double* __restrict__ me0,
                      const double* __restrict__ s, int natom, double* __restrict__ part) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < natom) {
        v[0] = pe[i]; v[1] = ke[i]; v[2] = me[i]; v[3] = me0[i];
        v[4] = s[3 * (size_t)i]; v[5] = s[3 * (size_t)i + 1]; v[6] = s[3 * (size_t)i + 2];
    }
    __shared__ double sh[32];
    for (int k = 0; k < 7; ++k) {
        double t = block_sum(v[k], sh);
        if (threadIdx.x == 0) part[8 * (size_t)blockIdx.x + k] = t;
    }
}

__global__ void __launch_bounds__(1024)
k_avg_static_final(const double* __restrict__ part, int nb, int natom, double* __restrict__ out) {
    __shared__ double sh[32];
    double v[7];
    for (int k = 0; k < 7; ++k) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) a += part[8 * (size_t)b + k];
        v[k] = block_sum(a, sh);
    }
    if (threadIdx.x == 0) {
        double n = (double)natom;
        out[0] = v[0] / n;
        out[1] = v[1] / n;
        out[2] = v[2] / n;
        out[3] = v[3] / n;
        out[4] = v[1] * 2.0 / 3.0 / n / SLD_BOLTZ;   // Tl (K), check_temperature_CPU.cpp:37
        out[5] = v[4] / n;
        out[6] = v[5] / n;
        out[7] = v[6] / n;
    }
}

// The device address of the scratch array on the current device.  The
// array's name in host code is only a host-side handle; cudaGetSymbolAddress
// gives the address on the device that is current when it is called.
int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "sld_averages_static: cudaGetDevice failed: %s\n",
                     cudaGetErrorString(e));
        return SLD_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return SLD_ERR_ARG;
    double* p = g_scratch[dev].load(std::memory_order_acquire);
    if (!p) {
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_static_partials);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "sld_averages_static: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return SLD_ERR_CUDA;
        }
        g_scratch[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return SLD_OK;
}

}  // namespace

extern "C" int sld_averages_static(const double* pe, const double* ke, const double* me,
                                   const double* me0, const double* s, int natom,
                                   double* out8, void* stream) {
    if (!pe || !ke || !me || !me0 || !s || !out8 || natom <= 0) return SLD_ERR_ARG;
    if (natom > SLD_AVERAGES_STATIC_MAX_ATOMS) {
        std::fprintf(stderr,
                     "sld_averages_static: %d atoms exceed this entry point's fixed scratch "
                     "(at most %d atoms); use sld_averages instead\n",
                     natom, SLD_AVERAGES_STATIC_MAX_ATOMS);
        return SLD_ERR_CAPACITY;
    }
    double* part = nullptr;
    int rc = scratch_for_current_device(&part);
    if (rc != SLD_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int nb = (natom + SLD_STATIC_BLOCK - 1) / SLD_STATIC_BLOCK;
    k_avg_static_partials<<<nb, SLD_STATIC_BLOCK, 0, st>>>(pe, ke, me, me0, s, natom, part);
    k_avg_static_final<<<1, 1024, 0, st>>>(part, nb, natom, out8);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "sld_averages_static: launch failed: %s\n", cudaGetErrorString(e));
        return SLD_ERR_CUDA;
    }
    return SLD_OK;
}
