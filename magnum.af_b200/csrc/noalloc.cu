// Mean magnetisation that allocates no device memory.
//
// maf_mean_m_noalloc computes the same quantity as maf_state_mean_m -- the
// sum of m over all cells divided by the number of cells with |m| != 0
// (magnumaf/src/state.cpp:39-45) -- for any FP64 field m[3][ncells] that
// already lives on the device.  maf_state_mean_m draws its block partials from
// a per-state buffer that it grows with cudaMalloc; this variant takes them
// from the fixed static device array below instead, so it can be called by
// code that must not allocate: a monitor that samples <m> between steps while
// other streams run (cudaMalloc may synchronise the whole device), or a host
// application that has already reserved all free device memory for its own
// pool.
//
// Scratch layout (g_noalloc_scratch, 128 KiB + 32 B, one copy per device):
//   [0, 4 * kMaxBlocks)        partial sums (mx, my, mz, nonzero count) per block
//   [4 * kMaxBlocks, + 4)      the three means (and one unused slot)
// Every partial that the combine pass reads is written by the chunk pass of the
// same call, and the result slots are written before they are copied out, so
// nothing in the scratch has to start at zero.
//
// Two calls whose work overlaps on the device (different streams or host
// threads on the same device, without ordering between them) share this one
// scratch array and race: their partial sums overwrite each other and both
// results are undefined.  Calls on the same stream are ordered and safe.
#include <string>

#include "../../include/maf_b200.h"
#include "capi_internal.hpp"
#include "common.cuh"

using namespace mafb;

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 32;
constexpr long long kCellsPerBlock = (long long)kThreads * kCellsPerThread;  // 8192
constexpr int kMaxBlocks = 4096;
constexpr long long kMaxCells = kCellsPerBlock * kMaxBlocks;  // 33,554,432 cells
constexpr int kResult = 4 * kMaxBlocks;

__device__ __align__(256) double g_noalloc_scratch[4 * kMaxBlocks + 4];

// Block b sums cells [b * kCellsPerBlock, min(N, (b + 1) * kCellsPerBlock)).
__global__ void __launch_bounds__(kThreads) k_mean_chunks(const double* __restrict__ m, long long N,
                                                          double* __restrict__ part) {
    const long long c0 = (long long)blockIdx.x * kCellsPerBlock;
    const long long c1 = c0 + kCellsPerBlock < N ? c0 + kCellsPerBlock : N;
    double v[4] = {0, 0, 0, 0};
    for (long long cell = c0 + threadIdx.x; cell < c1; cell += kThreads) {
        const double a = m[cell], b = m[N + cell], c = m[2 * N + cell];
        v[0] += a;
        v[1] += b;
        v[2] += c;
        v[3] += (sqrt(a * a + b * b + c * c) != 0) ? 1.0 : 0.0;
    }
    __shared__ double red[4][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) red[q][wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = lane < kThreads / 32 ? red[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) part[4 * blockIdx.x + q] = s;
        }
    }
}

// One block of 1024 threads: thread t sums partials t, t + 1024, ... in order,
// then a fixed shuffle/shared-memory tree; the result does not depend on timing.
__global__ void __launch_bounds__(1024) k_mean_combine(const double* __restrict__ part, int nb,
                                                       double* __restrict__ out) {
    double v[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += 1024)
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] += part[4 * b + q];
    __shared__ double red[4][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) red[q][wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
        double s[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            s[q] = red[q][lane];
            for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
        }
        if (lane == 0) {
            out[0] = s[0] / s[3];
            out[1] = s[1] / s[3];
            out[2] = s[2] / s[3];
            out[3] = s[3];
        }
    }
}

// Address of the current device's copy of g_noalloc_scratch.  The lookup is
// repeated on every call instead of being cached: a symbol address belongs to
// the current CUDA context, and a cached one would dangle after
// cudaDeviceReset or under another context.  Once this file's module is
// loaded in the context the lookup allocates nothing.
double* scratch_for_current_context() {
    void* p = nullptr;
    MAF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    return static_cast<double*>(p);
}

}  // namespace

// CUDA loads the module of this file (its code and the static scratch array)
// lazily, on the first use in a context, and that load allocates device memory
// and may synchronise the device.  maf_state_create calls this, so the load
// happens when the first state is created on a device -- a call that allocates
// anyway -- and maf_mean_m_noalloc's own calls then allocate nothing.
void mafb::noalloc_prepare_current_device() {
    (void)scratch_for_current_context();
    cudaFuncAttributes attr;
    MAF_CUDA(cudaFuncGetAttributes(&attr, k_mean_chunks));
    MAF_CUDA(cudaFuncGetAttributes(&attr, k_mean_combine));
}

extern "C" int maf_mean_m_noalloc(const double* m_dev, long long ncells, double out[3], void* cuda_stream) {
    return capi_run([&] {
        if (!m_dev || !out) throw Error(MAF_ERR_BADARG, "maf_mean_m_noalloc: NULL argument");
        if (ncells <= 0) throw Error(MAF_ERR_BADARG, "maf_mean_m_noalloc: ncells must be positive");
        if (ncells > kMaxCells)
            throw Error(MAF_ERR_BADARG, "maf_mean_m_noalloc: ncells = " + std::to_string(ncells) +
                                            " exceeds the fixed scratch limit of " + std::to_string(kMaxCells) +
                                            " cells; use maf_state_mean_m for larger meshes");
        double* scr = scratch_for_current_context();
        cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
        const int nb = (int)((ncells + kCellsPerBlock - 1) / kCellsPerBlock);
        k_mean_chunks<<<nb, kThreads, 0, st>>>(m_dev, ncells, scr);
        MAF_LAUNCH_CHECK();
        k_mean_combine<<<1, 1024, 0, st>>>(scr, nb, scr + kResult);
        MAF_LAUNCH_CHECK();
        MAF_CUDA(cudaMemcpyAsync(out, scr + kResult, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        MAF_CUDA(cudaStreamSynchronize(st));
    });
}
