// BF16 GEMM on the 5th-generation tensor cores (tcgen05), FP32 accumulation in
// tensor memory -- the contraction of the learned warm start's convolutions
// (implicit GEMM over im2col tiles, cnn.cu).
//
//   C[M][N] (FP32, row stride ldc) = A[M][K] . B[N][K]^T
//   A, B: BF16 with K contiguous (row strides lda, ldb in elements, multiples of
//   8; K a multiple of 8).
//
// One CTA of 128 threads computes a 128 x BN tile.  Per K block of 64, the four
// warps copy the A and B tiles into shared memory in the canonical K-major
// layout without swizzle (core matrices of 8 rows x 16 bytes; the two core
// matrices of one 16-wide K step LBO bytes apart, consecutive 8-row groups SBO
// bytes apart), one thread issues four tcgen05.mma (M = 128, N = BN, K = 16)
// into a TMEM accumulator of BN columns and commits them to an mbarrier, and
// the CTA waits for that barrier before the tiles are overwritten.  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w .. 32w + 31, i.e. rows 32w .. of the tile).  Every wait is bounded: a
// wait that gives up sets *err and the CTA skips to freeing its TMEM.
#include <cuda_bf16.h>

#include "../../include/maf_b200.h"
#include "capi_internal.hpp"
#include "engine.hpp"

namespace mafb {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr unsigned long long kWaitCycles = 4000000000ull;  // about 2 s at the boost clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0), the
// Blackwell descriptor version 1, addresses and offsets in 16-byte units.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
// M = 128, N = BN.
template <int BN> constexpr uint32_t idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    const unsigned long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

// blockIdx.z = split s of the K range (kchunk values each, a multiple of 64):
// its partial product goes to the slab C + s M ldc.
template <int BN>
__global__ void __launch_bounds__(128) k_umma_gemm(const __nv_bfloat16* __restrict__ A, int lda,
                                                   const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, int M, int N, int K, int kchunk, int* err) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "tile width");
    constexpr uint32_t A_KC = (kBM / 8) * 128;  // bytes between the K chunks of the A tile (LBO)
    constexpr uint32_t B_KC = (BN / 8) * 128;   // of the B tile
    __shared__ __align__(1024) uint8_t sA[kBM * kBK * 2];
    __shared__ __align__(1024) uint8_t sB[BN * kBK * 2];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_sh;
    __shared__ int failed;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const uint32_t mbar_a = smem_u32(&mbar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    uint32_t phase = 0;
    const uint32_t sa = smem_u32(sA), sb = smem_u32(sB);
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(K, kbeg + kchunk);
    C += (int64_t)blockIdx.z * M * ldc;
    for (int k0 = kbeg; k0 < kend; k0 += kBK) {
        // A tile: 128 rows x 8 chunks of 8 BF16 (16 bytes); thread q takes chunk (q & 7) of row q >> 3
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int q = tid + 128 * i, r = q >> 3, kc = q & 7;
            const int gm = m0 + r, gk = k0 + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gm < M && gk < kend) v = *reinterpret_cast<const uint4*>(A + (int64_t)gm * lda + gk);
            *reinterpret_cast<uint4*>(sA + kc * A_KC + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
#pragma unroll
        for (int i = 0; i < BN / 16; ++i) {
            const int q = tid + 128 * i, r = q >> 3, kc = q & 7;
            const int gn = n0 + r, gk = k0 + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gn < N && gk < kend) v = *reinterpret_cast<const uint4*>(B + (int64_t)gn * ldb + gk);
            *reinterpret_cast<uint4*>(sB + kc * B_KC + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
        // the tiles were written through the generic proxy; the MMA reads them through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < kBK / 16; ++s) {
                const uint64_t ad = sdesc(sa + 2 * s * A_KC, A_KC, 128);
                const uint64_t bd = sdesc(sb + 2 * s * B_KC, B_KC, 128);
                const uint32_t acc = (k0 > kbeg || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc<BN>()), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                         : "memory");
        }
        // the MMAs read the tiles: wait for them before the next block overwrites the tiles
        const bool ok = mbar_wait(mbar_a, phase);
        phase ^= 1u;
        if (!ok) atomicExch(&failed, 1);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (failed) break;
    }
    if (!failed) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n < N) C[(int64_t)row * ldc + n] = __uint_as_float(v[j]);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

DevBuf g_umma_err;  // device error flag of the tensor-core GEMM (one per process)

}  // namespace

// Host launcher (nn.cu and the C ABI): the tile width follows N; with splits > 1
// the K range is cut into that many chunks whose partial products land in
// consecutive slabs C + s M ldc (the caller sums them).
void umma_gemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
               cudaStream_t st, bool check, int splits = 1) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    if (splits < 1) splits = 1;
    const int kchunk = (int)ceil_div(ceil_div(K, splits), kBK) * kBK;
    splits = (int)ceil_div(K, kchunk);
    if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N || ((uintptr_t)A | (uintptr_t)B) % 16)
        throw Error(1, "bf16 gemm: K and the row strides must be multiples of 8 elements, rows 16-byte aligned");
    if (!g_umma_err.p) {
        g_umma_err.alloc(sizeof(int));
        MAF_CUDA(cudaMemset(g_umma_err.p, 0, sizeof(int)));
    }
    int* err = g_umma_err.as<int>();
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    const unsigned gx = (unsigned)ceil_div(M, kBM);
    const unsigned gz = (unsigned)splits;
    if (N <= 32) {
        k_umma_gemm<32><<<dim3(gx, 1, gz), 128, 0, st>>>(a, lda, b, ldb, C, ldc, M, N, K, kchunk, err);
    } else if (N <= 64) {
        k_umma_gemm<64><<<dim3(gx, 1, gz), 128, 0, st>>>(a, lda, b, ldb, C, ldc, M, N, K, kchunk, err);
    } else {
        k_umma_gemm<128><<<dim3(gx, (unsigned)ceil_div(N, 128), gz), 128, 0, st>>>(a, lda, b, ldb, C, ldc, M, N, K,
                                                                                    kchunk, err);
    }
    MAF_LAUNCH_CHECK();
    if (check) {
        int e = 0;
        MAF_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        MAF_CUDA(cudaStreamSynchronize(st));
        if (e) {
            MAF_CUDA(cudaMemset(err, 0, sizeof(int)));
            throw Error(5, "bf16 gemm: a tensor-core wait timed out");
        }
    }
}

}  // namespace mafb

extern "C" int maf_bf16_gemm(const void* A_dev, int lda, const void* B_dev, int ldb, float* C_dev, int ldc, int M,
                             int N, int K, void* stream) {
    return mafb::capi_run([&] {
        if (!A_dev || !B_dev || !C_dev) throw mafb::Error(1, "maf_bf16_gemm: NULL argument");
        mafb::umma_gemm(A_dev, lda, B_dev, ldb, C_dev, ldc, M, N, K, static_cast<cudaStream_t>(stream), true);
    });
}
