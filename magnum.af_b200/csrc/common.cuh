// Shared device/host helpers for the magnum.af B200 field/time-step library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace mafb {

constexpr double kMu0 = 4e-7 * 3.14159265358979323846;   // constants.hpp:11
constexpr double kPi = 3.14159265358979323846;
constexpr double kGamma = 1.760859644e11 * kMu0;          // constants.hpp:13
constexpr double kHbar = 1.0545718e-34;                   // constants.hpp:22
constexpr double kEneg = -1.6021766208e-19;               // constants.hpp:17
constexpr double kKb = 1.38064852e-23;                    // constants.hpp:22

// Library error carrying a C-ABI status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

#define MAF_CUDA(call)                                                                               \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            throw ::mafb::Error(e_ == cudaErrorMemoryAllocation ? 3 : 2,                             \
                                std::string(#call " failed: ") + cudaGetErrorString(e_) + " at " +   \
                                    __FILE__ + ":" + std::to_string(__LINE__));                      \
        }                                                                                            \
    } while (0)

#define MAF_LAUNCH_CHECK() MAF_CUDA(cudaGetLastError())

// ---------------------------------------------------------------------------
// complex arithmetic on float2/double2
// ---------------------------------------------------------------------------
template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };
template <typename R> using cplx_t = typename Cplx<R>::T;

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
    return mk(a.x * s, a.y * s);
}
// multiply by -i (forward) or +i (inverse): dir = -1 -> -i, dir = +1 -> +i
template <int DIR, typename C> __host__ __device__ __forceinline__ C cmul_i(C a) {
    return DIR < 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Streaming multiprocessors of the current device, queried once per device
// ordinal (grid sizes of the grid-stride kernels and the reduction partial
// buffers sized from them).
inline int sm_count() {
    constexpr int kMaxOrdinals = 64;
    static int cache[kMaxOrdinals] = {};
    int dev = 0;
    MAF_CUDA(cudaGetDevice(&dev));
    int v = (dev >= 0 && dev < kMaxOrdinals) ? __atomic_load_n(&cache[dev], __ATOMIC_RELAXED) : 0;
    if (v <= 0) {
        MAF_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        if (dev >= 0 && dev < kMaxOrdinals) __atomic_store_n(&cache[dev], v, __ATOMIC_RELAXED);
    }
    return v;
}

}  // namespace mafb
