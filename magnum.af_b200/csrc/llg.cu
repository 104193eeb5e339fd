// Runge-Kutta stage combine, error norm / candidate update, normalisation and
// small reductions for the adaptive LLG integrator.
//
// Reference: magnumaf/src/integrators/adaptive_runge_kutta.cpp:39-173,496-529
//   stage s:     m_s = m + sum_j a_sj k_j                    (FP64)
//   error norm:  err = max | rk_error / (atol + rtol |max(m, m + sumbk)|) |
//   accept:      m <- normalise(m + sumbk)   (normalize_even_zero_vectors, or
//                the zero-safe normalize when an Ms_field exists)
// magnumaf/src/math.cpp:6-8 (max_4d_abs), magnumaf/src/util/util.cpp:34-42.
#include "engine.hpp"
#include "rk.hpp"
#include "rng.cuh"

namespace mafb {

__global__ void k_combine(const double* __restrict__ m, KList kl, double* __restrict__ out64, float* __restrict__ out32,
                          int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = m[i];
        for (int j = 0; j < kl.n; ++j) acc = acc + kl.c[j] * kl.k[j][i];
        out64[i] = acc;
        if (out32) out32[i] = (float)acc;
    }
}

// The same combine with the number of k's a compile-time constant and two
// values per thread through 16-byte loads: each thread issues its NK + 1
// independent loads before the first use (the generic loop above issues them
// one trip at a time).  Same arithmetic and summation order, so bit-identical.
// Needs n even and 16-byte aligned buffers.
template <int NK>
__global__ void __launch_bounds__(256) k_combine_v(const double* __restrict__ m, KList kl, double* __restrict__ out64,
                                                   float* __restrict__ out32, int64_t n2) {
    const double2* m2 = reinterpret_cast<const double2*>(m);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
        double2 kv[NK];
#pragma unroll
        for (int j = 0; j < NK; ++j) kv[j] = reinterpret_cast<const double2*>(kl.k[j])[i];
        double2 acc = m2[i];
#pragma unroll
        for (int j = 0; j < NK; ++j) {
            acc.x = acc.x + kl.c[j] * kv[j].x;
            acc.y = acc.y + kl.c[j] * kv[j].y;
        }
        reinterpret_cast<double2*>(out64)[i] = acc;
        if (out32) reinterpret_cast<float2*>(out32)[i] = make_float2((float)acc.x, (float)acc.y);
    }
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

void rk_combine(const double* m, const KList& kl, double* out64, float* out32, int64_t n, cudaStream_t st) {
    bool vec = n % 2 == 0 && kl.n >= 1 && kl.n <= 7 && aligned16(m) && aligned16(out64) &&
               (!out32 || ((uintptr_t)out32 & 7) == 0);
    for (int j = 0; j < kl.n; ++j) vec = vec && aligned16(kl.k[j]);
    if (vec) {
        const int64_t n2 = n / 2;
        const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(n2, 256), (int64_t)sm_count() * 16);
        switch (kl.n) {
            case 1: k_combine_v<1><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            case 2: k_combine_v<2><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            case 3: k_combine_v<3><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            case 4: k_combine_v<4><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            case 5: k_combine_v<5><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            case 6: k_combine_v<6><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
            default: k_combine_v<7><<<blocks, 256, 0, st>>>(m, kl, out64, out32, n2); break;
        }
        MAF_LAUNCH_CHECK();
        return;
    }
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_combine<<<(unsigned)blocks, 256, 0, st>>>(m, kl, out64, out32, n);
    MAF_LAUNCH_CHECK();
}

// max with NaN propagation (NaN wins)
__device__ __forceinline__ double nanmax(double a, double b) {
    if (a != a) return a;
    if (b != b) return b;
    return a > b ? a : b;
}

__device__ __forceinline__ void block_max_store(double v, double* partials) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s = nanmax(s, __shfl_down_sync(0xffffffffu, s, o));
        if (lane == 0) partials[blockIdx.x] = s;
    }
}

// sumbk = sum bs_j k_j ; rk_error = (form 0) sum e_j k_j  or (form 1) sumbk - sum e_j k_j
__global__ void k_finalize(const double* __restrict__ m, KList kb, KList ke, int form, double atol, double rtol,
                           double* __restrict__ mcand, int norm_mode, int64_t N, double* __restrict__ partials) {
    double vmax = 0.0;
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        double out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * N + cell;
            double sumbk = kb.c[0] * kb.k[0][i];
            for (int j = 1; j < kb.n; ++j) sumbk = sumbk + kb.c[j] * kb.k[j][i];
            double e = ke.c[0] * ke.k[0][i];
            for (int j = 1; j < ke.n; ++j) e = e + ke.c[j] * ke.k[j][i];
            const double err = form == 0 ? e : sumbk - e;
            const double mi = m[i];
            const double mn = mi + sumbk;
            const double mx = mi > mn ? mi : mn;  // af::max(m, m + sumbk)
            const double sc = atol + rtol * fabs(mx);
            vmax = nanmax(vmax, fabs(err / sc));
            out[c] = mn;
        }
        if (norm_mode == 1) {
            const double nrm = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
            out[0] /= nrm; out[1] /= nrm; out[2] /= nrm;
        } else if (norm_mode == 2) {
            const double nrm = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
            if (nrm != 0) { out[0] /= nrm; out[1] /= nrm; out[2] /= nrm; }
            else { out[0] = 0; out[1] = 0; out[2] = 0; }
        }
        mcand[cell] = out[0];
        mcand[N + cell] = out[1];
        mcand[2 * N + cell] = out[2];
    }
    block_max_store(vmax, partials);
}

__global__ void k_max_partials(const double* __restrict__ p, int n, double* out) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v = nanmax(v, p[i]);
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s = nanmax(s, __shfl_down_sync(0xffffffffu, s, o));
        if (threadIdx.x == 0) *out = s;
    }
}

// The union of the b- and e-lists' k buffers, each loaded once: k[j] enters
// sumbk with cb[j] and the error sum with ce[j] (a zero coefficient: not in
// that list).  The lists' own orders are kept (checked by the caller), so the
// sums are formed in the same order as in k_finalize.
struct KUnion {
    const double* k[8] = {};
    double cb[8] = {};
    double ce[8] = {};
    int n = 0;
};

__device__ __forceinline__ double fin_one(double sumbk, double e, int form, double mi, double atol, double rtol,
                                          double& vmax) {
    const double err = form == 0 ? e : sumbk - e;
    const double mn = mi + sumbk;
    const double mx = mi > mn ? mi : mn;  // af::max(m, m + sumbk)
    const double sc = atol + rtol * fabs(mx);
    vmax = nanmax(vmax, fabs(err / sc));
    return mn;
}

__device__ __forceinline__ void fin_norm(double* o, int norm_mode) {
    if (norm_mode == 1) {
        const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        o[0] /= nrm; o[1] /= nrm; o[2] /= nrm;
    } else if (norm_mode == 2) {
        const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        if (nrm != 0) { o[0] /= nrm; o[1] /= nrm; o[2] /= nrm; }
        else { o[0] = 0; o[1] = 0; o[2] = 0; }
    }
}

// k_finalize with NU union buffers known at compile time and two cells per
// thread through 16-byte loads (N even, 16-byte aligned buffers); same
// arithmetic as k_finalize, bit-identical results.
template <int NU>
__global__ void __launch_bounds__(256) k_finalize_v(const double* __restrict__ m, KUnion ku, int form, double atol,
                                                    double rtol, double* __restrict__ mcand, int norm_mode, int64_t N,
                                                    double* __restrict__ partials) {
    const int64_t N2 = N / 2;
    double vmax = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N2; p += (int64_t)gridDim.x * blockDim.x) {
        double o0[3], o1[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * N2 + p;
            double2 kv[NU];
#pragma unroll
            for (int j = 0; j < NU; ++j) kv[j] = reinterpret_cast<const double2*>(ku.k[j])[i];
            const double2 mi = reinterpret_cast<const double2*>(m)[i];
            double b0 = 0.0, b1 = 0.0, e0 = 0.0, e1 = 0.0;
#pragma unroll
            for (int j = 0; j < NU; ++j) {
                if (ku.cb[j] != 0.0) {
                    b0 = b0 + ku.cb[j] * kv[j].x;
                    b1 = b1 + ku.cb[j] * kv[j].y;
                }
                if (ku.ce[j] != 0.0) {
                    e0 = e0 + ku.ce[j] * kv[j].x;
                    e1 = e1 + ku.ce[j] * kv[j].y;
                }
            }
            o0[c] = fin_one(b0, e0, form, mi.x, atol, rtol, vmax);
            o1[c] = fin_one(b1, e1, form, mi.y, atol, rtol, vmax);
        }
        fin_norm(o0, norm_mode);
        fin_norm(o1, norm_mode);
#pragma unroll
        for (int c = 0; c < 3; ++c) reinterpret_cast<double2*>(mcand)[c * N2 + p] = make_double2(o0[c], o1[c]);
    }
    block_max_store(vmax, partials);
}

// Union of the two lists with each list's order preserved, or false.
static bool make_union(const KList& kb, const KList& ke, KUnion& u) {
    for (int j = 0; j < kb.n; ++j) {
        if (kb.c[j] == 0.0) return false;
        u.k[u.n] = kb.k[j];
        u.cb[u.n] = kb.c[j];
        ++u.n;
    }
    int last = -1;
    for (int j = 0; j < ke.n; ++j) {
        if (ke.c[j] == 0.0) continue;  // adds nothing to the error sum
        int at = -1;
        for (int q = 0; q < u.n; ++q)
            if (u.k[q] == ke.k[j]) at = q;
        if (at < 0) {
            if (u.n == 8) return false;
            at = u.n++;
            u.k[at] = ke.k[j];
        }
        if (at <= last) return false;  // the e-list's order would change
        u.ce[at] = ke.c[j];
        last = at;
    }
    return u.n >= 1 && u.n <= 7;
}

int rk_finalize(const double* m, const KList& kb, const KList& ke, int form, double atol, double rtol, double* mcand,
                int norm_mode, int64_t N, double* partials, double* err_dev, cudaStream_t st) {
    const int threads = 256;
    KUnion u;
    bool vec = N % 2 == 0 && aligned16(m) && aligned16(mcand) && make_union(kb, ke, u);
    for (int j = 0; vec && j < u.n; ++j) vec = aligned16(u.k[j]);
    int blocks;
    if (vec) {
        blocks = (int)std::min<int64_t>(ceil_div(N / 2, threads), (int64_t)sm_count() * 8);
        switch (u.n) {
            case 1: k_finalize_v<1><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            case 2: k_finalize_v<2><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            case 3: k_finalize_v<3><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            case 4: k_finalize_v<4><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            case 5: k_finalize_v<5><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            case 6: k_finalize_v<6><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
            default: k_finalize_v<7><<<blocks, threads, 0, st>>>(m, u, form, atol, rtol, mcand, norm_mode, N, partials); break;
        }
    } else {
        blocks = (int)std::min<int64_t>(ceil_div(N, threads), (int64_t)sm_count() * 8);
        k_finalize<<<blocks, threads, 0, st>>>(m, kb, ke, form, atol, rtol, mcand, norm_mode, N, partials);
    }
    MAF_LAUNCH_CHECK();
    k_max_partials<<<1, 256, 0, st>>>(partials, blocks, err_dev);
    MAF_LAUNCH_CHECK();
    return blocks;
}

// normalize_handle_zero_vectors (util.cpp:37-42); counts cells of zero norm
__global__ void k_normalize(double* __restrict__ m, int64_t N, int mode, unsigned long long* zero_count) {
    unsigned long long z = 0;
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        double a = m[cell], b = m[N + cell], c = m[2 * N + cell];
        const double nrm = sqrt(a * a + b * b + c * c);
        if (mode == 1) {
            a /= nrm; b /= nrm; c /= nrm;
        } else if (nrm != 0) {
            a /= nrm; b /= nrm; c /= nrm;
        } else {
            a = 0; b = 0; c = 0;
            ++z;
        }
        m[cell] = a;
        m[N + cell] = b;
        m[2 * N + cell] = c;
    }
    if (zero_count && z) atomicAdd(zero_count, z);
}

void normalize_m(double* m, int64_t N, int mode, unsigned long long* zero_count_dev, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(N, 256), (int64_t)sm_count() * 8);
    k_normalize<<<(unsigned)blocks, 256, 0, st>>>(m, N, mode, zero_count_dev);
    MAF_LAUNCH_CHECK();
}

// Ms_field = Ms * (|m| != 0)   (state.cpp:71-89)
__global__ void k_ms_from_m(const double* __restrict__ m, double Ms, double* __restrict__ msf, float* __restrict__ msf32,
                            int64_t N) {
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        const double a = m[cell], b = m[N + cell], c = m[2 * N + cell];
        const double v = (sqrt(a * a + b * b + c * c) != 0) ? Ms : 0.0;
        msf[cell] = v;
        if (msf32) msf32[cell] = (float)v;
    }
}

void ms_field_from_m(const double* m, double Ms, double* msf, float* msf32, int64_t N, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(N, 256), (int64_t)sm_count() * 8);
    k_ms_from_m<<<(unsigned)blocks, 256, 0, st>>>(m, Ms, msf, msf32, N);
    MAF_LAUNCH_CHECK();
}

// <m>: per-block sums of the three components and of the nonzero-cell count,
// then a fixed-order final pass (state.cpp:32-43).
__global__ void k_mean_partials(const double* __restrict__ m, int64_t N, double* __restrict__ part) {
    double s0 = 0, s1 = 0, s2 = 0, cnt = 0;
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        const double a = m[cell], b = m[N + cell], c = m[2 * N + cell];
        s0 += a;
        s1 += b;
        s2 += c;
        cnt += (sqrt(a * a + b * b + c * c) != 0) ? 1.0 : 0.0;
    }
    __shared__ double red[4][32];
    double v[4] = {s0, s1, s2, cnt};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) red[q][wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = lane < nw ? red[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) part[4 * blockIdx.x + q] = s;
        }
    }
}

__global__ void k_mean_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s[4] = {0, 0, 0, 0};
        for (int b = 0; b < nb; ++b)
            for (int q = 0; q < 4; ++q) s[q] += part[4 * b + q];
        out[0] = s[0] / s[3];
        out[1] = s[1] / s[3];
        out[2] = s[2] / s[3];
    }
}

int mean_m_blocks() { return 2 * sm_count(); }

void mean_m(const double* m, int64_t N, double* scratch, double* out_dev, cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>(ceil_div(N, 256), mean_m_blocks());
    k_mean_partials<<<blocks, 256, 0, st>>>(m, N, scratch);
    MAF_LAUNCH_CHECK();
    k_mean_final<<<1, 32, 0, st>>>(scratch, blocks, out_dev);
    MAF_LAUNCH_CHECK();
}

// (a - b) -> d, with sum of squares partials (for the string method's Frobenius norm)
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

void f32_to_f64(const float* a, double* b, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_f2d<<<(unsigned)blocks, 256, 0, st>>>(a, b, n);
    MAF_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// vector operations of the LBFGS minimiser (lbfgs_minimizer.cpp:44-46, 96-177)
// ---------------------------------------------------------------------------
// reduction blocks of the LBFGS vector operations (partials at scratch[0, n),
// the result at scratch[n])
int red_blocks() { return 2 * sm_count(); }

// per-block partials: mode 0 sum a*b, mode 1 max |a| (NaN-propagating),
// mode 2 sum (a-b)^2 (the string method's Frobenius norm of image differences)
__global__ void k_red_partials(const double* __restrict__ a, const double* __restrict__ b, int64_t n, int mode,
                               double* __restrict__ part) {
    double v = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mode == 0) {
            v += a[i] * b[i];
        } else if (mode == 2) {
            const double d = a[i] - b[i];
            v += d * d;
        } else {
            v = nanmax(v, fabs(a[i]));
        }
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_down_sync(0xffffffffu, v, o);
        v = mode != 1 ? v + w : nanmax(v, w);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, s, o);
            s = mode != 1 ? s + w : nanmax(s, w);
        }
        if (lane == 0) part[blockIdx.x] = s;
    }
}

__global__ void k_red_final(const double* __restrict__ part, int nb, int mode, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < nb; ++i) s = mode != 1 ? s + part[i] : nanmax(s, part[i]);
        *out = s;
    }
}

double reduce_host(const double* a, const double* b, int64_t n, int mode, double* scratch, cudaStream_t st) {
    const int nred = red_blocks();
    const int blocks = (int)std::min<int64_t>(ceil_div(n, 256), nred);
    k_red_partials<<<blocks, 256, 0, st>>>(a, b, n, mode, scratch);
    MAF_LAUNCH_CHECK();
    k_red_final<<<1, 32, 0, st>>>(scratch, blocks, mode, scratch + nred);
    MAF_LAUNCH_CHECK();
    double v = 0;
    MAF_CUDA(cudaMemcpyAsync(&v, scratch + nred, sizeof(double), cudaMemcpyDeviceToHost, st));
    MAF_CUDA(cudaStreamSynchronize(st));
    return v;
}

double dot_host(const double* a, const double* b, int64_t n, double* scratch, cudaStream_t st) {
    return reduce_host(a, b, n, 0, scratch, st);
}

void reduce_dev(const double* a, const double* b, int64_t n, int mode, double* scratch, double* out, cudaStream_t st) {
    const int nred = red_blocks();
    const int blocks = (int)std::min<int64_t>(ceil_div(n, 256), nred);
    k_red_partials<<<blocks, 256, 0, st>>>(a, b, n, mode, scratch);
    MAF_LAUNCH_CHECK();
    k_red_final<<<1, 32, 0, st>>>(scratch, blocks, mode, out);
    MAF_LAUNCH_CHECK();
}

void dot_dev(const double* a, const double* b, int64_t n, double* scratch, double* out, cudaStream_t st) {
    reduce_dev(a, b, n, 0, scratch, out, st);
}

double maxabs_host(const double* a, int64_t n, double* scratch, cudaStream_t st) {
    return reduce_host(a, nullptr, n, 1, scratch, st);
}

double sqdiff_host(const double* a, const double* b, int64_t n, double* scratch, cudaStream_t st) {
    return reduce_host(a, b, n, 2, scratch, st);
}

// out = a + (c1 * (b - a)) / c2, the string method's linear re-interpolation
// in the reference's order of operations (string_method.cpp:94-95)
__global__ void k_lerp(double* __restrict__ out, const double* __restrict__ a, const double* __restrict__ b, double c1,
                       double c2, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] + (c1 * (b[i] - a[i])) / c2;
}

void lerp(double* out, const double* a, const double* b, double c1, double c2, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_lerp<<<(unsigned)blocks, 256, 0, st>>>(out, a, b, c1, c2, n);
    MAF_LAUNCH_CHECK();
}

__global__ void k_inc_counter(unsigned long long* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *c += 1;
}

void inc_counter(unsigned long long* c, cudaStream_t st) {
    k_inc_counter<<<1, 32, 0, st>>>(c);
    MAF_LAUNCH_CHECK();
}

__global__ void k_axpby(double* out, double a, const double* x, double b, const double* y, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = a * x[i];
        out[i] = y ? v + b * y[i] : v;
    }
}

void axpby(double* out, double a, const double* x, double b, const double* y, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_axpby<<<(unsigned)blocks, 256, 0, st>>>(out, a, x, b, y, n);
    MAF_LAUNCH_CHECK();
}

// k_axpby with a = 1 and the coefficient formed on the device from the dot
// product *d (every thread forms the same value)
__global__ void k_axpby_rho(double* q, const double* __restrict__ y, const double* __restrict__ d, double rho,
                            const double* __restrict__ alpha_in, double* __restrict__ alpha_out, int64_t n) {
    const double t = rho * *d;
    const double b = alpha_in ? *alpha_in - t : -t;
    if (alpha_out && blockIdx.x == 0 && threadIdx.x == 0) *alpha_out = t;
    const double a = 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = a * q[i];
        q[i] = v + b * y[i];
    }
}

void axpby_rho(double* q, const double* y, const double* d, double rho, const double* alpha_in, double* alpha_out,
               int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_axpby_rho<<<(unsigned)blocks, 256, 0, st>>>(q, y, d, rho, alpha_in, alpha_out, n);
    MAF_LAUNCH_CHECK();
}

// m = normalize(wa + stp * s) with the zero-safe normalize (lbfgs_minimizer.cpp:274-275)
__global__ void k_normalize_combine(double* __restrict__ m, const double* __restrict__ wa, double stp,
                                    const double* __restrict__ s, int64_t N) {
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        double v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = wa[c * N + cell] + stp * s[c * N + cell];
        const double nrm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) m[c * N + cell] = nrm != 0 ? v[c] / nrm : 0.0;
    }
}

void normalize_combine(double* m, const double* wa, double stp, const double* s, int64_t N, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(N, 256), (int64_t)sm_count() * 8);
    k_normalize_combine<<<(unsigned)blocks, 256, 0, st>>>(m, wa, stp, s, N);
    MAF_LAUNCH_CHECK();
}

// thermal field sigma * xi(seed, member, index, cell) [3][N] (the h_th of
// stochastic_integrator.cpp:11 as this library draws it)
__global__ void k_noise(double* __restrict__ out, int64_t N, double sigma, unsigned long long seed, unsigned member,
                        unsigned long long index) {
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        double xi[3];
        normal3(seed, member, index, (uint64_t)cell, xi);
        out[cell] = sigma * xi[0];
        out[N + cell] = sigma * xi[1];
        out[2 * N + cell] = sigma * xi[2];
    }
}

void thermal_field(double* out, int64_t N, double sigma, unsigned long long seed, unsigned member,
                   unsigned long long index, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(N, 256), (int64_t)sm_count() * 8);
    k_noise<<<(unsigned)blocks, 256, 0, st>>>(out, N, sigma, seed, member, index);
    MAF_LAUNCH_CHECK();
}

}  // namespace mafb
