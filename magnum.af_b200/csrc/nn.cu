// Layer kernels of the warm-start U-net (magnumaf/warmstart.py): pixel-major
// (NHWC) activations, 3x3 convolutions as im2col + the tensor-core BF16 GEMM of
// umma.cu with FP32 accumulation, bias/ReLU epilogues, 2x2 average pooling,
// nearest 2x upsampling with skip concatenation, their backward passes and
// Adam.  A pixel p = (b, y, x) is row p = (b H + y) W + x; a layer's channel
// count C is padded to Cp (a multiple of 8) in the BF16 tensors that feed a
// GEMM, the padding is zero.  Every reduction runs in a fixed order, so
// training is deterministic.
#include <cuda_bf16.h>

#include "../../include/maf_b200.h"
#include "capi_internal.hpp"
#include "engine.hpp"

namespace mafb {
void umma_gemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
               cudaStream_t st, bool check, int splits);
}

using namespace mafb;

namespace {

using bf16 = __nv_bfloat16;
constexpr int kT = 256;

unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>(ceil_div(n, kT), (int64_t)sm_count() * 32); }

#define GRID_STRIDE(i, n) for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// x [B][C][H][W] (FP32, channels first) -> act [P][Cp] BF16 (zero padded) and
// the magnetisation channels 0..2 as m [P][3] FP32
__global__ void k_in(const float* __restrict__ x, int B, int C, int H, int W, int Cp, bf16* __restrict__ act,
                     float* __restrict__ m) {
    const int64_t HW = (int64_t)H * W, P = B * HW;
    GRID_STRIDE(i, P * Cp) {
        const int64_t p = i / Cp;
        const int c = (int)(i - p * Cp);
        const int64_t b = p / HW, r = p - b * HW;
        const float v = c < C ? x[(b * C + c) * HW + r] : 0.f;
        act[i] = __float2bfloat16_rn(v);
        if (c < 3) m[p * 3 + c] = v;
    }
}

// im2col: col[p][t Cp + c] = act[pixel (y + t/3 - 1, x + t%3 - 1)][c] (zero outside);
// transposed: colT[t Cp + c][p].  Eight channels (16 bytes) per item.
__global__ void k_im2col(const bf16* __restrict__ act, int B, int H, int W, int Cp, bf16* __restrict__ col,
                         int transposed) {
    const int64_t HW = (int64_t)H * W, P = B * HW;
    const int c8 = Cp / 8;
    GRID_STRIDE(i, P * 9 * c8) {
        int64_t p;
        int t, cc;
        if (transposed) {  // consecutive items: consecutive pixels of one (t, channel group)
            p = i % P;
            const int64_t q = i / P;
            t = (int)(q / c8);
            cc = (int)(q - (int64_t)t * c8);
        } else {
            p = i / (9 * c8);
            const int q = (int)(i - p * 9 * c8);
            t = q / c8;
            cc = q - t * c8;
        }
        const int64_t b = p / HW, r = p - b * HW;
        const int y = (int)(r / W) + t / 3 - 1, x = (int)(r % W) + t % 3 - 1;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (y >= 0 && y < H && x >= 0 && x < W)
            v = *reinterpret_cast<const uint4*>(act + ((b * H + y) * W + x) * Cp + cc * 8);
        if (transposed) {
            const bf16* e = reinterpret_cast<const bf16*>(&v);
            const int64_t k0 = (int64_t)t * Cp + cc * 8;
#pragma unroll
            for (int j = 0; j < 8; ++j) col[(k0 + j) * P + p] = e[j];
        } else {
            *reinterpret_cast<uint4*>(col + p * 9 * Cp + (int64_t)t * Cp + cc * 8) = v;
        }
    }
}

// out = relu?(y + bias) in FP32 [P][C] and BF16 [P][Cp] (zero padded)
__global__ void k_bias_act(const float* __restrict__ y, int ldy, const float* __restrict__ bias, int64_t P, int C,
                           int relu, float* __restrict__ out, bf16* __restrict__ outb, int Cp) {
    GRID_STRIDE(i, P * Cp) {
        const int64_t p = i / Cp;
        const int c = (int)(i - p * Cp);
        float v = 0.f;
        if (c < C) {
            v = y[p * ldy + c] + bias[c];
            if (relu) v = fmaxf(v, 0.f);
            out[p * C + c] = v;
        }
        if (outb) outb[i] = __float2bfloat16_rn(v);
    }
}

// 2x2 average pooling of in [B][H][W][C] -> out [B][H/2][W/2][C] (FP32 and BF16 [.][Cp])
__global__ void k_pool(const float* __restrict__ in, int B, int H, int W, int C, float* __restrict__ out,
                       bf16* __restrict__ outb, int Cp) {
    const int h = H / 2, w = W / 2;
    GRID_STRIDE(i, (int64_t)B * h * w * Cp) {
        const int64_t p = i / Cp;
        const int c = (int)(i - p * Cp);
        const int64_t b = p / ((int64_t)h * w);
        const int r = (int)(p - b * h * w), y = r / w, x = r % w;
        float v = 0.f;
        if (c < C) {
            const float* s = in + ((b * H + 2 * y) * W + 2 * x) * C + c;
            v = 0.25f * ((s[0] + s[C]) + (s[(int64_t)W * C] + s[(int64_t)W * C + C]));
            out[p * C + c] = v;
        }
        outb[i] = __float2bfloat16_rn(v);
    }
}

__global__ void k_pool_bwd(const float* __restrict__ dout, int B, int H, int W, int C, float* __restrict__ din,
                           int accumulate) {
    GRID_STRIDE(i, (int64_t)B * H * W * C) {
        const int64_t p = i / C;
        const int c = (int)(i - p * C);
        const int64_t b = p / ((int64_t)H * W);
        const int r = (int)(p - b * H * W), y = r / W, x = r % W;
        const float v = 0.25f * dout[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
        din[i] = accumulate ? din[i] + v : v;
    }
}

// out[B][H][W][Cp] BF16 = up2(a [B][H/2][W/2][Ca]) | s [B][H][W][Cs], zero padded
__global__ void k_up_cat(const float* __restrict__ a, int Ca, const float* __restrict__ s, int Cs, int B, int H, int W,
                         bf16* __restrict__ out, int Cp) {
    GRID_STRIDE(i, (int64_t)B * H * W * Cp) {
        const int64_t p = i / Cp;
        const int c = (int)(i - p * Cp);
        const int64_t b = p / ((int64_t)H * W);
        const int r = (int)(p - b * H * W), y = r / W, x = r % W;
        float v = 0.f;
        if (c < Ca)
            v = a[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * Ca + c];
        else if (c < Ca + Cs)
            v = s[p * Cs + (c - Ca)];
        out[i] = __float2bfloat16_rn(v);
    }
}

// backward of k_up_cat: da [B][H/2][W/2][Ca] = sum of the four children; ds [.][Cs] += (skip part)
__global__ void k_up_cat_bwd_a(const float* __restrict__ dcat, int Cp, int Ca, int B, int H, int W,
                               float* __restrict__ da) {
    const int h = H / 2, w = W / 2;
    GRID_STRIDE(i, (int64_t)B * h * w * Ca) {
        const int64_t p = i / Ca;
        const int c = (int)(i - p * Ca);
        const int64_t b = p / ((int64_t)h * w);
        const int r = (int)(p - b * h * w), y = r / w, x = r % w;
        const float* d = dcat + ((b * H + 2 * y) * W + 2 * x) * Cp + c;
        da[i] = (d[0] + d[Cp]) + (d[(int64_t)W * Cp] + d[(int64_t)W * Cp + Cp]);
    }
}

__global__ void k_add_channels(const float* __restrict__ src, int lds, int off, int64_t P, int C,
                               float* __restrict__ dst) {
    GRID_STRIDE(i, P * C) {
        const int64_t p = i / C;
        const int c = (int)(i - p * C);
        dst[i] += src[p * lds + off + c];
    }
}

// dY = dA * relu'(A) (A the layer's output) in FP32 [P][C] and BF16 [P][Cp] (zero padded)
__global__ void k_relu_bwd(const float* __restrict__ dA, const float* __restrict__ A, int64_t P, int C, int relu,
                           float* __restrict__ dY, bf16* __restrict__ dYb, int Cp) {
    GRID_STRIDE(i, P * Cp) {
        const int64_t p = i / Cp;
        const int c = (int)(i - p * Cp);
        float v = 0.f;
        if (c < C) {
            v = dA[p * C + c];
            if (relu && !(A[p * C + c] > 0.f)) v = 0.f;
            dY[p * C + c] = v;
        }
        dYb[i] = __float2bfloat16_rn(v);
    }
}

// out [C][R] = in [R][C] (BF16)
__global__ void k_transpose(const bf16* __restrict__ in, int64_t R, int C, bf16* __restrict__ out) {
    __shared__ bf16 tile[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int64_t r = r0 + k;
        const int c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < R && c < C) ? in[r * C + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int c = c0 + k;
        const int64_t r = r0 + threadIdx.x;
        if (c < C && r < R) out[(int64_t)c * R + r] = tile[threadIdx.x][k];
    }
}

// col2im: dX[p][c] (+)= sum_t dcol[p'][t Cp + c] over the outputs p' whose tap t read pixel p
__global__ void k_col2im(const float* __restrict__ dcol, int B, int H, int W, int Cp, int C, float* __restrict__ dX,
                         int accumulate) {
    const int64_t HW = (int64_t)H * W;
    GRID_STRIDE(i, B * HW * C) {
        const int64_t p = i / C;
        const int c = (int)(i - p * C);
        const int64_t b = p / HW, r = p - b * HW;
        const int y = (int)(r / W), x = (int)(r % W);
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int yo = y - (t / 3 - 1), xo = x - (t % 3 - 1);  // output pixel whose tap t is (y, x)
            if (yo >= 0 && yo < H && xo >= 0 && xo < W) s += dcol[((b * H + yo) * W + xo) * 9 * Cp + t * Cp + c];
        }
        dX[i] = accumulate ? dX[i] + s : s;
    }
}

// db[c] = sum_p dY[p][c] (one block per channel, fixed order)
__global__ void k_colsum(const float* __restrict__ dY, int64_t P, int C, float* __restrict__ db) {
    const int c = blockIdx.x;
    double s = 0.0;
    for (int64_t p = threadIdx.x; p < P; p += blockDim.x) s += dY[p * C + c];
    __shared__ double red[kT / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kT / 32; ++k) t += red[k];
        db[c] = (float)t;
    }
}

// weights: W32 [Cout][9][Cin] FP32 (master) -> Wb [Cout][9 Cp] BF16 and the
// transposed WtB [9 Cp][CoutP] BF16 (zero padded) of the data gradient
__global__ void k_wcast(const float* __restrict__ W32, int Cout, int Cin, int Cp, int CoutP, bf16* __restrict__ Wb,
                        bf16* __restrict__ WtB) {
    GRID_STRIDE(i, (int64_t)CoutP * 9 * Cp) {
        const int co = (int)(i / (9 * Cp));
        const int k = (int)(i - (int64_t)co * 9 * Cp);
        const int t = k / Cp, c = k - t * Cp;
        const float v = (co < Cout && c < Cin) ? W32[((int64_t)co * 9 + t) * Cin + c] : 0.f;
        const bf16 b = __float2bfloat16_rn(v);
        if (co < Cout) Wb[i] = b;
        WtB[(int64_t)k * CoutP + co] = b;
    }
}

// dW32 [Cout][9][Cin] from the GEMM result g [Cout][9 Cp]
__global__ void k_wgrad(const float* __restrict__ g, int Cout, int Cin, int Cp, float* __restrict__ dW) {
    GRID_STRIDE(i, (int64_t)Cout * 9 * Cin) {
        const int co = (int)(i / (9 * Cin));
        const int k = (int)(i - (int64_t)co * 9 * Cin);
        const int t = k / Cin, c = k - t * Cin;
        dW[i] = g[(int64_t)co * 9 * Cp + t * Cp + c];
    }
}

// head: v = m + d, y = v / |v|; per-pixel loss |y - t|^2 and dL/dd (L = mean over
// pixels of |y - t|^2; t may be null: inference)
__global__ void k_head(const float* __restrict__ m, const float* __restrict__ d, int ldd,
                       const float* __restrict__ tgt, int64_t P, float* __restrict__ y, float* __restrict__ gd,
                       float* __restrict__ cell_loss) {
    const float inv = 1.f / (float)P;
    GRID_STRIDE(p, P) {
        float v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = m[p * 3 + c] + d[p * ldd + c];
        const float n = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const float in_ = n > 0.f ? 1.f / n : 0.f;
        float yy[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            yy[c] = v[c] * in_;
            if (y) y[p * 3 + c] = yy[c];
        }
        if (!tgt) continue;
        float gy[3], l = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float e = yy[c] - tgt[p * 3 + c];
            l += e * e;
            gy[c] = 2.f * e * inv;
        }
        cell_loss[p] = l;
        const float dot = yy[0] * gy[0] + yy[1] * gy[1] + yy[2] * gy[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) gd[p * 3 + c] = (gy[c] - yy[c] * dot) * in_;
    }
}

__global__ void k_mean(const float* __restrict__ v, int64_t n, float* __restrict__ out) {
    __shared__ double red[kT / 32];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kT / 32; ++k) t += red[k];
        *out = (float)(t / (double)n);
    }
}

__global__ void k_sum_slabs(const float* __restrict__ work, int ns, int64_t n, float* __restrict__ out) {
    GRID_STRIDE(i, n) {
        float s = 0.f;
        for (int k = 0; k < ns; ++k) s += work[(int64_t)k * n + i];
        out[i] = s;
    }
}

__global__ void k_adam_nn(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                          float* __restrict__ m2, int64_t n, float lr, float c1, float c2) {
    GRID_STRIDE(i, n) {
        const float gi = g[i];
        const float a = 0.9f * m1[i] + 0.1f * gi;
        const float b = 0.999f * m2[i] + 0.001f * gi * gi;
        m1[i] = a;
        m2[i] = b;
        w[i] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
    }
}

template <typename F> int run(F&& f) { return capi_run(f); }
cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

int maf_nn_input(const float* x, int B, int C, int H, int W, int Cp, void* act_bf16, float* m, void* st) {
    return run([&] {
        if (Cp % 8 || Cp < C || C < 3) throw Error(1, "maf_nn_input: Cp must be a multiple of 8 >= C >= 3");
        const int64_t n = (int64_t)B * H * W * Cp;
        k_in<<<grid_for(n), kT, 0, S(st)>>>(x, B, C, H, W, Cp, static_cast<bf16*>(act_bf16), m);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_im2col(const void* act, int B, int H, int W, int Cp, void* col, int transposed, void* st) {
    return run([&] {
        if (Cp % 8) throw Error(1, "maf_nn_im2col: Cp must be a multiple of 8");
        const int64_t n = (int64_t)B * H * W * 9 * (Cp / 8);
        k_im2col<<<grid_for(n), kT, 0, S(st)>>>(static_cast<const bf16*>(act), B, H, W, Cp, static_cast<bf16*>(col),
                                                transposed);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_gemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K, void* st) {
    return run([&] { umma_gemm(A, lda, B, ldb, C, ldc, M, N, K, S(st), false, 1); });
}

// GEMM with the K range split over `splits` chunks (partial slabs in work
// [splits][M][N]), summed into C [M][N] in split order
int maf_nn_gemm_splitk(const void* A, int lda, const void* B, int ldb, float* C, int M, int N, int K, int splits,
                       float* work, void* st) {
    return run([&] {
        umma_gemm(A, lda, B, ldb, work, N, M, N, K, S(st), false, splits);
        const int kchunk = (int)ceil_div(ceil_div(K, splits), 64) * 64;
        const int ns = (int)ceil_div(K, kchunk);
        k_sum_slabs<<<grid_for((int64_t)M * N), kT, 0, S(st)>>>(work, ns, (int64_t)M * N, C);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_bias_act(const float* y, int ldy, const float* bias, long long P, int C, int relu, float* out,
                    void* outb, int Cp, void* st) {
    return run([&] {
        k_bias_act<<<grid_for(P * Cp), kT, 0, S(st)>>>(y, ldy, bias, P, C, relu, out, static_cast<bf16*>(outb), Cp);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_pool(const float* in, int B, int H, int W, int C, float* out, void* outb, int Cp, void* st) {
    return run([&] {
        if (H % 2 || W % 2) throw Error(1, "maf_nn_pool: even H and W expected");
        k_pool<<<grid_for((int64_t)B * (H / 2) * (W / 2) * Cp), kT, 0, S(st)>>>(in, B, H, W, C, out,
                                                                               static_cast<bf16*>(outb), Cp);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_pool_bwd(const float* dout, int B, int H, int W, int C, float* din, int accumulate, void* st) {
    return run([&] {
        k_pool_bwd<<<grid_for((int64_t)B * H * W * C), kT, 0, S(st)>>>(dout, B, H, W, C, din, accumulate);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_up_cat(const float* a, int Ca, const float* s, int Cs, int B, int H, int W, void* out, int Cp, void* st) {
    return run([&] {
        k_up_cat<<<grid_for((int64_t)B * H * W * Cp), kT, 0, S(st)>>>(a, Ca, s, Cs, B, H, W, static_cast<bf16*>(out),
                                                                      Cp);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_up_cat_bwd(const float* dcat, int Cp, int Ca, int Cs, int B, int H, int W, float* da, float* ds,
                      void* st) {
    return run([&] {
        k_up_cat_bwd_a<<<grid_for((int64_t)B * (H / 2) * (W / 2) * Ca), kT, 0, S(st)>>>(dcat, Cp, Ca, B, H, W, da);
        MAF_LAUNCH_CHECK();
        k_add_channels<<<grid_for((int64_t)B * H * W * Cs), kT, 0, S(st)>>>(dcat, Cp, Ca, (int64_t)B * H * W, Cs, ds);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_relu_bwd(const float* dA, const float* A, long long P, int C, int relu, float* dY, void* dYb, int Cp,
                    void* st) {
    return run([&] {
        k_relu_bwd<<<grid_for(P * Cp), kT, 0, S(st)>>>(dA, A, P, C, relu, dY, static_cast<bf16*>(dYb), Cp);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_transpose(const void* in, long long R, int C, void* out, void* st) {
    return run([&] {
        dim3 grid((unsigned)ceil_div(R, 32), (unsigned)ceil_div(C, 32));
        k_transpose<<<grid, dim3(32, 8), 0, S(st)>>>(static_cast<const bf16*>(in), R, C, static_cast<bf16*>(out));
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_col2im(const float* dcol, int B, int H, int W, int Cp, int C, float* dX, int accumulate, void* st) {
    return run([&] {
        k_col2im<<<grid_for((int64_t)B * H * W * C), kT, 0, S(st)>>>(dcol, B, H, W, Cp, C, dX, accumulate);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_colsum(const float* dY, long long P, int C, float* db, void* st) {
    return run([&] {
        k_colsum<<<C, kT, 0, S(st)>>>(dY, P, C, db);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_wcast(const float* W32, int Cout, int Cin, int Cp, int CoutP, void* Wb, void* WtB, void* st) {
    return run([&] {
        if (Cp % 8 || CoutP % 8 || CoutP < Cout || Cp < Cin) throw Error(1, "maf_nn_wcast: bad padding");
        k_wcast<<<grid_for((int64_t)CoutP * 9 * Cp), kT, 0, S(st)>>>(W32, Cout, Cin, Cp, CoutP, static_cast<bf16*>(Wb),
                                                                    static_cast<bf16*>(WtB));
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_wgrad(const float* g, int Cout, int Cin, int Cp, float* dW, void* st) {
    return run([&] {
        k_wgrad<<<grid_for((int64_t)Cout * 9 * Cin), kT, 0, S(st)>>>(g, Cout, Cin, Cp, dW);
        MAF_LAUNCH_CHECK();
    });
}

int maf_nn_head(const float* m, const float* d, int ldd, const float* tgt, long long P, float* y, float* gd,
                float* cell_loss, float* loss, void* st) {
    return run([&] {
        k_head<<<grid_for(P), kT, 0, S(st)>>>(m, d, ldd, tgt, P, y, gd, cell_loss);
        MAF_LAUNCH_CHECK();
        if (tgt && loss) {
            k_mean<<<1, kT, 0, S(st)>>>(cell_loss, P, loss);
            MAF_LAUNCH_CHECK();
        }
    });
}

int maf_nn_adam(float* w, const float* g, float* m1, float* m2, long long n, float lr, int step, void* st) {
    return run([&] {
        const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
        k_adam_nn<<<grid_for(n), kT, 0, S(st)>>>(w, g, m1, m2, n, lr, c1, c2);
        MAF_LAUNCH_CHECK();
    });
}

}  // extern "C"
