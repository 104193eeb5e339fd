// Learned warm start for the LBFGS minimiser: a small convolutional network
// with hand-written training and inference kernels (FP32).
//
// Network: L layers of 3x3 convolutions (zero padding; layer l samples its
// input at offsets -d_l, 0, +d_l, the dilation d_l, 1 by default), ReLU after
// every layer but the last; input x [B][cin][H][W] whose first three channels are the
// magnetisation m, the rest material/field parameter maps; output
//     y = normalize(m + conv_L(...relu(conv_1(x))...))      [B][3][H][W],
// a proposal for the relaxed magnetisation.  Loss: mean over cells of
// |y - target|^2.  Parameters are one flat buffer, per layer W[cout][cin][3][3]
// then b[cout]; Adam updates them.  Every reduction (weight gradients, loss) is
// done in a fixed order, so training is deterministic.
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "../../include/maf_b200.h"
#include "capi_internal.hpp"
#include "common.cuh"
#include "engine.hpp"

using namespace mafb;

namespace {

constexpr int kMaxC = 32;      // channels per layer
constexpr int kPixPerBlk = 256;

// out[b][co][y][x] = bias[co] + sum_ci,dy,dx W[co][ci][dy][dx] in[b][ci][y+(dy-1)d][x+(dx-1)d]
// (relu on the output when RELU).  One thread per output pixel, all cout outputs.
template <bool RELU>
__global__ void k_conv_fwd(const float* __restrict__ in, const float* __restrict__ W, const float* __restrict__ bias,
                           float* __restrict__ out, int B, int cin, int cout, int H, int Wd, int dil) {
    __shared__ float w[kMaxC * kMaxC * 9];
    for (int i = threadIdx.x; i < cout * cin * 9; i += blockDim.x) w[i] = W[i];
    __syncthreads();
    const int64_t HW = (int64_t)H * Wd;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)B * HW) return;
    const int b = (int)(p / HW);
    const int r = (int)(p - (int64_t)b * HW);
    const int y = r / Wd, x = r - (r / Wd) * Wd;
    float acc[kMaxC];
    for (int co = 0; co < cout; ++co) acc[co] = bias[co];
    for (int ci = 0; ci < cin; ++ci) {
        const float* src = in + ((int64_t)b * cin + ci) * HW;
        float v[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int yy = y + (t / 3 - 1) * dil, xx = x + (t % 3 - 1) * dil;
            v[t] = (yy >= 0 && yy < H && xx >= 0 && xx < Wd) ? src[yy * Wd + xx] : 0.f;
        }
        for (int co = 0; co < cout; ++co) {
            const float* wk = w + (co * cin + ci) * 9;
            float a = acc[co];
#pragma unroll
            for (int t = 0; t < 9; ++t) a = fmaf(wk[t], v[t], a);
            acc[co] = a;
        }
    }
    for (int co = 0; co < cout; ++co) {
        const float a = acc[co];
        out[((int64_t)b * cout + co) * HW + r] = RELU ? fmaxf(a, 0.f) : a;
    }
}

// grad_in[b][ci][y][x] = sum_co,dy,dx W[co][ci][dy][dx] g[b][co][y-(dy-1)d][x-(dx-1)d],
// masked by relu'(in) when the input came out of a ReLU (in > 0).
__global__ void k_conv_bwd_data(const float* __restrict__ g, const float* __restrict__ W,
                                const float* __restrict__ act_in, float* __restrict__ gin, int B, int cin, int cout,
                                int H, int Wd, int relu_mask, int dil) {
    __shared__ float w[kMaxC * kMaxC * 9];
    for (int i = threadIdx.x; i < cout * cin * 9; i += blockDim.x) w[i] = W[i];
    __syncthreads();
    const int64_t HW = (int64_t)H * Wd;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)B * HW) return;
    const int b = (int)(p / HW);
    const int r = (int)(p - (int64_t)b * HW);
    const int y = r / Wd, x = r - (r / Wd) * Wd;
    float acc[kMaxC];
    for (int ci = 0; ci < cin; ++ci) acc[ci] = 0.f;
    for (int co = 0; co < cout; ++co) {
        const float* src = g + ((int64_t)b * cout + co) * HW;
        float v[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int yy = y - (t / 3 - 1) * dil, xx = x - (t % 3 - 1) * dil;
            v[t] = (yy >= 0 && yy < H && xx >= 0 && xx < Wd) ? src[yy * Wd + xx] : 0.f;
        }
        for (int ci = 0; ci < cin; ++ci) {
            const float* wk = w + (co * cin + ci) * 9;
            float a = acc[ci];
#pragma unroll
            for (int t = 0; t < 9; ++t) a = fmaf(wk[t], v[t], a);
            acc[ci] = a;
        }
    }
    for (int ci = 0; ci < cin; ++ci) {
        const int64_t o = ((int64_t)b * cin + ci) * HW + r;
        float a = acc[ci];
        if (relu_mask && !(act_in[o] > 0.f)) a = 0.f;
        gin[o] = a;
    }
}

// Partial weight/bias gradients: block (k, chunk) sums over the pixels of its
// chunk for weight entry k = (co, ci, t) (or bias co when k >= cout*cin*9).
__global__ void k_conv_bwd_w_part(const float* __restrict__ g, const float* __restrict__ in, float* __restrict__ part,
                                  int B, int cin, int cout, int H, int Wd, int nchunk, int dil) {
    const int nw = cout * cin * 9;
    const int k = blockIdx.x;
    const int chunk = blockIdx.y;
    const int64_t HW = (int64_t)H * Wd, P = (int64_t)B * HW;
    const int64_t per = (P + nchunk - 1) / nchunk;
    const int64_t p0 = chunk * per, p1 = p0 + per < P ? p0 + per : P;
    float acc = 0.f;
    if (k < nw) {
        const int co = k / (cin * 9), ci = (k / 9) % cin, t = k % 9;
        const int dy = (t / 3 - 1) * dil, dx = (t % 3 - 1) * dil;
        for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const int b = (int)(p / HW);
            const int r = (int)(p - (int64_t)b * HW);
            const int y = r / Wd, x = r - (r / Wd) * Wd;
            const int yy = y + dy, xx = x + dx;
            if (yy >= 0 && yy < H && xx >= 0 && xx < Wd)
                acc = fmaf(g[((int64_t)b * cout + co) * HW + r], in[((int64_t)b * cin + ci) * HW + yy * Wd + xx], acc);
        }
    } else {
        const int co = k - nw;
        for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const int b = (int)(p / HW);
            const int r = (int)(p - (int64_t)b * HW);
            acc += g[((int64_t)b * cout + co) * HW + r];
        }
    }
    __shared__ float red[kPixPerBlk / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
        part[(int64_t)k * nchunk + chunk] = s;
    }
}

// grad[k] = sum over chunks (fixed order)
__global__ void k_sum_chunks(const float* __restrict__ part, float* __restrict__ grad, int nk, int nchunk) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    float s = 0.f;
    for (int c = 0; c < nchunk; ++c) s += part[(int64_t)k * nchunk + c];
    grad[k] = s;
}

// head: v = m + d, y = v / |v|; loss terms |y - t|^2 per cell and dL/dd
// (L = mean over B*H*W cells of |y - t|^2).
__global__ void k_head(const float* __restrict__ x, int cin, const float* __restrict__ d, const float* __restrict__ tgt,
                       float* __restrict__ y, float* __restrict__ gd, float* __restrict__ cell_loss, int B, int64_t HW,
                       float inv_cells) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)B * HW) return;
    const int b = (int)(p / HW);
    const int64_t r = p - (int64_t)b * HW;
    float v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = x[((int64_t)b * cin + c) * HW + r] + d[((int64_t)b * 3 + c) * HW + r];
    const float n = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float in_ = n > 0.f ? 1.f / n : 0.f;
    float yy[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        yy[c] = v[c] * in_;
        if (y) y[((int64_t)b * 3 + c) * HW + r] = yy[c];
    }
    if (!tgt) return;
    float gy[3], l = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float e = yy[c] - tgt[((int64_t)b * 3 + c) * HW + r];
        l += e * e;
        gy[c] = 2.f * e * inv_cells;
    }
    cell_loss[p] = l;
    const float dot = yy[0] * gy[0] + yy[1] * gy[1] + yy[2] * gy[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) gd[((int64_t)b * 3 + c) * HW + r] = (gy[c] - yy[c] * dot) * in_;
}

__global__ void k_sum_loss(const float* __restrict__ cl, int64_t n, float inv_cells, float* __restrict__ out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += cl[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
        *out = (float)(t * inv_cells);
    }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

}  // namespace

struct maf_cnn_s {
    int cin = 0, width = 0, depth = 0;
    std::vector<int> ch;        // channels: ch[0] = cin, ..., ch[depth] = 3
    std::vector<int> dil;       // dilation per layer
    std::vector<int64_t> woff;  // offset of layer l's W in the flat buffer; b follows W
    int64_t nparams = 0;
    DevBuf params, grads, m1, m2, part;
    std::vector<DevBuf> act;    // activations per layer output (post-ReLU), act[depth-1] = d
    std::vector<DevBuf> gact;   // gradients of the activations
    DevBuf cell_loss, loss;
    int64_t cap = 0;            // B*H*W the buffers hold
    unsigned long long adam_t = 0;
    cudaStream_t stream = nullptr;
};

namespace {

void cnn_ensure(maf_cnn_s* h, int64_t cells) {
    if (cells <= h->cap) return;
    h->act.resize(h->depth);
    h->gact.resize(h->depth);
    for (int l = 0; l < h->depth; ++l) {
        h->act[l].alloc(sizeof(float) * h->ch[l + 1] * cells);
        h->gact[l].alloc(sizeof(float) * h->ch[l + 1] * cells);
    }
    h->cell_loss.alloc(sizeof(float) * cells);
    h->loss.alloc(sizeof(float) * 4);
    h->cap = cells;
}

void check_dims(const maf_cnn_s* h, int B, int H, int W) {
    if (!h || B <= 0 || H <= 0 || W <= 0) throw Error(MAF_ERR_BADARG, "maf_cnn: bad batch or image size");
}

// forward through all layers; d = act[depth-1]; y (optional) = normalised output
void cnn_forward(maf_cnn_s* h, const float* x, int B, int H, int W) {
    const int64_t cells = (int64_t)B * H * W;
    cnn_ensure(h, cells);
    const float* P = h->params.as<float>();
    const unsigned blocks = (unsigned)ceil_div(cells, 256);
    const float* in = x;
    for (int l = 0; l < h->depth; ++l) {
        const float* Wl = P + h->woff[l];
        const float* bl = Wl + (int64_t)h->ch[l + 1] * h->ch[l] * 9;
        float* out = h->act[l].as<float>();
        const int d = h->dil[l];
        if (l + 1 < h->depth)
            k_conv_fwd<true><<<blocks, 256, 0, h->stream>>>(in, Wl, bl, out, B, h->ch[l], h->ch[l + 1], H, W, d);
        else
            k_conv_fwd<false><<<blocks, 256, 0, h->stream>>>(in, Wl, bl, out, B, h->ch[l], h->ch[l + 1], H, W, d);
        MAF_LAUNCH_CHECK();
        in = out;
    }
}

// loss and gradients of all parameters into h->grads (forward included)
void cnn_loss_grad(maf_cnn_s* h, const float* x, const float* tgt, int B, int H, int W) {
    cnn_forward(h, x, B, H, W);
    const int64_t HW = (int64_t)H * W, cells = (int64_t)B * HW;
    const unsigned blocks = (unsigned)ceil_div(cells, 256);
    const float inv = 1.f / (float)cells;
    const int L = h->depth;
    k_head<<<blocks, 256, 0, h->stream>>>(x, h->cin, h->act[L - 1].as<float>(), tgt, nullptr,
                                          h->gact[L - 1].as<float>(), h->cell_loss.as<float>(), B, HW, inv);
    MAF_LAUNCH_CHECK();
    k_sum_loss<<<1, 1024, 0, h->stream>>>(h->cell_loss.as<float>(), cells, 1.0 / (double)cells, h->loss.as<float>());
    MAF_LAUNCH_CHECK();
    float* G = h->grads.as<float>();
    const float* P = h->params.as<float>();
    const int nchunk = (int)std::min<int64_t>(64, ceil_div(cells, 4096));
    for (int l = L - 1; l >= 0; --l) {
        const int ci = h->ch[l], co = h->ch[l + 1];
        const float* in = l == 0 ? x : h->act[l - 1].as<float>();
        const int nk = co * ci * 9 + co;
        h->part.ensure(sizeof(float) * (size_t)nk * nchunk);
        k_conv_bwd_w_part<<<dim3(nk, nchunk), kPixPerBlk, 0, h->stream>>>(h->gact[l].as<float>(), in,
                                                                            h->part.as<float>(), B, ci, co, H, W,
                                                                            nchunk, h->dil[l]);
        MAF_LAUNCH_CHECK();
        k_sum_chunks<<<(unsigned)ceil_div(nk, 256), 256, 0, h->stream>>>(h->part.as<float>(), G + h->woff[l], nk,
                                                                         nchunk);
        MAF_LAUNCH_CHECK();
        if (l > 0) {
            k_conv_bwd_data<<<blocks, 256, 0, h->stream>>>(h->gact[l].as<float>(), P + h->woff[l],
                                                           h->act[l - 1].as<float>(), h->gact[l - 1].as<float>(), B,
                                                           ci, co, H, W, 1, h->dil[l]);
            MAF_LAUNCH_CHECK();
        }
    }
}

}  // namespace

extern "C" {

int maf_cnn_create(maf_cnn* out, int cin, int width, int depth, unsigned long long seed) {
    return capi_run([&] {
        if (!out || cin < 3 || cin > kMaxC || width < 1 || width > kMaxC || depth < 2 || depth > 16)
            throw Error(MAF_ERR_BADARG, "maf_cnn_create: need 3 <= cin <= 32, 1 <= width <= 32, 2 <= depth <= 16");
        auto h = std::make_unique<maf_cnn_s>();
        h->cin = cin;
        h->width = width;
        h->depth = depth;
        h->ch.push_back(cin);
        for (int l = 1; l < depth; ++l) h->ch.push_back(width);
        h->ch.push_back(3);
        h->dil.assign(depth, 1);
        int64_t off = 0;
        for (int l = 0; l < depth; ++l) {
            h->woff.push_back(off);
            off += (int64_t)h->ch[l + 1] * h->ch[l] * 9 + h->ch[l + 1];
        }
        h->nparams = off;
        // He-style initialisation; the last layer starts at zero so the untrained
        // network returns normalize(m), the input magnetisation
        std::vector<float> p(off, 0.f);
        std::mt19937_64 rng(seed);
        for (int l = 0; l + 1 < depth; ++l) {
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (9.f * h->ch[l])));
            const int64_t nw = (int64_t)h->ch[l + 1] * h->ch[l] * 9;
            for (int64_t i = 0; i < nw; ++i) p[h->woff[l] + i] = nd(rng);
        }
        MAF_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->params.alloc(sizeof(float) * off);
        h->grads.alloc(sizeof(float) * off);
        h->m1.alloc(sizeof(float) * off);
        h->m2.alloc(sizeof(float) * off);
        MAF_CUDA(cudaMemcpyAsync(h->params.p, p.data(), sizeof(float) * off, cudaMemcpyHostToDevice, h->stream));
        MAF_CUDA(cudaMemsetAsync(h->m1.p, 0, sizeof(float) * off, h->stream));
        MAF_CUDA(cudaMemsetAsync(h->m2.p, 0, sizeof(float) * off, h->stream));
        MAF_CUDA(cudaStreamSynchronize(h->stream));
        *out = h.release();
    });
}

int maf_cnn_destroy(maf_cnn h) {
    return capi_run([&] {
        if (h && h->stream) cudaStreamSynchronize(h->stream);
        cudaStream_t s = h ? h->stream : nullptr;
        delete h;
        if (s) cudaStreamDestroy(s);
    });
}

int maf_cnn_set_dilation(maf_cnn h, const int* dilation, int n) {
    return capi_run([&] {
        if (!h || !dilation || n != h->depth) throw Error(MAF_ERR_BADARG, "maf_cnn_set_dilation: one value per layer");
        for (int l = 0; l < n; ++l)
            if (dilation[l] < 1 || dilation[l] > 64) throw Error(MAF_ERR_BADARG, "maf_cnn_set_dilation: 1 <= d <= 64");
        h->dil.assign(dilation, dilation + n);
    });
}

int maf_cnn_n_params(maf_cnn h, long long* n) {
    return capi_run([&] {
        if (!h || !n) throw Error(MAF_ERR_BADARG, "NULL argument");
        *n = h->nparams;
    });
}

int maf_cnn_get_params(maf_cnn h, float* host) {
    return capi_run([&] {
        if (!h || !host) throw Error(MAF_ERR_BADARG, "NULL argument");
        MAF_CUDA(cudaMemcpyAsync(host, h->params.p, sizeof(float) * h->nparams, cudaMemcpyDeviceToHost, h->stream));
        MAF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int maf_cnn_set_params(maf_cnn h, const float* host) {
    return capi_run([&] {
        if (!h || !host) throw Error(MAF_ERR_BADARG, "NULL argument");
        MAF_CUDA(cudaMemcpyAsync(h->params.p, host, sizeof(float) * h->nparams, cudaMemcpyHostToDevice, h->stream));
        MAF_CUDA(cudaMemsetAsync(h->m1.p, 0, sizeof(float) * h->nparams, h->stream));
        MAF_CUDA(cudaMemsetAsync(h->m2.p, 0, sizeof(float) * h->nparams, h->stream));
        MAF_CUDA(cudaStreamSynchronize(h->stream));
        h->adam_t = 0;
    });
}

int maf_cnn_forward(maf_cnn h, const float* x_dev, int B, int H, int W, float* y_dev) {
    return capi_run([&] {
        check_dims(h, B, H, W);
        if (!x_dev || !y_dev) throw Error(MAF_ERR_BADARG, "NULL argument");
        cnn_forward(h, x_dev, B, H, W);
        const int64_t HW = (int64_t)H * W;
        k_head<<<(unsigned)ceil_div((int64_t)B * HW, 256), 256, 0, h->stream>>>(
            x_dev, h->cin, h->act[h->depth - 1].as<float>(), nullptr, y_dev, nullptr, nullptr, B, HW, 0.f);
        MAF_LAUNCH_CHECK();
        MAF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int maf_cnn_loss_grad(maf_cnn h, const float* x_dev, const float* target_dev, int B, int H, int W, float* loss,
                      float* grad_host) {
    return capi_run([&] {
        check_dims(h, B, H, W);
        if (!x_dev || !target_dev || !loss) throw Error(MAF_ERR_BADARG, "NULL argument");
        cnn_loss_grad(h, x_dev, target_dev, B, H, W);
        MAF_CUDA(cudaMemcpyAsync(loss, h->loss.p, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        if (grad_host)
            MAF_CUDA(cudaMemcpyAsync(grad_host, h->grads.p, sizeof(float) * h->nparams, cudaMemcpyDeviceToHost,
                                     h->stream));
        MAF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int maf_cnn_train_step(maf_cnn h, const float* x_dev, const float* target_dev, int B, int H, int W, float lr,
                       float* loss) {
    return capi_run([&] {
        check_dims(h, B, H, W);
        if (!x_dev || !target_dev) throw Error(MAF_ERR_BADARG, "NULL argument");
        cnn_loss_grad(h, x_dev, target_dev, B, H, W);
        ++h->adam_t;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)h->adam_t), c2 = 1.f - std::pow(b2, (float)h->adam_t);
        k_adam<<<(unsigned)ceil_div(h->nparams, 256), 256, 0, h->stream>>>(
            h->params.as<float>(), h->grads.as<float>(), h->m1.as<float>(), h->m2.as<float>(), h->nparams, lr, b1, b2,
            1e-8f, c1, c2);
        MAF_LAUNCH_CHECK();
        if (loss) MAF_CUDA(cudaMemcpyAsync(loss, h->loss.p, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        MAF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

}  // extern "C"
