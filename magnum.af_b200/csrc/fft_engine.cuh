// Batched mixed-radix FFT in shared memory (Stockham autosort, decimation in
// time), used by every demag pass.  A CTA transforms `nb` columns of length L
// that sit in shared memory; each stage reads all its butterfly inputs into
// registers, synchronises, and writes the outputs back in place, so one
// buffer of L*nb complex values suffices.  Radices 2, 4, 8 are hard-coded,
// odd primes up to 13 use a direct DFT whose roots come from the same twiddle
// table.  Twiddles W_L^k = exp(-2*pi*i*k/L) are computed once on the host in
// extended precision and rounded to the transform's precision.
#pragma once
#include "common.cuh"

namespace mafb {

constexpr int kMaxStages = 24;
constexpr int kRegElems = 16;  // complex values a thread holds per stage
constexpr int kMaxFftThreads = 512;  // CTA size cap of the FFT pass kernels (128 registers per thread)

struct FFTPlan {
    int L = 1;
    int nstages = 0;
    int radix[kMaxStages] = {};
    const void* tw = nullptr;  // cplx_t<R>[L]
};

// Threads needed so that every stage of `plan` fits the register staging
// (each thread owns kRegElems/R butterflies of radix R).
inline int fft_threads_needed(const FFTPlan& p, int ncols) {
    int need = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        const int per = (kRegElems / R);
        const int bfly = (p.L / R) * ncols;
        const int t = (int)ceil_div(bfly, per);
        need = t > need ? t : need;
    }
    return need;
}

// Padded shared-memory index: one spare slot every 16 elements breaks the
// power-of-two strides of the first stages.
__host__ __device__ __forceinline__ int spad(int i) { return i + (i >> 4); }
__host__ __device__ __forceinline__ int spad_len(int L) { return L <= 0 ? 0 : spad(L - 1) + 1; }

// Element (i, b) of the tile: BFAST -> column index fastest (i-major rows of
// nb values); otherwise each column is a contiguous padded run of length sb.
template <bool BFAST> struct SLay {
    int nb;  // number of columns
    int sb;  // column stride (only for !BFAST)
    __device__ __forceinline__ int at(int i, int b) const { return BFAST ? spad(i) * nb + b : spad(i) + b * sb; }
};

// ---------------------------------------------------------------------------
// butterflies: y[k] = sum_r v[r] W_R^{r k}, W_R = exp(DIR*2*pi*i/R)
// ---------------------------------------------------------------------------
template <int DIR, typename C> __host__ __device__ __forceinline__ void bfly2(C& a, C& b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR, typename C> __host__ __device__ __forceinline__ void bfly4(C* v) {
    C t0 = cadd(v[0], v[2]);
    C t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]);
    C t3 = cmul_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <int DIR, typename R> __host__ __device__ __forceinline__ void bfly8(cplx_t<R>* v) {
    using C = cplx_t<R>;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    bfly4<DIR>(e);
    bfly4<DIR>(o);
    const R h = (R)0.70710678118654752440;  // 1/sqrt(2)
    // W8^1, W8^2, W8^3 for the sign convention DIR
    C w1 = mk(h, (R)DIR * h);
    C w3 = mk(-h, (R)DIR * h);
    C o1 = cmul(o[1], w1);
    C o2 = cmul_i<DIR>(o[2]);
    C o3 = cmul(o[3], w3);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

// direct DFT of odd prime size with roots W_R^m = tw[m * L / R]
template <int RAD, int DIR, typename R>
__device__ __forceinline__ void bfly_dft(cplx_t<R>* v, const cplx_t<R>* __restrict__ tw, int L) {
    using C = cplx_t<R>;
    C y[RAD];
    const int st = L / RAD;
#pragma unroll
    for (int k = 0; k < RAD; ++k) {
        C acc = v[0];
#pragma unroll
        for (int r = 1; r < RAD; ++r) {
            const int m = (r * k) % RAD;
            const C w = tw[m * st];
            acc = cadd(acc, DIR < 0 ? cmul(v[r], w) : cmulc(v[r], w));
        }
        y[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < RAD; ++k) v[k] = y[k];
}

template <int RAD, int DIR, typename R>
__device__ __forceinline__ void butterfly(cplx_t<R>* v, const cplx_t<R>* __restrict__ tw, int L) {
    if constexpr (RAD == 2) {
        bfly2<DIR>(v[0], v[1]);
    } else if constexpr (RAD == 4) {
        bfly4<DIR>(v);
    } else if constexpr (RAD == 8) {
        bfly8<DIR, R>(v);
    } else {
        bfly_dft<RAD, DIR, R>(v, tw, L);
    }
}

// One Stockham stage: inputs (j + r*L/R), twiddled by W_{Ns R}^{r (j mod Ns)},
// outputs to ((j - j mod Ns) R + j mod Ns + r Ns).
template <typename R, int RAD, int DIR, bool BFAST>
__device__ __forceinline__ void fft_stage(cplx_t<R>* s, const SLay<BFAST>& lay, int L, int Ns,
                                          const cplx_t<R>* __restrict__ tw) {
    using C = cplx_t<R>;
    constexpr int BPT = kRegElems / RAD;
    const int nbf = L / RAD;
    const int total = nbf * lay.nb;
    const int twst = L / (Ns * RAD);
    C v[BPT][RAD];
    int qj[BPT], qb[BPT];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * blockDim.x;
        qj[k] = -1;
        qb[k] = 0;
        if (q < total) {
            int b, j;
            if (BFAST) {
                b = q % lay.nb;
                j = q / lay.nb;
            } else {
                j = q % nbf;
                b = q / nbf;
            }
            qj[k] = j;
            qb[k] = b;
            const int jm = j % Ns;
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                C x = s[lay.at(j + r * nbf, b)];
                if (r > 0) {
                    const C w = tw[r * jm * twst];
                    x = DIR < 0 ? cmul(x, w) : cmulc(x, w);
                }
                v[k][r] = x;
            }
            butterfly<RAD, DIR, R>(v[k], tw, L);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        if (qj[k] >= 0) {
            const int j = qj[k];
            const int jm = j % Ns;
            const int d = (j - jm) * RAD + jm;
#pragma unroll
            for (int r = 0; r < RAD; ++r) s[lay.at(d + r * Ns, qb[k])] = v[k][r];
        }
    }
    __syncthreads();
}

// Full transform of the tile; callers synchronise before (data loaded) and
// the last stage ends with a barrier.
template <typename R, int DIR, bool BFAST>
__device__ void run_fft(cplx_t<R>* s, const SLay<BFAST>& lay, const FFTPlan& p) {
    const cplx_t<R>* __restrict__ tw = static_cast<const cplx_t<R>*>(p.tw);
    int Ns = 1;
    for (int st = 0; st < p.nstages; ++st) {
        const int R_ = p.radix[st];
        switch (R_) {
            case 2: fft_stage<R, 2, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 3: fft_stage<R, 3, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 4: fft_stage<R, 4, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 5: fft_stage<R, 5, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 7: fft_stage<R, 7, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 8: fft_stage<R, 8, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 11: fft_stage<R, 11, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            case 13: fft_stage<R, 13, DIR, BFAST>(s, lay, p.L, Ns, tw); break;
            default: break;  // plans are validated on the host
        }
        Ns *= R_;
    }
}

}  // namespace mafb
