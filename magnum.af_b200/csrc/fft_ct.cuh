// Compile-time specialised FFT stages for power-of-two lengths and three times
// a power of two.
//
// The transform length, the radix sequence, the number of columns in the tile
// and the CTA size are template parameters, so every index is a constant
// expression (shifts and masks), each thread holds exactly kE = 16 complex
// values in registers per stage, and nothing spills.  Same Stockham
// formulation as fft_engine.cuh (inputs j + r L/R, twiddle W_{Ns R}^{r (j mod
// Ns)}, outputs (j - j mod Ns) R + j mod Ns + r Ns), radix 16 as 4 x 4.
#pragma once
#include "fft_engine.cuh"

namespace mafb {

constexpr int kE = 16;

template <int... Rs> struct Radices {};

// 16-point DFT as two layers of radix 4 with the W16 twiddles in between.
template <int DIR, typename R> __host__ __device__ __forceinline__ void bfly16(cplx_t<R>* v) {
    using C = cplx_t<R>;
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;  // cos, sin (pi/8)
    const R h = (R)0.70710678118654752440;
    C a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        C t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
        bfly4<DIR>(t);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    // a[n2][k1] *= W16^(n2 k1), W16 = exp(DIR 2 pi i / 16)
    const R sd = (R)DIR;
    const C w1 = mk(c1, sd * s1), w2 = mk(h, sd * h), w3 = mk(s1, sd * c1);
    a[1][1] = cmul(a[1][1], w1);
    a[1][2] = cmul(a[1][2], w2);
    a[1][3] = cmul(a[1][3], w3);
    a[2][1] = cmul(a[2][1], w2);
    a[2][2] = cmul_i<DIR>(a[2][2]);
    a[2][3] = cmul(a[2][3], mk(-h, sd * h));  // W16^6
    a[3][1] = cmul(a[3][1], w3);
    a[3][2] = cmul(a[3][2], mk(-h, sd * h));  // W16^6
    a[3][3] = cmul(a[3][3], mk(-c1, -sd * s1));  // W16^9 = -W16^1
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
        bfly4<DIR>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
}

// 16-point DFT of v[0..7] with v[8..15] = 0, the zero-padded upper half of a
// transform's input: the first radix-4 layer sees two nonzero inputs per group,
// (a, b, 0, 0) -> (a + b, a + i b, a - b, a - i b) with i = W4^1 in the sign of DIR.
template <int DIR, typename R> __host__ __device__ __forceinline__ void bfly16_half(cplx_t<R>* v) {
    using C = cplx_t<R>;
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;  // cos, sin (pi/8)
    const R h = (R)0.70710678118654752440;
    C a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        const C p = v[n2], q = v[4 + n2];
        const C iq = cmul_i<DIR>(q);
        a[n2][0] = cadd(p, q);
        a[n2][1] = cadd(p, iq);
        a[n2][2] = csub(p, q);
        a[n2][3] = csub(p, iq);
    }
    const R sd = (R)DIR;
    const C w1 = mk(c1, sd * s1), w2 = mk(h, sd * h), w3 = mk(s1, sd * c1);
    a[1][1] = cmul(a[1][1], w1);
    a[1][2] = cmul(a[1][2], w2);
    a[1][3] = cmul(a[1][3], w3);
    a[2][1] = cmul(a[2][1], w2);
    a[2][2] = cmul_i<DIR>(a[2][2]);
    a[2][3] = cmul(a[2][3], mk(-h, sd * h));  // W16^6
    a[3][1] = cmul(a[3][1], w3);
    a[3][2] = cmul(a[3][2], mk(-h, sd * h));  // W16^6
    a[3][3] = cmul(a[3][3], mk(-c1, -sd * s1));  // W16^9 = -W16^1
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
        bfly4<DIR>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
}

// 3-point DFT: with W3 = -1/2 + i DIR sqrt(3)/2, y0 = a + (b + c),
// y1,2 = a - (b + c)/2 +- i DIR (sqrt(3)/2) (b - c).
template <int DIR, typename R> __host__ __device__ __forceinline__ void bfly3(cplx_t<R>* v) {
    const R h3 = (R)0.86602540378443864676;  // sqrt(3)/2
    const cplx_t<R> t1 = cadd(v[1], v[2]);
    const cplx_t<R> t2 = csub(v[0], cscale(t1, (R)0.5));
    const cplx_t<R> d = csub(v[1], v[2]);
    const cplx_t<R> t3 = mk(-(R)DIR * h3 * d.y, (R)DIR * h3 * d.x);  // i DIR h3 (b - c)
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
}

template <int RAD, int DIR, typename R> __device__ __forceinline__ void bfly_ct(cplx_t<R>* v) {
    if constexpr (RAD == 2) {
        bfly2<DIR>(v[0], v[1]);
    } else if constexpr (RAD == 3) {
        bfly3<DIR, R>(v);
    } else if constexpr (RAD == 4) {
        bfly4<DIR>(v);
    } else if constexpr (RAD == 8) {
        bfly8<DIR, R>(v);
    } else {
        static_assert(RAD == 16, "radix 2, 3, 4, 8 or 16");
        bfly16<DIR, R>(v);
    }
}

// ----------------------------------------------------------------------------
// Index arithmetic.  Element i of column b sits at sidx(i, b) of the tile.
// Between the elements i and i + STEP of a column, spad is linear whenever
// STEP is a multiple of 16 (for any i), and so is the run i = 16q + r,
// r < 16; the stages below then address a butterfly's RAD elements as one base
// index plus compile-time offsets instead of evaluating spad per element.
// ----------------------------------------------------------------------------
template <bool BFAST, int NB> __device__ __forceinline__ int sidx(int i, int b, int sb) {
    return BFAST ? spad(i) * NB + b : spad(i) + b * sb;
}
// index distance of STEP consecutive elements of a column (STEP % 16 == 0)
template <bool BFAST, int NB, int STEP> constexpr int sdist() { return (STEP + STEP / 16) * (BFAST ? NB : 1); }

// Twiddle layout of the compile-time transforms (ct_twiddles on the host): the
// table W_L^k, k in [0, L), followed, for every stage after the first, by one
// row of its RAD - 1 twiddles per jm in [0, NS): entry (jm, r - 1) =
// W_L^(r jm L / (NS RAD)), the same values as the table's.  A butterfly reads
// its twiddles from one row at compile-time offsets.
template <int NS, int RAD> constexpr int tw_rows() { return NS > 1 ? NS * (RAD - 1) : 0; }

// How a stage after the first gets its twiddles (build options per precision):
// 0 every twiddle of a butterfly is loaded from its row when the stage starts
// (correctly rounded twiddles); 1 only W^t, W^2t, W^4t and W^8t are loaded
// (t = the butterfly's row step) and the others are formed as products of at
// most four of them (a few ulp; 8-10 % faster x and y passes in FP32, field
// error unchanged at the 6e-8 level); 2 as 1, with the loads issued by the
// previous stage right before its closing barrier.  The FP64 form, the
// accuracy reference, keeps 0.
#ifndef MAF_TW_MODE_F32
#define MAF_TW_MODE_F32 1
#endif
#ifndef MAF_TW_MODE_F64
#define MAF_TW_MODE_F64 0
#endif
static_assert(MAF_TW_MODE_F32 >= 0 && MAF_TW_MODE_F32 <= 2 && MAF_TW_MODE_F64 >= 0 && MAF_TW_MODE_F64 <= 2,
              "twiddle mode");
template <typename R> constexpr int tw_mode() { return sizeof(R) == 4 ? MAF_TW_MODE_F32 : MAF_TW_MODE_F64; }

template <int A, int... REST> struct FirstOf { static constexpr int value = A; };

// The twiddles of this thread's butterflies in one stage (nothing for NS = 1).
template <typename R, int RAD, int NS, int L, int NB, int NT, bool BFAST, int TWO> struct TwStage {
    using C = cplx_t<R>;
    static constexpr int NBF = L / RAD;
    static constexpr int TOTAL = NBF * NB;
    static constexpr int BPT = (TOTAL + NT - 1) / NT;
    // (a radix-3 stage loads both of its twiddles)
    static constexpr bool FULL = tw_mode<R>() == 0 || RAD == 3;
    static constexpr int NBASE = NS == 1 ? 0 : FULL ? RAD - 1 : (RAD == 16 ? 4 : RAD == 8 ? 3 : RAD == 4 ? 2 : 1);
    C w[BPT][NBASE > 0 ? NBASE : 1];
    __device__ __forceinline__ void load(const C* __restrict__ tw) {
        if constexpr (NBASE > 0) {
#pragma unroll
            for (int k = 0; k < BPT; ++k) {
                const int q = threadIdx.x + k * NT;
                if (TOTAL % NT == 0 || q < TOTAL) {
                    const int j = BFAST ? q / NB : q % NBF;
                    const C* __restrict__ twr = tw + TWO + (j % NS) * (RAD - 1) - 1;
                    if constexpr (FULL) {
#pragma unroll
                        for (int r = 1; r < RAD; ++r) w[k][r - 1] = twr[r];
                    } else {
#pragma unroll
                        for (int e = 0; e < NBASE; ++e) w[k][e] = twr[1 << e];
                    }
                }
            }
        }
    }
    // the RAD - 1 twiddles of butterfly k: out[r] = W^(r t), r = 1 .. RAD - 1
    __device__ __forceinline__ void expand(int k, C* out) const {
        if constexpr (FULL || RAD == 2) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) out[r] = w[k][r - 1];
        } else {
            out[1] = w[k][0];
            out[2] = w[k][1];
            out[3] = cmul(out[1], out[2]);
            if constexpr (RAD >= 8) {
                out[4] = w[k][2];
                out[5] = cmul(out[1], out[4]);
                out[6] = cmul(out[2], out[4]);
                out[7] = cmul(out[3], out[4]);
            }
            if constexpr (RAD == 16) {
                out[8] = w[k][3];
#pragma unroll
                for (int r = 9; r < 16; ++r) out[r] = cmul(out[r - 8], out[8]);
            }
        }
    }
};

// One stage over NB columns of length L with NT threads; TWO is the offset of
// the stage's twiddle rows.  HOUT (last stage only): just the outputs i < L/2
// are written, the arithmetic only the others need is dropped.
// cur: the stage's twiddles (preloaded in mode 2, else loaded here); pre() runs
// after the outputs are written, before the closing barrier (the next stage's
// twiddle prefetch).
template <typename R, int RAD, int DIR, bool BFAST, int L, int NS, int NB, int NT, int TWO, bool HOUT = false,
          typename TWC, typename PRE>
__device__ __forceinline__ void ct_stage(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, TWC& cur, PRE&& pre) {
    static_assert(!HOUT || NS * RAD == L, "output pruning is for the last stage");
    if constexpr (tw_mode<R>() != 2) cur.load(tw);
    using C = cplx_t<R>;
    constexpr int NBF = L / RAD;
    constexpr int TOTAL = NBF * NB;
    constexpr int BPT = (TOTAL + NT - 1) / NT;
    constexpr bool LIN_IN = NBF % 16 == 0;
    constexpr int DIN = LIN_IN ? sdist<BFAST, NB, NBF>() : 0;
    constexpr bool LIN_OUT = (NS % 16 == 0) || (NS == 1 && 16 % RAD == 0);
    constexpr int DOUT = NS == 1 ? (BFAST ? NB : 1) : (LIN_OUT ? sdist<BFAST, NB, NS>() : 0);
    C v[BPT][RAD];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * NT;
        if (TOTAL % NT == 0 || q < TOTAL) {
            const int b = BFAST ? q % NB : q / NBF;
            const int j = BFAST ? q / NB : q % NBF;
            const int base = LIN_IN ? sidx<BFAST, NB>(j, b, sb) : 0;
            C w[RAD];
            if constexpr (NS > 1) cur.expand(k, w);
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                C x = s[LIN_IN ? base + r * DIN : sidx<BFAST, NB>(j + r * NBF, b, sb)];
                if (NS > 1 && r > 0) x = DIR < 0 ? cmul(x, w[r]) : cmulc(x, w[r]);
                v[k][r] = x;
            }
            bfly_ct<RAD, DIR, R>(v[k]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * NT;
        if (TOTAL % NT == 0 || q < TOTAL) {
            const int b = BFAST ? q % NB : q / NBF;
            const int j = BFAST ? q / NB : q % NBF;
            const int jm = j % NS;
            const int d = (j - jm) * RAD + jm;
            const int base = LIN_OUT ? sidx<BFAST, NB>(d, b, sb) : 0;
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                if (HOUT && r >= RAD / 2) continue;
                s[LIN_OUT ? base + r * DOUT : sidx<BFAST, NB>(d + r * NS, b, sb)] = v[k][r];
            }
        }
    }
    pre();
    __syncthreads();
}

// the twiddle set of the stage with radix RAD after NS, whose rows start at TWO
template <typename R, int RAD, int NS, int L, int NB, int NT, bool BFAST, int TWO>
using TwOf = TwStage<R, RAD, NS, L, NB, NT, BFAST, TWO>;

template <typename R, int DIR, bool BFAST, int L, int NS, int NB, int NT, bool HOUT, int TWO, typename TWC, int RAD,
          int... REST>
__device__ __forceinline__ void ct_run(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, TWC& cur) {
    if constexpr (sizeof...(REST) > 0) {
        constexpr int TWN = TWO + tw_rows<NS, RAD>();
        TwOf<R, FirstOf<REST...>::value, NS * RAD, L, NB, NT, BFAST, TWN> nxt;
        ct_stage<R, RAD, DIR, BFAST, L, NS, NB, NT, TWO>(s, sb, tw, cur, [&] {
            if constexpr (tw_mode<R>() == 2) nxt.load(tw);
        });
        ct_run<R, DIR, BFAST, L, NS * RAD, NB, NT, HOUT, TWN, decltype(nxt), REST...>(s, sb, tw, nxt);
    } else {
        ct_stage<R, RAD, DIR, BFAST, L, NS, NB, NT, TWO, HOUT>(s, sb, tw, cur, [] {});
    }
}

template <typename R, int DIR, bool BFAST, int L, int NB, int NT, int... RS>
__device__ __forceinline__ void ct_fft(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, Radices<RS...>) {
    TwOf<R, FirstOf<RS...>::value, 1, L, NB, NT, BFAST, L> none;
    ct_run<R, DIR, BFAST, L, 1, NB, NT, false, L, decltype(none), RS...>(s, sb, tw, none);
}

// ----------------------------------------------------------------------------
// Stages with global I/O fused in.  The first stage (Ns = 1, no twiddles) takes
// its RAD inputs j + r L/RAD of column b from ld(b, j, r L/RAD) -- straight from
// global memory into registers, so the zero-padded half of a transform costs no
// shared-memory traffic -- and writes its outputs j RAD + r to shared memory.
// The last stage (Ns = L/RAD) reads shared memory and hands its outputs
// j + r Ns to st(b, j, r Ns, value), so rows that are truncated are never
// stored.  The loader and the storer get the element as a per-butterfly part
// (b, j) and a compile-time offset, so that they can form one address per
// butterfly and add constant offsets to it.
// ----------------------------------------------------------------------------
template <bool BFAST, int NB, int NBF> __device__ __forceinline__ void ct_bj(int q, int& b, int& j) {
    b = BFAST ? q % NB : q / NBF;
    j = BFAST ? q / NB : q % NBF;
}

// The caller synchronises before s is overwritten; ends with a barrier.
// HIN: the inputs i >= L/2 are zero (a zero-padded transform) -- with a radix-16
// first stage they are neither loaded nor fed through the butterfly.
template <typename R, int RAD, int DIR, bool BFAST, int L, int NB, int NT, bool HIN, typename LD, typename PRE>
__device__ __forceinline__ void ct_stage_in(cplx_t<R>* s, int sb, LD&& ld, PRE&& pre) {
    using C = cplx_t<R>;
    constexpr int NBF = L / RAD;
    constexpr int TOTAL = NBF * NB;
    constexpr int BPT = (TOTAL + NT - 1) / NT;
    constexpr bool HALF = HIN && RAD == 16;
    constexpr bool LIN_OUT = 16 % RAD == 0;
    C v[BPT][RAD];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * NT;
        if (TOTAL % NT == 0 || q < TOTAL) {
            int b, j;
            ct_bj<BFAST, NB, NBF>(q, b, j);
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[k][r] = (HALF && r >= RAD / 2) ? mk((R)0, (R)0) : ld(b, j, r * NBF);
        }
    }
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * NT;
        if (TOTAL % NT == 0 || q < TOTAL) {
            int b, j;
            ct_bj<BFAST, NB, NBF>(q, b, j);
            if constexpr (HALF)
                bfly16_half<DIR, R>(v[k]);
            else
                bfly_ct<RAD, DIR, R>(v[k]);
            const int base = sidx<BFAST, NB>(j * RAD, b, sb);
#pragma unroll
            for (int r = 0; r < RAD; ++r)
                s[LIN_OUT ? base + r * (BFAST ? NB : 1) : sidx<BFAST, NB>(j * RAD + r, b, sb)] = v[k][r];
        }
    }
    pre();
    __syncthreads();
}

// Reads s written by the previous stage (which ended with a barrier); no
// barrier at the end: the caller synchronises before s is reused.
// HOUT: only the outputs i < L/2 are wanted (a truncated transform): the others
// are not stored, and the arithmetic that only they need is dropped.
template <typename R, int RAD, int DIR, bool BFAST, int L, int NB, int NT, bool HOUT, int TWO, typename TWC, typename ST>
__device__ __forceinline__ void ct_stage_out(const cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, TWC& cur,
                                             ST&& st) {
    using C = cplx_t<R>;
    if constexpr (tw_mode<R>() != 2) cur.load(tw);
    constexpr int NBF = L / RAD;
    constexpr int NS = NBF;
    constexpr int TOTAL = NBF * NB;
    constexpr int BPT = (TOTAL + NT - 1) / NT;
    constexpr bool LIN_IN = NBF % 16 == 0;
    constexpr int DIN = LIN_IN ? sdist<BFAST, NB, NBF>() : 0;
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int q = threadIdx.x + k * NT;
        if (TOTAL % NT == 0 || q < TOTAL) {
            int b, j;
            ct_bj<BFAST, NB, NBF>(q, b, j);
            const int base = LIN_IN ? sidx<BFAST, NB>(j, b, sb) : 0;
            C v[RAD], w[RAD];
            if constexpr (NS > 1) cur.expand(k, w);
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                C x = s[LIN_IN ? base + r * DIN : sidx<BFAST, NB>(j + r * NBF, b, sb)];
                if (NS > 1 && r > 0) x = DIR < 0 ? cmul(x, w[r]) : cmulc(x, w[r]);
                v[r] = x;
            }
            bfly_ct<RAD, DIR, R>(v);
#pragma unroll
            for (int r = 0; r < RAD; ++r)
                if (!HOUT || r < RAD / 2) st(b, j, r * NS, v[r]);
        }
    }
}

template <typename R, int DIR, bool BFAST, int L, int NS, int NB, int NT, bool HOUT, int TWO, typename ST,
          typename TWC, int RAD, int... REST>
__device__ __forceinline__ void ct_run_out(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, TWC& cur, ST&& st) {
    if constexpr (sizeof...(REST) == 0) {
        static_assert(NS * RAD == L, "radix sequence");
        ct_stage_out<R, RAD, DIR, BFAST, L, NB, NT, HOUT, TWO>(s, sb, tw, cur, st);
    } else {
        constexpr int TWN = TWO + tw_rows<NS, RAD>();
        TwOf<R, FirstOf<REST...>::value, NS * RAD, L, NB, NT, BFAST, TWN> nxt;
        ct_stage<R, RAD, DIR, BFAST, L, NS, NB, NT, TWO>(s, sb, tw, cur, [&] {
            if constexpr (tw_mode<R>() == 2) nxt.load(tw);
        });
        ct_run_out<R, DIR, BFAST, L, NS * RAD, NB, NT, HOUT, TWN, ST, decltype(nxt), REST...>(s, sb, tw, nxt, st);
    }
}

// global -> first stage -> ... -> last stage, result in shared memory
// (HIN: the inputs i >= L/2 are zero; HOUT: only the outputs i < L/2 are written)
template <typename R, int DIR, bool BFAST, int L, int NB, int NT, bool HIN = false, bool HOUT = false, typename LD,
          int R0, int... RS>
__device__ __forceinline__ void ct_fft_in(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, LD&& ld,
                                          Radices<R0, RS...>) {
    static_assert(!HOUT || sizeof...(RS) > 0, "output pruning needs a separate last stage");
    if constexpr (sizeof...(RS) > 0) {
        TwOf<R, FirstOf<RS...>::value, R0, L, NB, NT, BFAST, L> nxt;
        ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [&] {
            if constexpr (tw_mode<R>() == 2) nxt.load(tw);
        });
        ct_run<R, DIR, BFAST, L, R0, NB, NT, HOUT, L, decltype(nxt), RS...>(s, sb, tw, nxt);
    } else {
        ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [] {});
    }
}

// ct_fft_in with a hook between the first stage and the others: the first stage
// ends with a barrier, so when mid() runs no thread reads the load source any more
// (a pipelined kernel refills it there).
template <typename R, int DIR, bool BFAST, int L, int NB, int NT, bool HIN, typename LD, typename MID, int R0,
          int... RS>
__device__ __forceinline__ void ct_fft_in_hook(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, LD&& ld,
                                               MID&& mid, Radices<R0, RS...>) {
    if constexpr (sizeof...(RS) > 0) {
        TwOf<R, FirstOf<RS...>::value, R0, L, NB, NT, BFAST, L> nxt;
        ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [&] {
            if constexpr (tw_mode<R>() == 2) nxt.load(tw);
        });
        mid();
        ct_run<R, DIR, BFAST, L, R0, NB, NT, false, L, decltype(nxt), RS...>(s, sb, tw, nxt);
    } else {
        ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [] {});
        mid();
    }
}

// shared memory -> ... -> last stage -> global (HOUT: only outputs i < L/2 are stored)
template <typename R, int DIR, bool BFAST, int L, int NB, int NT, bool HOUT = false, typename ST, int... RS>
__device__ __forceinline__ void ct_fft_out(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, ST&& st,
                                           Radices<RS...>) {
    TwOf<R, FirstOf<RS...>::value, 1, L, NB, NT, BFAST, L> none;
    ct_run_out<R, DIR, BFAST, L, 1, NB, NT, HOUT, L, ST, decltype(none), RS...>(s, sb, tw, none, st);
}

// global -> ... -> global; the caller synchronises before s is reused
template <typename R, int DIR, bool BFAST, int L, int NB, int NT, bool HIN = false, bool HOUT = false, typename LD,
          typename ST, int R0, int... RS>
__device__ __forceinline__ void ct_fft_io(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, LD&& ld, ST&& st,
                                          Radices<R0, RS...>) {
    if constexpr (sizeof...(RS) == 0) {
        // one stage: load, butterfly, store; shared memory is not used
        static_assert(R0 == L, "radix sequence");
        using C = cplx_t<R>;
        constexpr int BPT = (NB + NT - 1) / NT;
        constexpr bool HALF = HIN && R0 == 16;
#pragma unroll
        for (int k = 0; k < BPT; ++k) {
            const int q = threadIdx.x + k * NT;
            if (NB % NT == 0 || q < NB) {
                C v[R0];
#pragma unroll
                for (int r = 0; r < R0; ++r) v[r] = (HALF && r >= R0 / 2) ? mk((R)0, (R)0) : ld(q, 0, r);
                if constexpr (HALF)
                    bfly16_half<DIR, R>(v);
                else
                    bfly_ct<R0, DIR, R>(v);
#pragma unroll
                for (int r = 0; r < R0; ++r)
                    if (!HOUT || r < R0 / 2) st(q, 0, r, v[r]);
            }
        }
    } else {
        TwOf<R, FirstOf<RS...>::value, R0, L, NB, NT, BFAST, L> nxt;
        ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [&] {
            if constexpr (tw_mode<R>() == 2) nxt.load(tw);
        });
        ct_run_out<R, DIR, BFAST, L, R0, NB, NT, HOUT, L, ST, decltype(nxt), RS...>(s, sb, tw, nxt, st);
    }
}

// ct_fft_io with a hook between the first stage and the others (the first stage
// ends with a barrier: its load source is free when mid() runs); more than one stage.
template <typename R, int DIR, bool BFAST, int L, int NB, int NT, bool HIN, bool HOUT, typename LD, typename MID,
          typename ST, int R0, int... RS>
__device__ __forceinline__ void ct_fft_io_hook(cplx_t<R>* s, int sb, const cplx_t<R>* __restrict__ tw, LD&& ld,
                                               MID&& mid, ST&& st, Radices<R0, RS...>) {
    static_assert(sizeof...(RS) > 0, "a hook needs more than one stage");
    TwOf<R, FirstOf<RS...>::value, R0, L, NB, NT, BFAST, L> nxt;
    ct_stage_in<R, R0, DIR, BFAST, L, NB, NT, HIN>(s, sb, ld, [&] {
        if constexpr (tw_mode<R>() == 2) nxt.load(tw);
    });
    mid();
    ct_run_out<R, DIR, BFAST, L, R0, NB, NT, HOUT, L, ST, decltype(nxt), RS...>(s, sb, tw, nxt, st);
}

// radix sequence of a compile-time plan as a host array (for the twiddle rows)
template <int... RS> constexpr int radix_count(Radices<RS...>) { return (int)sizeof...(RS); }
template <int... RS> inline void radix_list(Radices<RS...>, int* out) {
    const int v[] = {RS...};
    for (int i = 0; i < (int)sizeof...(RS); ++i) out[i] = v[i];
}

// radix sequence per power-of-two length (16 first, smaller radices last)
template <int L> struct CtPlan;
template <> struct CtPlan<2> { using T = Radices<2>; };
template <> struct CtPlan<4> { using T = Radices<4>; };
template <> struct CtPlan<8> { using T = Radices<8>; };
template <> struct CtPlan<16> { using T = Radices<16>; };
template <> struct CtPlan<32> { using T = Radices<16, 2>; };
template <> struct CtPlan<64> { using T = Radices<16, 4>; };
template <> struct CtPlan<128> { using T = Radices<16, 8>; };
template <> struct CtPlan<256> { using T = Radices<16, 16>; };
template <> struct CtPlan<512> { using T = Radices<16, 16, 2>; };
template <> struct CtPlan<1024> { using T = Radices<16, 16, 4>; };
template <> struct CtPlan<2048> { using T = Radices<16, 16, 8>; };
template <> struct CtPlan<4096> { using T = Radices<16, 16, 16>; };
// three times a power of two: the radix-3 stage second (after the pruned radix-16
// first stage, before an even last stage that output pruning can halve)
template <> struct CtPlan<96> { using T = Radices<16, 3, 2>; };
template <> struct CtPlan<192> { using T = Radices<16, 3, 4>; };
template <> struct CtPlan<384> { using T = Radices<16, 3, 8>; };
template <> struct CtPlan<768> { using T = Radices<16, 3, 16>; };
template <> struct CtPlan<1536> { using T = Radices<16, 3, 16, 2>; };

// Radix sequences the autotuner can choose for the column passes: V = 0 the
// plan above, V = 1 the small radix in the middle (16 R 16) for lengths whose
// plan ends in one (the pruned first stage keeps its radix 16 either way).
template <int L, int V> struct CtPlanV { using T = typename CtPlan<L>::T; };
template <> struct CtPlanV<512, 1> { using T = Radices<16, 2, 16>; };
template <> struct CtPlanV<1024, 1> { using T = Radices<16, 4, 16>; };
template <> struct CtPlanV<2048, 1> { using T = Radices<16, 8, 16>; };

}  // namespace mafb
