// Demag pass kernels specialised at compile time for power-of-two transform
// lengths 8..4096 and three times a power of two, 96..1536 (every configuration
// of the benchmarks).  Same data flow and
// arithmetic as the generic kernels in fields.cu; the transform length, radix
// sequence, tile width and CTA size are constants, each thread keeps 16
// complex values in registers per FFT stage, global loads are issued as a
// batch into registers before they are written to shared memory, and the
// z convolution handles the rows ky and Py - ky in one CTA so that the stored
// tensor quadrant is read from HBM once.
#include <algorithm>

#include "ct_dispatch.hpp"
#include "epilogue.cuh"
#include "fft_ct.cuh"

namespace mafb {

// Resident CTAs per SM that a kernel is compiled for (a register cap): at
// least T32 threads per SM in FP32, T64 in FP64.
template <typename R, int NT, int T32, int T64>
constexpr int kMinBlocks = (sizeof(R) == 4 ? T32 : T64) / NT > 1 ? (sizeof(R) == 4 ? T32 : T64) / NT : 1;

// cells per run of the x-inverse fast epilogue (2 or 4; nx % 4 == 0 either way); a build option
#ifndef MAF_RUN_CELLS
#define MAF_RUN_CELLS 2
#endif
constexpr int kRunCells = MAF_RUN_CELLS;
static_assert(kRunCells == 2 || kRunCells == 4, "run length");
// resident threads per SM the x-inverse kernels are compiled for (register caps; build options):
// FP64 two 192-thread CTAs (168 registers, no spill); FP32 four 192-thread CTAs (80 registers:
// the power-of-two lengths up to 1024) and 576 threads for the other CTA sizes
#ifndef MAF_XINV_THREADS_F64
#define MAF_XINV_THREADS_F64 384
#endif
#ifndef MAF_XINV_THREADS_192
#define MAF_XINV_THREADS_192 768
#endif
#ifndef MAF_XINV_THREADS
#define MAF_XINV_THREADS 576
#endif

// Byte offset of the staging buffer behind the transform tile of k_xfwd_pipe
// (16-byte aligned), and that kernel's shared memory.
template <typename R, int LC, int NB> constexpr size_t xfwd_stage_offset() {
    constexpr size_t SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    return (sizeof(cplx_t<R>) * NB * SB + 15) / 16 * 16;
}
template <typename R, int LC, int NB> constexpr size_t xfwd_pipe_smem() {
    return xfwd_stage_offset<R, LC, NB>() + sizeof(R) * NB * LC;
}

// ------------------------------------------------------------------ x forward
// HIN: n_in <= LC, so the packed values k >= LC/2 are the zero padding (pruned
// from the first stage)
// (tile body: rows [tile NB, tile NB + NB); k_xfwd_ct runs tile blockIdx.x, the
// batched kernel the tile of its work item)
template <typename R, int LC, int NB, int NT, bool HIN>
__device__ __forceinline__ void xfwd_ct_tile(const R* __restrict__ in, int n_in, int64_t rows, int64_t rows_pc,
                                             const R* __restrict__ msf, R ms, cplx_t<R>* __restrict__ out,
                                             int pitch, const cplx_t<R>* __restrict__ tw,
                                             const cplx_t<R>* __restrict__ twP, int64_t tile) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    constexpr int SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    static_assert(LC * NB % NT == 0, "tile");
    const int64_t r0 = tile * NB;
    const bool even = (n_in & 1) == 0;
    // packed pair (in[2k], in[2k+1]) * Ms of row b, k = j + dk, loaded straight into the first stage
    auto ld = [&](int b, int j, int dk) -> C {
        const int k = j + dk;
        const int64_t row = r0 + b;
        R a = 0, c = 0;
        if (row < rows) {
            const R* rp = in + row * n_in;
            const int x0 = 2 * k, x1 = 2 * k + 1;
            if (even) {
                if (x0 < n_in) {
                    const auto v2 = *reinterpret_cast<const cplx_t<R>*>(rp + x0);
                    a = v2.x;
                    c = v2.y;
                }
            } else {
                if (x0 < n_in) a = rp[x0];
                if (x1 < n_in) c = rp[x1];
            }
            if (msf) {
                const R* mp = msf + (row % rows_pc) * n_in;
                if (x0 < n_in) a *= mp[x0];
                if (x1 < n_in) c *= mp[x1];
            } else {
                a *= ms;
                c *= ms;
            }
        }
        return mk(a, c);
    };
    ct_fft_in<R, -1, false, LC, NB, NT, HIN>(s, SB, tw, ld, typename CtPlan<LC>::T());
    // R2C post-processing by pairs: with E = (Z_k + Z*_{L-k})/2, O = -i (Z_k - Z*_{L-k})/2
    // and t = W_{2L}^k O, X[k] = E + t and X[L-k] = (E - t)*  (W_{2L}^{L-k} = -(W_{2L}^k)*),
    // so one pair of shared-memory reads and one twiddle give two outputs.
    const R half = (R)0.5;
    constexpr int KH = LC / 2 + 1;
    for (int idx = threadIdx.x; idx < NB * KH; idx += NT) {
        const int b = idx / KH;
        const int k = idx - b * KH;
        const int64_t row = r0 + b;
        if (row >= rows) continue;
        const C Zk = s[spad(k) + b * SB];
        const C Zm = s[spad(k == 0 ? 0 : LC - k) + b * SB];
        const C E_ = cscale(cadd(Zk, cconj(Zm)), half);
        const C O = cscale(cmul_i<-1>(csub(Zk, cconj(Zm))), half);
        const C t = cmul(twP[k], O);
        C* o = out + row * pitch;
        o[k] = cadd(E_, t);
        if (k < LC / 2) o[LC - k] = cconj(csub(E_, t));
    }
}

template <typename R, int LC, int NB, int NT, bool HIN>
__global__ void __launch_bounds__(NT) k_xfwd_ct(const R* __restrict__ in, int n_in, int64_t rows, int64_t rows_pc,
                                                const R* __restrict__ msf, R ms, cplx_t<R>* __restrict__ out,
                                                int pitch, const cplx_t<R>* __restrict__ tw,
                                                const cplx_t<R>* __restrict__ twP) {
    xfwd_ct_tile<R, LC, NB, NT, HIN>(in, n_in, rows, rows_pc, msf, ms, out, pitch, tw, twP, blockIdx.x);
}

// x forward, persistent and pipelined: each CTA walks tiles of NB rows; the m rows
// of the next tile are copied into a shared-memory staging buffer with cp.async
// while the current tile's transform runs (issued right after the first stage,
// the staging buffer's only reader).  For a scalar Ms, n_in <= LC (zero-padded
// half pruned) and rows of whole 16-byte chunks; the same arithmetic as k_xfwd_ct.
// CTAs per SM the kernel is compiled for: 1024 (FP32) / 512 (FP64) resident threads for
// power-of-two lengths, 576 / 288 for three times a power of two, whose radix-3 stage
// holds more values per thread
template <typename R, int NT>
constexpr int kXfwdPipeBlocks = ((sizeof(R) == 4 ? (NT % 3 == 0 ? 576 : 1024) : (NT % 3 == 0 ? 288 : 512)) / NT > 1)
                                    ? (sizeof(R) == 4 ? (NT % 3 == 0 ? 576 : 1024) : (NT % 3 == 0 ? 288 : 512)) / NT
                                    : 1;
template <typename R, int LC, int NB, int NT>
__global__ void __launch_bounds__(NT, (kXfwdPipeBlocks<R, NT>)) k_xfwd_pipe(const R* __restrict__ in, int n_in, int64_t rows, R ms,
                                                  cplx_t<R>* __restrict__ out, int pitch,
                                                  const cplx_t<R>* __restrict__ tw,
                                                  const cplx_t<R>* __restrict__ twP) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    constexpr int SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    R* stage = reinterpret_cast<R*>(smem_raw + xfwd_stage_offset<R, LC, NB>());
    constexpr int E16 = 16 / (int)sizeof(R);
    const int64_t ntiles = (rows + NB - 1) / NB;
    auto prefetch = [&](int64_t tile) {
        const int64_t r0 = tile * NB;
        const int nrow = (int)min((int64_t)NB, rows - r0);
        const int nchunk = nrow * n_in / E16;
        const R* src = in + r0 * n_in + threadIdx.x * E16;
        unsigned dst = (unsigned)__cvta_generic_to_shared(stage + threadIdx.x * E16);
#pragma unroll 1
        for (int q = threadIdx.x; q < nchunk; q += NT, src += NT * E16, dst += NT * 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int64_t tile = blockIdx.x;
    if (tile < ntiles) prefetch(tile);
    for (; tile < ntiles; tile += gridDim.x) {
        const int64_t r0 = tile * NB;
        asm volatile("cp.async.wait_all;\n" ::);
        __syncthreads();
        // the packed values k = j + dk < LC/2 of a pruned first stage are all inside the row (n_in = LC)
        auto ld = [&](int b, int j, int dk) -> C {
            if (r0 + b >= rows) return mk((R)0, (R)0);
            const C v = reinterpret_cast<const C*>(stage + b * n_in)[j + dk];
            return mk(v.x * ms, v.y * ms);
        };
        const int64_t next = tile + gridDim.x;
        ct_fft_in_hook<R, -1, false, LC, NB, NT, true>(
            s, SB, tw, ld, [&] { if (next < ntiles) prefetch(next); }, typename CtPlan<LC>::T());
        const R half = (R)0.5;
        constexpr int KH = LC / 2 + 1;
        for (int idx = threadIdx.x; idx < NB * KH; idx += NT) {
            const int b = idx / KH;
            const int k = idx - b * KH;
            const int64_t row = r0 + b;
            if (row >= rows) continue;
            const C Zk = s[spad(k) + b * SB];
            const C Zm = s[spad(k == 0 ? 0 : LC - k) + b * SB];
            const C E_ = cscale(cadd(Zk, cconj(Zm)), half);
            const C O = cscale(cmul_i<-1>(csub(Zk, cconj(Zm))), half);
            const C t = cmul(twP[k], O);
            C* o = out + row * pitch;
            o[k] = cadd(E_, t);
            if (k < LC / 2) o[LC - k] = cconj(csub(E_, t));
        }
        __syncthreads();  // s is rewritten by the next tile's first stage
    }
}

// ------------------------------------------------------------ strided columns
// Batched column transforms (the y passes): the first radix stage loads its
// inputs straight from global memory (rows >= n_in are the zero padding and
// are not read), the last stage stores straight to global memory (rows >=
// n_out are truncated and not written).
// HIN: n_in <= L/2 (zero-padded input), HOUT: n_out <= L/2 (truncated output);
// both prune the transform at compile time
template <typename R, int DIR, int L, int NB, int NT, bool HIN, bool HOUT, int PV>
__global__ void __launch_bounds__(NT, (kMinBlocks<R, NT * (L * NB / kE > NT ? L * NB / kE / NT : 1), 1024, 512>)) k_cols_ct(const cplx_t<R>* in, cplx_t<R>* out, int n_in, int n_out, int ncols,
                                                int64_t in_si, int64_t out_si, int64_t in_sbat, int64_t out_sbat,
                                                const cplx_t<R>* __restrict__ tw) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int c0 = blockIdx.x * NB;
    const C* ib = in + (int64_t)blockIdx.y * in_sbat + c0;
    C* ob = out + (int64_t)blockIdx.y * out_sbat + c0;
    const int ncv = min(NB, ncols - c0);
    // element i = j + di of column b; the host guarantees n_in = L/2 (HIN) or L and
    // n_out = L/2 (HOUT) or L, so every element the stages touch is in range
    auto ld = [&](int b, int j, int di) -> C {
        return b < ncv ? ib[(int64_t)j * in_si + b + (int64_t)di * in_si] : mk((R)0, (R)0);
    };
    auto st = [&](int b, int j, int di, C v) {
        if (b < ncv) ob[(int64_t)j * out_si + b + (int64_t)di * out_si] = v;
    };
    ct_fft_io<R, DIR, true, L, NB, NT, HIN, HOUT>(s, 0, tw, ld, st, typename CtPlanV<L, PV>::T());
}

// Column transforms, persistent and pipelined: each CTA walks tiles of NB
// columns (tile = column block x batch); the NIN input rows of the next tile
// (L/2 with a zero-padded input, else L) are copied into a shared-memory
// staging buffer [NIN][NB] with cp.async while the current tile's later stages
// and stores run (issued right after the first stage, the buffer's only
// reader).  Needs 16-byte row segments (NB * sizeof(C) and the pitch multiples
// of 16 bytes); chunks beyond the pitch are skipped.
template <typename R, int L, int NB> constexpr size_t cols_stage_offset() {
    return (sizeof(cplx_t<R>) * NB * ((L - 1) + ((L - 1) >> 4) + 1) + 15) / 16 * 16;
}
template <typename R, int L, int NB, bool HIN> constexpr size_t cols_pipe_smem() {
    return cols_stage_offset<R, L, NB>() + sizeof(cplx_t<R>) * NB * (HIN ? L / 2 : L);
}

template <typename R, int DIR, int L, int NB, int NT, bool HIN, bool HOUT, int PV>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2) k_cols_pipe(const cplx_t<R>* in, cplx_t<R>* out, int ncols, int64_t in_si,
                                                   int64_t out_si, int64_t in_sbat, int64_t out_sbat, int nbat,
                                                   int pitch, const cplx_t<R>* __restrict__ tw) {
    using C = cplx_t<R>;
    constexpr int NIN = HIN ? L / 2 : L;
    constexpr int CPR = NB * (int)sizeof(C) / 16;  // 16-byte chunks per staged row
    static_assert(NB * sizeof(C) % 16 == 0, "16-byte row segments");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    C* stage = reinterpret_cast<C*>(smem_raw + cols_stage_offset<R, L, NB>());
    const int ntx = (ncols + NB - 1) / NB;
    const int64_t ntiles = (int64_t)ntx * nbat;
    constexpr int EPC = 16 / (int)sizeof(C);  // complex values per chunk
    auto prefetch = [&](int64_t tile) {
        const int tx = (int)(tile % ntx), bat = (int)(tile / ntx);
        const unsigned char* src0 = reinterpret_cast<const unsigned char*>(in + bat * in_sbat + tx * NB);
        const unsigned dst0 = (unsigned)__cvta_generic_to_shared(stage);
        // chunks that start beyond the row pitch are not copied (their columns are
        // beyond ncols: read from the staging buffer, never stored)
        const int cmax = min(CPR, (pitch - tx * NB) / EPC);
#pragma unroll 4
        for (int q = threadIdx.x; q < NIN * CPR; q += NT) {
            const int i = q / CPR, c = q - i * CPR;
            if (c >= cmax) continue;
            const unsigned char* src = src0 + (int64_t)i * in_si * (int64_t)sizeof(C) + c * 16;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst0 + (unsigned)q * 16u), "l"(src));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int64_t tile = blockIdx.x;
    if (tile < ntiles) prefetch(tile);
    for (; tile < ntiles; tile += gridDim.x) {
        const int tx = (int)(tile % ntx), bat = (int)(tile / ntx);
        const int c0 = tx * NB;
        const int ncv = min(NB, ncols - c0);
        C* ob = out + bat * out_sbat + c0;
        asm volatile("cp.async.wait_all;\n" ::);
        __syncthreads();
        // element i = j + di of column b, from the staging buffer
        auto ld = [&](int b, int j, int di) -> C { return stage[(j + di) * NB + b]; };
        auto st = [&](int b, int j, int di, C v) {
            if (b < ncv) ob[(int64_t)j * out_si + b + (int64_t)di * out_si] = v;
        };
        const int64_t next = tile + gridDim.x;
        ct_fft_io_hook<R, DIR, true, L, NB, NT, HIN, HOUT>(
            s, 0, tw, ld, [&] { if (next < ntiles) prefetch(next); }, st, typename CtPlanV<L, PV>::T());
        __syncthreads();  // s is rewritten by the next tile's first stage
    }
}

// -------------------------------------------------- z convolution (3-D meshes)
// CTA (kx tile, ky) with ky in [0, ny]: rows ky and Py - ky (same tensor quadrant
// row, sign of Nxy and Nyz flipped for the second); ky = 0 and ky = ny are
// their own mirrors and run alone.
template <typename R, int L, int NB, int NT>
__global__ void __launch_bounds__(NT, (kMinBlocks<R, NT, 768, 512>)) k_convz_ct(cplx_t<R>* S, const R* __restrict__ Nred, int nz, int ny, int nxh,
                                                 int pitch, const cplx_t<R>* __restrict__ tw) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    constexpr int NC = 6 * NB;  // columns: (row, comp, b)
    static_assert(L * NC % NT == 0, "tile");
    const int Py = 2 * ny;
    const int ky = blockIdx.y;
    const bool two = ky != 0 && ky != ny;
    const int ky2 = Py - ky;
    const int c0 = blockIdx.x * NB;
    const int ncv = min(NB, nxh - c0);
    const int64_t si = (int64_t)Py * pitch;        // z stride
    const int64_t cs = (int64_t)nz * Py * pitch;   // component stride
    // column col = (row, comp, b) of the tile at z = i; rows i >= nz are padding
    auto at = [&](int col, int i, bool& ok) -> int64_t {
        const int row = col / (3 * NB);
        const int comp = (col / NB) % 3;
        const int b = col % NB;
        ok = i < nz && b < ncv && (row == 0 || two);
        return comp * cs + i * si + (int64_t)(row ? ky2 : ky) * pitch + c0 + b;
    };
    auto ld = [&](int col, int j, int di) -> C {
        bool ok;
        const int64_t o = at(col, j + di, ok);
        return ok ? S[o] : mk((R)0, (R)0);
    };
    // L = 2 nz: the upper half of the input is the padding, of the output the truncation
    ct_fft_in<R, -1, true, L, NC, NT, true>(s, 0, tw, ld, typename CtPlan<L>::T());
    const int Pz = 2 * nz;
    const int64_t tcs = (int64_t)(nz + 1) * (ny + 1) * nxh;
    for (int idx = threadIdx.x; idx < L * NB; idx += NT) {
        const int kz = idx / NB;
        const int b = idx % NB;
        if (b >= ncv) continue;
        const int kzr = kz <= nz ? kz : Pz - kz;
        const R sz = kz <= nz ? (R)1 : (R)-1;
        const int64_t o = ((int64_t)kzr * (ny + 1) + ky) * nxh + c0 + b;
        const R Nxx = Nred[o], Nxy = Nred[tcs + o], Nxz = sz * Nred[2 * tcs + o];
        const R Nyy = Nred[3 * tcs + o], Nyz = sz * Nred[4 * tcs + o], Nzz = Nred[5 * tcs + o];
#pragma unroll
        for (int row = 0; row < 2; ++row) {
            if (row == 1 && !two) break;
            const R sy = row ? (R)-1 : (R)1;
            const int base = spad(kz) * NC + row * 3 * NB + b;
            const C mx = s[base], my = s[base + NB], mz = s[base + 2 * NB];
            const R xy = sy * Nxy, yz = sy * Nyz;
            s[base] = cadd(cadd(cscale(mx, Nxx), cscale(my, xy)), cscale(mz, Nxz));
            s[base + NB] = cadd(cadd(cscale(mx, xy), cscale(my, Nyy)), cscale(mz, yz));
            s[base + 2 * NB] = cadd(cadd(cscale(mx, Nxz), cscale(my, yz)), cscale(mz, Nzz));
        }
    }
    __syncthreads();
    auto st = [&](int col, int j, int di, C v) {
        bool ok;
        const int64_t o = at(col, j + di, ok);
        if (ok) S[o] = v;
    };
    ct_fft_out<R, 1, true, L, NC, NT, true>(s, 0, tw, st, typename CtPlan<L>::T());
}

// ------------------------------------------- z-transform twiddles as constants
// cos(pi k / 64) for k = 0 .. 32 (21 digits, from the Taylor series of cos
// evaluated in 50-digit decimal arithmetic).
__host__ __device__ constexpr double cos_pi64(int k) {
    constexpr double t[33] = {
        1.000000000000000000000, 0.998795456205172392715, 0.995184726672196886245, 0.989176509964780973452,
        0.980785280403230449126, 0.970031253194543992604, 0.956940335732208864936, 0.941544065183020778413,
        0.923879532511286756128, 0.903989293123443331586, 0.881921264348355029713, 0.857728610000272069902,
        0.831469612302545237079, 0.803207531480644909807, 0.773010453362736960811, 0.740951125354959091176,
        0.707106781186547524401, 0.671558954847018400625, 0.634393284163645498215, 0.595699304492433343467,
        0.555570233019602224743, 0.514102744193221726594, 0.471396736825997648556, 0.427555093430282094321,
        0.382683432365089771728, 0.336889853392220050689, 0.290284677254462367636, 0.242980179903263889948,
        0.195090322016128267848, 0.146730474455361751659, 0.098017140329560601994, 0.049067674327418014255,
        0.0,
    };
    return t[k];
}

// W_{2 NZ}^n = exp(-i pi n / NZ) (the forward sign) for n < NZ, NZ a divisor of
// 64: with n a compile-time constant (an unrolled loop) the value is an
// immediate operand, no table load.
template <typename R, int NZ> __device__ __forceinline__ cplx_t<R> wz_const(int n) {
    static_assert(64 % NZ == 0, "NZ divides 64");
    const int k = n * (64 / NZ);  // angle pi k / 64, 0 <= k < 64
    const double c = k <= 32 ? cos_pi64(k) : -cos_pi64(64 - k);
    const double s = k <= 32 ? cos_pi64(32 - k) : cos_pi64(k - 32);
    return mk((R)c, (R)-s);
}

// ------------------------------ z convolution, transforms in registers (nz <= 16)
// Same tile as k_convz_ct, one thread per column (row, comp, b).  The zero-padded
// length-L (= 2 nz) transform is two length-nz DFTs held in registers:
//   X[2k] = DFT(x)[k],  X[2k+1] = DFT(x_n W_L^n)[k]            (forward)
//   y[n]  = IDFT(Y_even)[n] + W_L^-n IDFT(Y_odd)[n],  n < nz   (inverse, truncated)
// so only the padded half's zeros are skipped for free, no shared-memory stage
// is needed inside the transforms, and shared memory carries only the spectra
// between the transforms and the 3-component tensor product.
template <typename R, int NZ, int NB>
__global__ void __launch_bounds__(6 * NB, (kMinBlocks<R, 6 * NB, 576, 288>))
    k_convz_reg(cplx_t<R>* S, const R* __restrict__ Nred, int ny, int nxh, int pitch,
                const cplx_t<R>* __restrict__ tw) {
    using C = cplx_t<R>;
    constexpr int L = 2 * NZ;
    constexpr int NC = 6 * NB;  // columns (row, comp, b) = threads
    constexpr int NT6 = 6 * (NZ + 1) * NB;  // tensor slice: [6][NZ+1][NB]
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);  // [L][NC]
    R* tsl = reinterpret_cast<R*>(s + L * NC);
    const int Py = 2 * ny;
    const int ky = blockIdx.y;
    const bool two = ky != 0 && ky != ny;
    const int c0 = blockIdx.x * NB;
    const int ncv = min(NB, nxh - c0);
    const int64_t si = (int64_t)Py * pitch;       // z stride
    const int64_t cs = (int64_t)NZ * Py * pitch;  // component stride
    const int col = threadIdx.x;
    const int64_t tcs = (int64_t)(NZ + 1) * (ny + 1) * nxh;
    // the tensor rows of this tile go to shared memory asynchronously, under the
    // spectrum loads and the forward transforms (columns b >= ncv are not read)
    // (thread col = (component c, column b): one pointer step per kz row)
    static_assert(NT6 == NC * (NZ + 1), "one slice column per thread");
    {
        const int c = col / NB, b = col % NB;
        if (b < ncv) {
            const R* src = Nred + c * tcs + (int64_t)ky * nxh + c0 + b;
            const int64_t sstep = (int64_t)(ny + 1) * nxh;
            unsigned dst = (unsigned)__cvta_generic_to_shared(tsl + c * (NZ + 1) * NB + b);
#pragma unroll 1
            for (int kz = 0; kz <= NZ; ++kz, src += sstep, dst += NB * sizeof(R)) {
                if constexpr (sizeof(R) == 4)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src));
                else
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
            }
        }
    }
    asm volatile("cp.async.commit_group;\n" ::);
    {
        const int row = col / (3 * NB);
        const int comp = (col / NB) % 3;
        const int b = col % NB;
        const bool ok = b < ncv && (row == 0 || two);
        const C* src = S + comp * cs + (int64_t)(row ? Py - ky : ky) * pitch + c0 + b;
        C e[NZ], o[NZ];
#pragma unroll
        for (int n = 0; n < NZ; ++n) e[n] = ok ? src[n * si] : mk((R)0, (R)0);
        // the twiddles W_L^n: immediates in FP32, the correctly rounded table in FP64
        auto wz = [&](int n) -> C {
            if constexpr (sizeof(R) == 4) return wz_const<R, NZ>(n);
            else return tw[n];
        };
#pragma unroll
        for (int n = 0; n < NZ; ++n) o[n] = cmul(e[n], wz(n));
        bfly_ct<NZ, -1, R>(e);
        bfly_ct<NZ, -1, R>(o);
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
            s[(2 * k) * NC + col] = e[k];
            s[(2 * k + 1) * NC + col] = o[k];
        }
    }
    asm volatile("cp.async.wait_all;\n" ::);
    __syncthreads();
    for (int idx = threadIdx.x; idx < L * NB; idx += NC) {
        const int kz = idx / NB;
        const int b = idx % NB;
        if (b >= ncv) continue;
        const int kzr = kz <= NZ ? kz : L - kz;
        const R sz = kz <= NZ ? (R)1 : (R)-1;
        const R* tp = tsl + kzr * NB + b;
        constexpr int TC = (NZ + 1) * NB;  // component stride of the slice
        const R Nxx = tp[0], Nxy = tp[TC], Nxz = sz * tp[2 * TC];
        const R Nyy = tp[3 * TC], Nyz = sz * tp[4 * TC], Nzz = tp[5 * TC];
#pragma unroll
        for (int row = 0; row < 2; ++row) {
            if (row == 1 && !two) break;
            const R sy = row ? (R)-1 : (R)1;
            const int base = kz * NC + row * 3 * NB + b;
            const C mx = s[base], my = s[base + NB], mz = s[base + 2 * NB];
            const R xy = sy * Nxy, yz = sy * Nyz;
            s[base] = cadd(cadd(cscale(mx, Nxx), cscale(my, xy)), cscale(mz, Nxz));
            s[base + NB] = cadd(cadd(cscale(mx, xy), cscale(my, Nyy)), cscale(mz, yz));
            s[base + 2 * NB] = cadd(cadd(cscale(mx, Nxz), cscale(my, yz)), cscale(mz, Nzz));
        }
    }
    __syncthreads();
    {
        const int row = col / (3 * NB);
        const int comp = (col / NB) % 3;
        const int b = col % NB;
        const bool ok = b < ncv && (row == 0 || two);
        C e[NZ], o[NZ];
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
            e[k] = s[(2 * k) * NC + col];
            o[k] = s[(2 * k + 1) * NC + col];
        }
        bfly_ct<NZ, 1, R>(e);
        bfly_ct<NZ, 1, R>(o);
        if (ok) {
            C* dst = S + comp * cs + (int64_t)(row ? Py - ky : ky) * pitch + c0 + b;
#pragma unroll
            for (int n = 0; n < NZ; ++n) {
                C w;
                if constexpr (sizeof(R) == 4) w = wz_const<R, NZ>(n);
                else w = tw[n];
                dst[n * si] = cadd(e[n], cmulc(o[n], w));
            }
        }
    }
}

// -------------------------------------------------- y convolution (nz == 1)
// (tile body: kx columns [tile NB, tile NB + NB))
template <typename R, int L, int NB, int NT>
__device__ __forceinline__ void convy_ct_tile(cplx_t<R>* S, const R* __restrict__ Nred, int ny, int nxh, int pitch,
                                              const cplx_t<R>* __restrict__ tw, int tile) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    constexpr int NC = 3 * NB;
    static_assert(L * NC % NT == 0, "tile");
    const int c0 = tile * NB;
    const int ncv = min(NB, nxh - c0);
    const int64_t cs = (int64_t)ny * pitch;
    // column col = (comp, b) at y = i; rows i >= ny are padding
    auto ld = [&](int col, int j, int di) -> C {
        const int comp = col / NB, b = col % NB;
        const int i = j + di;
        return (i < ny && b < ncv) ? S[comp * cs + (int64_t)i * pitch + c0 + b] : mk((R)0, (R)0);
    };
    // L = 2 ny: zero-padded input, truncated output
    ct_fft_in<R, -1, true, L, NC, NT, true>(s, 0, tw, ld, typename CtPlan<L>::T());
    const int64_t tcs = (int64_t)(ny + 1) * nxh;
    for (int idx = threadIdx.x; idx < L * NB; idx += NT) {
        const int ky = idx / NB;
        const int b = idx % NB;
        if (b >= ncv) continue;
        const int kyr = ky <= ny ? ky : L - ky;
        const R sy = ky <= ny ? (R)1 : (R)-1;
        const int64_t o = (int64_t)kyr * nxh + c0 + b;
        const R Nxx = Nred[o], Nxy = sy * Nred[tcs + o], Nyy = Nred[2 * tcs + o], Nzz = Nred[3 * tcs + o];
        const int base = spad(ky) * NC + b;
        const C mx = s[base], my = s[base + NB], mz = s[base + 2 * NB];
        s[base] = cadd(cscale(mx, Nxx), cscale(my, Nxy));
        s[base + NB] = cadd(cscale(mx, Nxy), cscale(my, Nyy));
        s[base + 2 * NB] = cscale(mz, Nzz);
    }
    __syncthreads();
    auto st = [&](int col, int j, int di, C v) {
        const int comp = col / NB, b = col % NB;
        const int i = j + di;
        if (i < ny && b < ncv) S[comp * cs + (int64_t)i * pitch + c0 + b] = v;
    };
    ct_fft_out<R, 1, true, L, NC, NT, true>(s, 0, tw, st, typename CtPlan<L>::T());
}

template <typename R, int L, int NB, int NT>
__global__ void __launch_bounds__(NT) k_convy_ct(cplx_t<R>* S, const R* __restrict__ Nred, int ny, int nxh, int pitch,
                                                 const cplx_t<R>* __restrict__ tw) {
    convy_ct_tile<R, L, NB, NT>(S, Nred, ny, nxh, pitch, tw, blockIdx.x);
}

// --------------------------------------------------- x inverse + epilogue
// (tile body: (y, z) rows [tile NBR, tile NBR + NBR))
template <typename R, int EPI, int LC, int NBR, int NT, int RN>
__device__ __forceinline__ void xinv_ct_tile(const cplx_t<R>* __restrict__ S1, int pitch,
                                             const cplx_t<R>* __restrict__ tw, const cplx_t<R>* __restrict__ twP,
                                             const Geom& g, R scale, const R* __restrict__ m, const MsInfo& ms,
                                             const TermList& tl, const EpilogueArgs& ep, int run4, int tile) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    constexpr int NC = 3 * NBR;
    constexpr int SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    static_assert(LC * NC % NT == 0, "tile");
    const int rows_pc = g.ny * g.nz;
    const int ry0 = tile * NBR;
    // Z[k] = (X[k] + X*[LC-k]) + i (X[k] - X*[LC-k]) W^-k of column (comp, row),
    // formed from global memory straight into the first stage
    auto ld = [&](int col, int j, int dk) -> C {
        const int comp = col / NBR;
        const int ry = ry0 + col % NBR;
        if (ry >= rows_pc) return mk((R)0, (R)0);
        const C* rp = S1 + ((int64_t)comp * rows_pc + ry) * pitch;
        const C Xk = (rp + j)[dk];
        const C Xm = (rp + (LC - j))[-dk];
        const C E_ = cadd(Xk, cconj(Xm));
        const C O = cmulc(csub(Xk, cconj(Xm)), (twP + j)[dk]);
        return cadd(E_, cmul_i<1>(O));
    };
    // only the first nx of the 2 LC real outputs (packed values k < LC/2) are kept
    if constexpr (LC >= 32)
        ct_fft_in<R, 1, false, LC, NC, NT, false, true>(s, SB, tw, ld, typename CtPlan<LC>::T());
    else
        ct_fft_in<R, 1, false, LC, NC, NT>(s, SB, tw, ld, typename CtPlan<LC>::T());
    if constexpr (EPI == EPI_H || EPI == EPI_LLG) {
        if (run4) {
            // the rows are nx = LC cells long (the x padding doubles nx), so the run
            // index arithmetic is compile-time; (y, z) of the CTA's first row once
            constexpr int runs = LC / RN;
            const int z0 = ry0 / g.ny;
            const int y0 = ry0 - z0 * g.ny;
            for (int idx = threadIdx.x; idx < NBR * runs; idx += NT) {
                const int b = idx / runs;
                const int x0 = (idx - b * runs) * RN;
                const int ry = ry0 + b;
                if (ry >= rows_pc) continue;
                int y = y0 + b, z = z0;
                while (y >= g.ny) {
                    y -= g.ny;
                    ++z;
                }
                const int64_t cell0 = (int64_t)ry * LC + x0;
                RunN<R, RN> r;
                runN_load<R, RN>(m, g, x0, y, z, cell0, r);
                R hd[RN][3];
#pragma unroll
                for (int i = 0; i < RN; i += 2) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        // cells x0 + i and x0 + i + 1 are the two halves of one packed value
                        const C val = s[spad((x0 + i) >> 1) + (c * NBR + b) * SB];
                        hd[i][c] = scale * val.x;
                        hd[i + 1][c] = scale * val.y;
                    }
                }
                runN_epilogue<R, EPI, RN>(tl, g, r, cell0, hd, ep);
            }
            return;
        }
    }
    double eacc = 0;
    for (int idx = threadIdx.x; idx < NBR * g.nx; idx += NT) {
        const int b = idx / g.nx;
        const int x = idx - b * g.nx;
        const int ry = ry0 + b;
        if (ry >= rows_pc) continue;
        const int z = ry / g.ny;
        const int y = ry - z * g.ny;
        const int64_t cell = (int64_t)ry * g.nx + x;
        R hd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const C val = s[spad(x >> 1) + (c * NBR + b) * SB];
            hd[c] = scale * ((x & 1) ? val.y : val.x);
        }
        epilogue_cell<R, EPI>(g, x, y, z, cell, m, ms, tl, ep, hd, eacc);
    }
    if constexpr (EPI == EPI_EDENS || EPI == EPI_EGRAD) block_sum_store(eacc, ep.partials);
}

template <typename R, int EPI, int LC, int NBR, int NT, int RN>
__global__ void __launch_bounds__(NT, (kMinBlocks<R, NT, (RN == 2 ? (NT == 192 ? MAF_XINV_THREADS_192 : MAF_XINV_THREADS) : 384), MAF_XINV_THREADS_F64>)) k_xinv_ct(const cplx_t<R>* __restrict__ S1, int pitch,
                                                const cplx_t<R>* __restrict__ tw, const cplx_t<R>* __restrict__ twP,
                                                Geom g, R scale, const R* __restrict__ m, MsInfo ms, TermList tl,
                                                EpilogueArgs ep, int run4) {
    xinv_ct_tile<R, EPI, LC, NBR, NT, RN>(S1, pitch, tw, twP, g, scale, m, ms, tl, ep, run4, blockIdx.x);
}

// ---------------------------------------------- batched (work-table) passes
// One CTA per work item (item, tile): the item's arguments come from a device
// array, the tile body is the per-state kernel's.
template <typename R, int LC, int NB, int NT>
__global__ void __launch_bounds__(NT) kbt_xfwd(const CtXfwdItem<R>* __restrict__ items, const int2* __restrict__ work,
                                               const cplx_t<R>* __restrict__ tw, const cplx_t<R>* __restrict__ twP) {
    const int2 w = work[blockIdx.x];
    const CtXfwdItem<R> d = items[w.x];
    xfwd_ct_tile<R, LC, NB, NT, true>(d.in, d.n_in, d.rows, d.rows, nullptr, d.ms, d.out, d.pitch, tw, twP, w.y);
}

template <typename R, int L, int NB, int NT>
__global__ void __launch_bounds__(NT) kbt_convy(const CtConvyItem<R>* __restrict__ items, const int2* __restrict__ work,
                                                const cplx_t<R>* __restrict__ tw) {
    const int2 w = work[blockIdx.x];
    const CtConvyItem<R> d = items[w.x];
    convy_ct_tile<R, L, NB, NT>(d.S, d.Nred, L / 2, d.nxh, d.pitch, tw, w.y);
}

template <typename R, int LC, int NBR, int NT, int RN>
__global__ void __launch_bounds__(NT, (kMinBlocks<R, NT, (RN == 2 ? (NT == 192 ? MAF_XINV_THREADS_192 : MAF_XINV_THREADS) : 384), MAF_XINV_THREADS_F64>))
    kbt_xinv(const CtXinvItem<R>* __restrict__ items, const int2* __restrict__ work, const cplx_t<R>* __restrict__ tw,
             const cplx_t<R>* __restrict__ twP) {
    const int2 w = work[blockIdx.x];
    const CtXinvItem<R>& d = items[w.x];
    xinv_ct_tile<R, EPI_LLG, LC, NBR, NT, RN>(d.S1, d.pitch, tw, twP, d.g, d.scale, d.m, d.ms, d.tl, d.ep, d.run4, w.y);
}

// ------------------------------------------------------------------ launches
template <typename K> static void ct_smem(K kernel, size_t bytes) {
    // opt in above 32 KB: the 48 KB default also has to hold the static shared memory
    if (bytes > 32 * 1024) MAF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// tile widths: about 4096 (FP32) / 2048 (FP64) complex values per CTA for the
// x passes, 8192 / 4096 for the column passes (a 32-byte row segment at least)
template <typename R> constexpr int kTileX = sizeof(R) == 4 ? 4096 : 2048;
// the pipelined x forward: about 1024 values per tile (one row at length 1024, so
// 64-thread CTAs, sixteen per SM in FP32): the small CTAs keep more tiles in different
// phases per SM than 4-row tiles at the same resident warps (0.172 -> 0.158 ms FP32,
// 0.348 -> 0.338 ms FP64 at 1024x1024x16)
template <typename R> constexpr int kTileXP = 1024;
template <typename R> constexpr int kTileC = sizeof(R) == 4 ? 8192 : 4096;
// complex values per CTA tile of the y passes (columns x length); a build option
#ifndef MAF_COLS_TILE_F32
#define MAF_COLS_TILE_F32 8192
#endif
template <typename R> constexpr int kTileCols = sizeof(R) == 4 ? MAF_COLS_TILE_F32 : 4096;
// radix-16 butterflies per thread and stage in the FP32 y passes (1 or 2; a build
// option): two halve the CTA to 256 threads at 128 registers, two CTAs per SM as
// with one, and each thread keeps twice the loads in flight
#ifndef MAF_COLS_BPT_F32
#define MAF_COLS_BPT_F32 2
#endif
template <typename R> constexpr int kColsBpt = sizeof(R) == 4 ? MAF_COLS_BPT_F32 : 1;
static_assert(MAF_COLS_BPT_F32 == 1 || MAF_COLS_BPT_F32 == 2, "butterflies per thread");
constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }
constexpr int pow2floor(int x) {
    int p = 1;
    while (p * 2 <= x) p *= 2;
    return p;
}

// twiddles of the compile-time transform of length L: the W_L table and the
// stage rows of its radix sequence
template <int L, int PV = 0> static const void* ct_tw(Twiddles& tw, bool f64) {
    using P = typename CtPlanV<L, PV>::T;
    int rad[8] = {};
    radix_list(P(), rad);
    return tw.get_ct(L, f64, rad, radix_count(P()));
}

template <typename R, int LC, bool HIN>
static void xfwd_L(const R* in, int n_in, int64_t rows, int64_t rows_pc, const R* msf, R ms, cplx_t<R>* out, int pitch,
                   const void* tw, const void* twP, cudaStream_t st) {
    constexpr int NB = pow2floor(cmax(1, kTileX<R> / LC));
    constexpr int NT = LC * NB / kE;
    static_assert(NT <= kMaxFftThreads, "CTA size");
    constexpr int SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    const size_t smem = sizeof(cplx_t<R>) * (size_t)NB * SB;
    if constexpr (HIN) {
        // the pipelined persistent kernel: scalar Ms, rows of whole 16-byte chunks
        constexpr int NB = pow2floor(cmax(1, kTileXP<R> / LC));
        constexpr int NT = LC * NB / kE;
        constexpr int E16 = 16 / (int)sizeof(R);
        if (!msf && n_in % E16 == 0 && (uintptr_t)in % 16 == 0) {
            auto kp = k_xfwd_pipe<R, LC, NB, NT>;
            const size_t smem_p = xfwd_pipe_smem<R, LC, NB>();
            ct_smem(kp, smem_p);
            static int per_sm[2] = {0, 0}, sms = 0;  // per precision, measured once per process
            int& ps = per_sm[sizeof(R) == 8];
            if (!ps) {
                MAF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, kp, NT, smem_p));
                int dev = 0;
                MAF_CUDA(cudaGetDevice(&dev));
                MAF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
                if (ps < 1) ps = 1;
            }
            const int64_t ntiles = ceil_div(rows, NB);
            const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)ps * sms);
            kp<<<grid, NT, smem_p, st>>>(in, n_in, rows, ms, out, pitch, static_cast<const cplx_t<R>*>(tw),
                                         static_cast<const cplx_t<R>*>(twP));
            MAF_LAUNCH_CHECK();
            return;
        }
    }
    auto k = k_xfwd_ct<R, LC, NB, NT, HIN>;
    ct_smem(k, smem);
    k<<<(unsigned)ceil_div(rows, NB), NT, smem, st>>>(in, n_in, rows, rows_pc, msf, ms, out, pitch,
                                                       static_cast<const cplx_t<R>*>(tw),
                                                       static_cast<const cplx_t<R>*>(twP));
    MAF_LAUNCH_CHECK();
}

template <typename R, int DIR, int L, int TILE, bool HIN, bool HOUT, int PV>
static void cols_L(const cplx_t<R>* in, cplx_t<R>* out, int n_in, int n_out, int ncols, int64_t in_si, int64_t out_si,
                   int64_t in_sbat, int64_t out_sbat, int nbat, const void* tw, int pipe, int pitch, cudaStream_t st) {
    constexpr int NB = pow2floor(cmin(32, cmax(1, TILE / L)));
    constexpr int NT = L * NB / (kE * kColsBpt<R>) > 0 ? L * NB / (kE * kColsBpt<R>) : 1;
    static_assert(NT <= 1024, "CTA size");
    const size_t smem = sizeof(cplx_t<R>) * (size_t)NB * ((L - 1) + ((L - 1) >> 4) + 1);
    if constexpr (HIN && !HOUT && L >= 256 && NB * sizeof(cplx_t<R>) % 16 == 0) {
        // pipelined persistent variant: the column tiles stay inside the row pitch,
        // 16-byte aligned rows and batches
        const int ntx = (int)ceil_div(ncols, NB);
        const bool ok = pipe && ncols <= pitch && (pitch * sizeof(cplx_t<R>)) % 16 == 0 && (uintptr_t)in % 16 == 0 &&
                        (in_si * (int64_t)sizeof(cplx_t<R>)) % 16 == 0 &&
                        (in_sbat * (int64_t)sizeof(cplx_t<R>)) % 16 == 0;
        if (ok) {
            auto kp = k_cols_pipe<R, DIR, L, NB, NT, HIN, HOUT, PV>;
            const size_t smem_p = cols_pipe_smem<R, L, NB, HIN>();
            ct_smem(kp, smem_p);
            int per_sm = 0;
            MAF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, NT, smem_p));
            const int64_t ntiles = (int64_t)ntx * nbat;
            const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)std::max(per_sm, 1) * sm_count());
            kp<<<grid, NT, smem_p, st>>>(in, out, ncols, in_si, out_si, in_sbat, out_sbat, nbat, pitch,
                                         static_cast<const cplx_t<R>*>(tw));
            MAF_LAUNCH_CHECK();
            return;
        }
    }
    auto k = k_cols_ct<R, DIR, L, NB, NT, HIN, HOUT, PV>;
    ct_smem(k, smem);
    dim3 grid((unsigned)ceil_div(ncols, NB), (unsigned)nbat);
    k<<<grid, NT, smem, st>>>(in, out, n_in, n_out, ncols, in_si, out_si, in_sbat, out_sbat,
                              static_cast<const cplx_t<R>*>(tw));
    MAF_LAUNCH_CHECK();
}

template <typename R, int L, bool REG>
static void convz_L(cplx_t<R>* S, const R* Nred, int nz, int ny, int nxh, int pitch, const void* tw, cudaStream_t st) {
    constexpr int NB = pow2floor(cmin(32, cmax(1, kTileC<R> / (6 * L))));
    constexpr int NT = L * 6 * NB / kE;
    static_assert(NT <= kMaxFftThreads, "CTA size");
    const size_t smem = sizeof(cplx_t<R>) * (size_t)6 * NB * ((L - 1) + ((L - 1) >> 4) + 1);
    if constexpr (L <= 32 && REG) {
        // transforms in registers: one thread per column, 16 columns of kx per CTA
        // (96 threads; at nz = 16 in FP32, 96 registers and 31 KB of shared memory:
        // seven CTAs per SM, where 32-column CTAs fit three)
        constexpr int NBR = 16;
        // spectra [L][6 NBR] plus the tensor slice [6][L/2 + 1][NBR]
        constexpr size_t smem_r = sizeof(cplx_t<R>) * (size_t)L * 6 * NBR + sizeof(R) * (size_t)6 * (L / 2 + 1) * NBR;
        auto kr = k_convz_reg<R, L / 2, NBR>;
        ct_smem(kr, smem_r);
        dim3 grid((unsigned)ceil_div(nxh, NBR), (unsigned)(ny + 1));
        kr<<<grid, 6 * NBR, smem_r, st>>>(S, Nred, ny, nxh, pitch, static_cast<const cplx_t<R>*>(tw));
    } else {
        auto k = k_convz_ct<R, L, NB, NT>;
        ct_smem(k, smem);
        dim3 grid((unsigned)ceil_div(nxh, NB), (unsigned)(ny + 1));
        k<<<grid, NT, smem, st>>>(S, Nred, nz, ny, nxh, pitch, static_cast<const cplx_t<R>*>(tw));
    }
    MAF_LAUNCH_CHECK();
}

template <typename R, int L>
static void convy_L(cplx_t<R>* S, const R* Nred, int ny, int nxh, int pitch, const void* tw, cudaStream_t st) {
    constexpr int NB = pow2floor(cmin(32, cmax(1, kTileC<R> / (3 * L))));
    constexpr int NT0 = L * 3 * NB / kE;
    static_assert(NT0 >= 1 && NT0 <= kMaxFftThreads, "CTA size");
    const size_t smem = sizeof(cplx_t<R>) * (size_t)3 * NB * ((L - 1) + ((L - 1) >> 4) + 1);
    auto k = k_convy_ct<R, L, NB, NT0>;
    ct_smem(k, smem);
    k<<<(unsigned)ceil_div(nxh, NB), NT0, smem, st>>>(S, Nred, ny, nxh, pitch, static_cast<const cplx_t<R>*>(tw));
    MAF_LAUNCH_CHECK();
}

template <typename R, int LC, int RN>
static void xinv_L(const cplx_t<R>* S1, int pitch, const void* tw, const void* twP, const Geom& g, R scale, const R* m,
                   const MsInfo& ms, const TermList& tl_in, const EpilogueArgs& ep, cudaStream_t st, int* nblocks) {
    // half the column-pass tile: the epilogue's register demand allows one
    // 384-thread CTA per SM, two CTAs of half the rows overlap their phases
    constexpr int NBR = pow2floor(cmax(1, kTileC<R> / (6 * LC)));
    constexpr int NC = 3 * NBR;
    constexpr int NT = LC * NC / kE;
    static_assert(NT <= kMaxFftThreads, "CTA size");
    constexpr int SB = (LC - 1) + ((LC - 1) >> 4) + 1;
    const size_t smem = sizeof(cplx_t<R>) * (size_t)NC * SB;
    const int64_t rows_pc = (int64_t)g.ny * g.nz;
    const unsigned blocks = (unsigned)ceil_div(rows_pc, NBR);
    const int run4 = run4_eligible(g, m, ms, tl_in, ep) ? 1 : 0;
    TermList tl = tl_in;
    if (run4) prepare_run4(tl, g, ms.Ms);
    if (nblocks) *nblocks = (int)blocks;
    const auto* t = static_cast<const cplx_t<R>*>(tw);
    const auto* tp = static_cast<const cplx_t<R>*>(twP);
    switch (ep.kind) {
        case EPI_H: {
            auto k = k_xinv_ct<R, EPI_H, LC, NBR, NT, RN>;
            ct_smem(k, smem);
            k<<<blocks, NT, smem, st>>>(S1, pitch, t, tp, g, scale, m, ms, tl, ep, run4);
            break;
        }
        case EPI_LLG: {
            auto k = k_xinv_ct<R, EPI_LLG, LC, NBR, NT, RN>;
            ct_smem(k, smem);
            k<<<blocks, NT, smem, st>>>(S1, pitch, t, tp, g, scale, m, ms, tl, ep, run4);
            break;
        }
        case EPI_EGRAD: {
            auto k = k_xinv_ct<R, EPI_EGRAD, LC, NBR, NT, RN>;
            ct_smem(k, smem);
            k<<<blocks, NT, smem, st>>>(S1, pitch, t, tp, g, scale, m, ms, tl, ep, run4);
            break;
        }
        default: {
            auto k = k_xinv_ct<R, EPI_EDENS, LC, NBR, NT, RN>;
            ct_smem(k, smem);
            k<<<blocks, NT, smem, st>>>(S1, pitch, t, tp, g, scale, m, ms, tl, ep, run4);
            break;
        }
    }
    MAF_LAUNCH_CHECK();
}

// Tile shapes of the per-state launches (xfwd_L, convy_L, xinv_L), shared by the batched ones.
template <typename R, int LC> struct XfwdShape {
    static constexpr int NB = pow2floor(cmax(1, kTileX<R> / LC));
    static constexpr int NT = LC * NB / kE;
    static constexpr size_t smem = sizeof(cplx_t<R>) * (size_t)NB * ((LC - 1) + ((LC - 1) >> 4) + 1);
};
template <typename R, int L> struct ConvyShape {
    static constexpr int NB = pow2floor(cmin(32, cmax(1, kTileC<R> / (3 * L))));
    static constexpr int NT = L * 3 * NB / kE;
    static constexpr size_t smem = sizeof(cplx_t<R>) * (size_t)3 * NB * ((L - 1) + ((L - 1) >> 4) + 1);
};
template <typename R, int LC> struct XinvShape {
    static constexpr int NBR = pow2floor(cmax(1, kTileC<R> / (6 * LC)));
    static constexpr int NT = LC * 3 * NBR / kE;
    static constexpr size_t smem = sizeof(cplx_t<R>) * (size_t)3 * NBR * ((LC - 1) + ((LC - 1) >> 4) + 1);
};

template <typename R, int LC>
static void batch_xfwd_L(const CtXfwdItem<R>* items, const int2* work, int nwork, const void* tw, const void* twP,
                         cudaStream_t st) {
    using S = XfwdShape<R, LC>;
    auto k = kbt_xfwd<R, LC, S::NB, S::NT>;
    ct_smem(k, S::smem);
    k<<<(unsigned)nwork, S::NT, S::smem, st>>>(items, work, static_cast<const cplx_t<R>*>(tw),
                                                static_cast<const cplx_t<R>*>(twP));
    MAF_LAUNCH_CHECK();
}

template <typename R, int L>
static void batch_convy_L(const CtConvyItem<R>* items, const int2* work, int nwork, const void* tw, cudaStream_t st) {
    using S = ConvyShape<R, L>;
    auto k = kbt_convy<R, L, S::NB, S::NT>;
    ct_smem(k, S::smem);
    k<<<(unsigned)nwork, S::NT, S::smem, st>>>(items, work, static_cast<const cplx_t<R>*>(tw));
    MAF_LAUNCH_CHECK();
}

template <typename R, int LC, int RN>
static void batch_xinv_L(const CtXinvItem<R>* items, const int2* work, int nwork, const void* tw, const void* twP,
                         cudaStream_t st) {
    using S = XinvShape<R, LC>;
    auto k = kbt_xinv<R, LC, S::NBR, S::NT, RN>;
    ct_smem(k, S::smem);
    k<<<(unsigned)nwork, S::NT, S::smem, st>>>(items, work, static_cast<const cplx_t<R>*>(tw),
                                                static_cast<const cplx_t<R>*>(twP));
    MAF_LAUNCH_CHECK();
}

#define MAF_CT_SWITCH(L, CALL) \
    switch (L) {               \
        case 16: CALL(16); return true;     \
        case 32: CALL(32); return true;     \
        case 64: CALL(64); return true;     \
        case 128: CALL(128); return true;   \
        case 256: CALL(256); return true;   \
        case 512: CALL(512); return true;   \
        case 1024: CALL(1024); return true; \
        case 2048: CALL(2048); return true; \
        case 4096: CALL(4096); return true; \
        case 96: CALL(96); return true;     \
        case 192: CALL(192); return true;   \
        case 384: CALL(384); return true;   \
        case 768: CALL(768); return true;   \
        case 1536: CALL(1536); return true; \
        default: return false;              \
    }

template <typename R>
bool ct_xfwd(const R* in, int n_in, int64_t rows, int64_t rows_pc, const R* msf, R ms, cplx_t<R>* out, int pitch,
             int Px, Twiddles& tw, cudaStream_t st) {
    const int LC = Px / 2;
    const bool f64 = sizeof(R) == 8;
    // a zero-padded input (n_in <= LC: the magnetisation) runs the pruned first stage;
    // a full input (the tensor, assembled in FP64) the complete one
    const bool half = n_in <= LC;
    if (!half && !f64) return false;
#define X(N)                                                                                                   \
    do {                                                                                                       \
        if (half)                                                                                              \
            xfwd_L<R, N, true>(in, n_in, rows, rows_pc, msf, ms, out, pitch, ct_tw<N>(tw, f64), tw.get(Px, f64), st); \
        else if constexpr (sizeof(R) == 8)                                                                     \
            xfwd_L<R, N, false>(in, n_in, rows, rows_pc, msf, ms, out, pitch, ct_tw<N>(tw, f64), tw.get(Px, f64), st); \
    } while (0)
    MAF_CT_SWITCH(LC, X)
#undef X
}

template <typename R, int DIR>
bool ct_cols(const cplx_t<R>* in, cplx_t<R>* out, int L, int n_in, int n_out, int ncols, int64_t in_si, int64_t out_si,
             int64_t in_sbat, int64_t out_sbat, int nbat, Twiddles& tw, const TuneChoice& tc, cudaStream_t st) {
    const bool f64 = sizeof(R) == 8;
    // pruned variants: the forward y pass (zero-padded input), the inverse y pass
    // (truncated output); the tensor's full transforms (FP64) run unpruned
    const bool hin = 2 * n_in <= L, hout = 2 * n_out <= L;
    if (hin && hout) return false;
    // the kernels read exactly L/2 (pruned) or L rows and write L/2 or L
    if ((hin ? 2 * n_in : n_in) != L || (hout ? 2 * n_out : n_out) != L) return false;
    // the row stride bounds the column tiles the pipelined kernel copies whole
    const int pitch = (int)std::min<int64_t>(in_si, 1 << 30);
    if (!hin && !hout && !f64) return false;
    // radix plan of this pass (TuneChoice::cols_plan: 0 both 16 16 R, 1 both 16 R 16,
    // 2 only the inverse pass 16 R 16, 3 only the forward pass 16 R 16)
    const bool alt = DIR < 0 ? (tc.cols_plan == 1 || tc.cols_plan == 3) : (tc.cols_plan == 1 || tc.cols_plan == 2);
#define C3(N, T, HI, HO, V)                                                                                \
    cols_L<R, DIR, N, T, HI, HO, V>(in, out, n_in, n_out, ncols, in_si, out_si, in_sbat, out_sbat, nbat,     \
                                    ct_tw<N, V>(tw, f64), tc.cols_pipe, pitch, st)
#define C2(N, T, HI, HO)               \
    do {                               \
        if constexpr (N >= 512 && (N & (N - 1)) == 0) {  \
            if (alt)                   \
                C3(N, T, HI, HO, 1);   \
            else                       \
                C3(N, T, HI, HO, 0);   \
        } else {                       \
            C3(N, T, HI, HO, 0);       \
        }                              \
    } while (0)
#define C1(N, T)                                                \
    do {                                                        \
        if (hin)                                                \
            C2(N, T, true, false);                              \
        else if (hout)                                          \
            C2(N, T, false, true);                              \
        else if constexpr (sizeof(R) == 8)                      \
            C2(N, T, false, false);                             \
    } while (0)
#define X(N)                                                    \
    do {                                                        \
        if (tc.cols_wide)                                       \
            C1(N, 2 * kTileCols<R>);                            \
        else                                                    \
            C1(N, kTileCols<R>);                                \
    } while (0)
    MAF_CT_SWITCH(L, X)
#undef X
#undef C1
#undef C2
#undef C3
}

template <typename R>
bool ct_convz(cplx_t<R>* S, const R* Nred, int nz, int ny, int nxh, int pitch, Twiddles& tw, const TuneChoice& tc,
              cudaStream_t st) {
    const bool f64 = sizeof(R) == 8;
    const int L = 2 * nz;
#define X(N)                                                                 \
    do {                                                                     \
        if (tc.convz_reg)                                                    \
            convz_L<R, N, true>(S, Nred, nz, ny, nxh, pitch, ct_tw<N>(tw, f64), st);  \
        else                                                                 \
            convz_L<R, N, false>(S, Nred, nz, ny, nxh, pitch, ct_tw<N>(tw, f64), st); \
    } while (0)
    switch (L) {
        case 8: X(8); return true;
        case 16: X(16); return true;
        case 32: X(32); return true;
        case 64: X(64); return true;
        default: return false;
    }
#undef X
}

template <typename R>
bool ct_convy(cplx_t<R>* S, const R* Nred, int ny, int nxh, int pitch, Twiddles& tw, cudaStream_t st) {
    const bool f64 = sizeof(R) == 8;
    const int L = 2 * ny;
#define X(N) convy_L<R, N>(S, Nred, ny, nxh, pitch, ct_tw<N>(tw, f64), st)
    switch (L) {
        case 16: X(16); return true;
        case 32: X(32); return true;
        case 64: X(64); return true;
        case 128: X(128); return true;
        case 256: X(256); return true;
        case 512: X(512); return true;
        case 1024: X(1024); return true;
        case 2048: X(2048); return true;
        case 96: X(96); return true;
        case 192: X(192); return true;
        case 384: X(384); return true;
        case 768: X(768); return true;
        case 1536: X(1536); return true;
        default: return false;
    }
#undef X
}

template <typename R>
bool ct_xinv(const cplx_t<R>* S1, int pitch, int Px, Twiddles& tw, const Geom& g, R scale, const R* m,
             const MsInfo& ms, const TermList& tl, const EpilogueArgs& ep, const TuneChoice& tc, cudaStream_t st,
             int* nblocks) {
    const int LC = Px / 2;
    if (g.nx != LC) return false;  // the kernels take the row length from LC
    const bool f64 = sizeof(R) == 8;
    const int run = tc.xinv_run ? tc.xinv_run : kRunCells;
#define X(N)                                                                                                    \
    do {                                                                                                        \
        if (run == 4)                                                                                           \
            xinv_L<R, N, 4>(S1, pitch, ct_tw<N>(tw, f64), tw.get(Px, f64), g, scale, m, ms, tl, ep, st, nblocks);  \
        else                                                                                                    \
            xinv_L<R, N, 2>(S1, pitch, ct_tw<N>(tw, f64), tw.get(Px, f64), g, scale, m, ms, tl, ep, st, nblocks);  \
    } while (0)
    switch (LC) {
        case 16: X(16); return true;
        case 32: X(32); return true;
        case 64: X(64); return true;
        case 128: X(128); return true;
        case 256: X(256); return true;
        case 512: X(512); return true;
        case 1024: X(1024); return true;
        case 2048: X(2048); return true;
        case 96: X(96); return true;
        case 192: X(192); return true;
        case 384: X(384); return true;
        case 768: X(768); return true;
        case 1536: X(1536); return true;
        default: return false;
    }
#undef X
}

// lengths of the batched kernels: x passes L = Px / 2 and y convolution L = Py in 16..2048 (powers of two)
// and 96..1536 (three times a power of two)
#define MAF_CT_BATCH_SWITCH(L, CALL)  \
    switch (L) {                      \
        case 16: CALL(16); break;     \
        case 32: CALL(32); break;     \
        case 64: CALL(64); break;     \
        case 128: CALL(128); break;   \
        case 256: CALL(256); break;   \
        case 512: CALL(512); break;   \
        case 1024: CALL(1024); break; \
        case 2048: CALL(2048); break; \
        case 96: CALL(96); break;     \
        case 192: CALL(192); break;   \
        case 384: CALL(384); break;   \
        case 768: CALL(768); break;   \
        case 1536: CALL(1536); break; \
        default: break;               \
    }

template <typename R> int ct_batch_tile(int pass, int L) {
    int t = 0;
#define X(N) t = pass == 0 ? XfwdShape<R, N>::NB : pass == 1 ? ConvyShape<R, N>::NB : XinvShape<R, N>::NBR
    MAF_CT_BATCH_SWITCH(L, X)
#undef X
    return t;
}

template <typename R> const void* ct_batch_twiddles(int pass, int L, Twiddles& tw) {
    (void)pass;  // every pass of these lengths runs the default radix plan
    const void* p = nullptr;
#define X(N) p = ct_tw<N>(tw, sizeof(R) == 8)
    MAF_CT_BATCH_SWITCH(L, X)
#undef X
    return p;
}

template <typename R> void ct_batch_xinv_prepare(CtXinvItem<R>& it) {
    it.run4 = run4_eligible(it.g, it.m, it.ms, it.tl, it.ep) ? 1 : 0;
    if (it.run4) prepare_run4(it.tl, it.g, it.ms.Ms);
}

template <typename R>
void ct_batch_xfwd(const CtXfwdItem<R>* items, const int2* work, int nwork, int L, const void* tw, const void* twP,
                   cudaStream_t st) {
    if (nwork <= 0) return;
#define X(N) batch_xfwd_L<R, N>(items, work, nwork, tw, twP, st)
    MAF_CT_BATCH_SWITCH(L, X)
#undef X
}

template <typename R>
void ct_batch_convy(const CtConvyItem<R>* items, const int2* work, int nwork, int L, const void* tw, cudaStream_t st) {
    if (nwork <= 0) return;
#define X(N) batch_convy_L<R, N>(items, work, nwork, tw, st)
    MAF_CT_BATCH_SWITCH(L, X)
#undef X
}

template <typename R>
void ct_batch_xinv(const CtXinvItem<R>* items, const int2* work, int nwork, int L, int run, const void* tw,
                   const void* twP, cudaStream_t st) {
    if (nwork <= 0) return;
#define X(N)                                                        \
    do {                                                            \
        if (run == 4)                                               \
            batch_xinv_L<R, N, 4>(items, work, nwork, tw, twP, st); \
        else                                                        \
            batch_xinv_L<R, N, 2>(items, work, nwork, tw, twP, st); \
    } while (0)
    MAF_CT_BATCH_SWITCH(L, X)
#undef X
}

// The instantiations are split over several compilations of this file
// (MAF_CT_PART = 1: x forward and convolutions, 2: y passes, 3: x inverse;
// MAF_CT_REAL = 4 or 8 selects FP32 or FP64), so that the build compiles them
// in parallel; without the macros every instantiation is made here.
#if !defined(MAF_CT_PART) || MAF_CT_PART == 1
#define MAF_INST1(R)                                                                                                  \
    template bool ct_xfwd<R>(const R*, int, int64_t, int64_t, const R*, R, cplx_t<R>*, int, int, Twiddles&,          \
                             cudaStream_t);                                                                          \
    template bool ct_convz<R>(cplx_t<R>*, const R*, int, int, int, int, Twiddles&, const TuneChoice&,                \
                              cudaStream_t);                                                                         \
    template bool ct_convy<R>(cplx_t<R>*, const R*, int, int, int, Twiddles&, cudaStream_t);                    \
    template int ct_batch_tile<R>(int, int);                                                                      \
    template const void* ct_batch_twiddles<R>(int, int, Twiddles&);                                               \
    template void ct_batch_xinv_prepare<R>(CtXinvItem<R>&);                                                       \
    template void ct_batch_xfwd<R>(const CtXfwdItem<R>*, const int2*, int, int, const void*, const void*,        \
                                   cudaStream_t);                                                                \
    template void ct_batch_convy<R>(const CtConvyItem<R>*, const int2*, int, int, const void*, cudaStream_t);
#else
#define MAF_INST1(R)
#endif
#if !defined(MAF_CT_PART) || MAF_CT_PART == 2
#define MAF_INST2(R)                                                                                                  \
    template bool ct_cols<R, -1>(const cplx_t<R>*, cplx_t<R>*, int, int, int, int, int64_t, int64_t, int64_t,        \
                                 int64_t, int, Twiddles&, const TuneChoice&, cudaStream_t);                          \
    template bool ct_cols<R, 1>(const cplx_t<R>*, cplx_t<R>*, int, int, int, int, int64_t, int64_t, int64_t, int64_t, \
                                int, Twiddles&, const TuneChoice&, cudaStream_t);
#else
#define MAF_INST2(R)
#endif
#if !defined(MAF_CT_PART) || MAF_CT_PART == 3
#define MAF_INST3(R)                                                                                                  \
    template bool ct_xinv<R>(const cplx_t<R>*, int, int, Twiddles&, const Geom&, R, const R*, const MsInfo&,          \
                             const TermList&, const EpilogueArgs&, const TuneChoice&, cudaStream_t, int*);        \
    template void ct_batch_xinv<R>(const CtXinvItem<R>*, const int2*, int, int, int, const void*, const void*,      \
                                   cudaStream_t);
#else
#define MAF_INST3(R)
#endif
#define MAF_INST(R) MAF_INST1(R) MAF_INST2(R) MAF_INST3(R)
#if !defined(MAF_CT_REAL) || MAF_CT_REAL == 4
MAF_INST(float)
#endif
#if !defined(MAF_CT_REAL) || MAF_CT_REAL == 8
MAF_INST(double)
#endif

}  // namespace mafb
