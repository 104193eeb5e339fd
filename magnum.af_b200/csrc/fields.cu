// Effective-field kernels: the zero-padded demag FFT convolution in five (3-D)
// or three (nz == 1) passes, with the local terms and the chosen epilogue
// fused into the last pass.
//
// Reference: magnumaf/src/field_terms/micro/demag_field.cpp:215-264
//   H = IFFT( N^ . FFT(pad(Ms m)) ) / (Px Py Pz), truncated to the mesh,
// with P = (2nx, 2ny, nz == 1 ? 1 : 2nz) and the tensor of demag_field.cpp:104-147.
//
// HBM layout (x fastest everywhere):
//   m, H            [3][nz][ny][nx]            real (FP32 or FP64)
//   S1 half spectrum [3][nz][ny][pitch]         complex, kx in [0, nx]
//   S2               [3][nz][Py][pitch]         complex (3-D meshes only)
//   tensor (reduced) [ncomp][nz+1 or 1][ny+1][nx+1] real: the spectral Newell
//                    tensor is real and even/odd in ky and kz, so only the
//                    quadrant ky <= ny, kz <= nz is stored (6 components; 4
//                    when nz == 1 because Nxz = Nyz = 0 in a single layer).
//
// Passes (3-D): x-fwd R2C (zero pad fused into the load) -> y-fwd (pad fused)
//   -> z-fwd . tensor . z-inv (in place, truncation fused) -> y-inv (truncation
//   fused into the store) -> x-inv C2R + local terms + epilogue.
// Passes (nz == 1): x-fwd -> y-fwd . tensor . y-inv (in place) -> x-inv + epilogue.
#include <algorithm>
#include <cmath>

#include "engine.hpp"
#include "epilogue.cuh"
#include "ct_dispatch.hpp"
#include "passes_generic.cuh"

namespace mafb {

// ---------------------------------------------------------------------------
// twiddles and plans
// ---------------------------------------------------------------------------
const void* Twiddles::get(int L, bool fp64) {
    auto key = std::make_pair(L, fp64 ? 1 : 0);
    auto it = tables_.find(key);
    if (it != tables_.end()) return it->second.p;
    // W_L^k = exp(-2 pi i k / L) in long double, reduced to the first octant
    // so that the table is symmetric to the last bit.
    std::vector<long double> c(L), s(L);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < L; ++k) {
        // angle = 2 pi k / L; use k/L in [0,1)
        long double a = 2.0L * pi * (long double)k / (long double)L;
        // symmetric evaluation about the quarter points
        int64_t k4 = 4 * (int64_t)k;
        long double cv, sv;
        if (k4 == 0) { cv = 1; sv = 0; }
        else if (k4 == L) { cv = 0; sv = 1; }
        else if (k4 == 2 * (int64_t)L) { cv = -1; sv = 0; }
        else if (k4 == 3 * (int64_t)L) { cv = 0; sv = -1; }
        else { cv = cosl(a); sv = sinl(a); }
        c[k] = cv;
        s[k] = -sv;  // exp(-i a)
    }
    DevBuf buf;
    if (fp64) {
        std::vector<double2> h(L);
        for (int k = 0; k < L; ++k) h[k] = make_double2((double)c[k], (double)s[k]);
        buf.alloc(sizeof(double2) * L);
        MAF_CUDA(cudaMemcpy(buf.p, h.data(), sizeof(double2) * L, cudaMemcpyHostToDevice));
    } else {
        std::vector<float2> h(L);
        for (int k = 0; k < L; ++k) h[k] = make_float2((float)c[k], (float)s[k]);
        buf.alloc(sizeof(float2) * L);
        MAF_CUDA(cudaMemcpy(buf.p, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
    }
    const void* p = buf.p;
    tables_.emplace(key, std::move(buf));
    return p;
}

const void* Twiddles::get_ct(int L, bool fp64, const int* radix, int nstages) {
    // (L, precision, radix sequence) identifies the layout
    int code = 0;
    for (int i = 0; i < nstages; ++i) code = code * 17 + radix[i];
    auto key = std::make_pair(L, 2 + (fp64 ? 1 : 0) + 2 * code);
    auto it = tables_.find(key);
    if (it != tables_.end()) return it->second.p;
    const void* base = get(L, fp64);
    const size_t esz = fp64 ? sizeof(double2) : sizeof(float2);
    std::vector<unsigned char> tab((size_t)L * esz);
    MAF_CUDA(cudaMemcpy(tab.data(), base, (size_t)L * esz, cudaMemcpyDeviceToHost));
    std::vector<unsigned char> out(tab);
    int NS = 1;
    for (int st = 0; st < nstages; ++st) {
        const int RAD = radix[st];
        if (NS > 1) {
            const int twst = L / (NS * RAD);
            for (int jm = 0; jm < NS; ++jm)
                for (int r = 1; r < RAD; ++r) {
                    const size_t k = (size_t)r * jm * twst;  // < L
                    out.insert(out.end(), tab.begin() + k * esz, tab.begin() + (k + 1) * esz);
                }
        }
        NS *= RAD;
    }
    DevBuf buf(out.size());
    MAF_CUDA(cudaMemcpy(buf.p, out.data(), out.size(), cudaMemcpyHostToDevice));
    const void* p = buf.p;
    tables_.emplace(key, std::move(buf));
    return p;
}

FFTPlan make_fft_plan(int L, const void* tw) {
    FFTPlan p;
    p.L = L;
    p.tw = tw;
    int n = L;
    auto push = [&](int r) {
        if (p.nstages >= kMaxStages) throw Error(6, "FFT plan: too many stages");
        p.radix[p.nstages++] = r;
    };
    while (n % 8 == 0) { push(8); n /= 8; }
    if (n % 4 == 0) { push(4); n /= 4; }
    if (n % 2 == 0) { push(2); n /= 2; }
    for (int r : {3, 5, 7, 11, 13}) {
        while (n % r == 0) { push(r); n /= r; }
    }
    if (n != 1)
        throw Error(6, "FFT length " + std::to_string(L) +
                           " has a prime factor > 13; choose mesh sizes whose doubled sizes factor into 2,3,5,7,11,13");
    return p;
}

// ---------------------------------------------------------------------------
// pass kernels
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kMaxFftThreads) k_xfwd(const R* __restrict__ in, int n_in, int64_t rows, int64_t rows_pc,
                                               const R* __restrict__ msf, R ms, cplx_t<R>* __restrict__ out, int pitch,
                                               FFTPlan plan, const cplx_t<R>* __restrict__ twP, int nb) {
    xfwd_tile<R>(in, n_in, rows, rows_pc, msf, ms, out, pitch, plan, twP, nb, blockIdx.x);
}

// Strided batched column FFT: element i of column c of batch b at
// base + b*sbat + i*si + c.  Loads n_in values (zero pad to L), stores n_out.
template <typename R, int DIR>
__global__ void __launch_bounds__(kMaxFftThreads) k_fft_cols(const cplx_t<R>* in, cplx_t<R>* out, FFTPlan plan, int n_in,
                                                   int n_out, int ncols, int64_t in_si, int64_t out_si, int64_t in_sbat,
                                                   int64_t out_sbat, int nb) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int L = plan.L;
    const SLay<true> lay{nb, 0};
    const int c0 = blockIdx.x * nb;
    const C* ib = in + (int64_t)blockIdx.y * in_sbat + c0;
    C* ob = out + (int64_t)blockIdx.y * out_sbat + c0;
    const int ncv = min(nb, ncols - c0);
    for (int idx = threadIdx.x; idx < L * nb; idx += blockDim.x) {
        const int i = idx / nb;
        const int b = idx - i * nb;
        C v = mk((R)0, (R)0);
        if (i < n_in && b < ncv) v = ib[i * in_si + b];
        s[lay.at(i, b)] = v;
    }
    __syncthreads();
    run_fft<R, DIR, true>(s, lay, plan);
    for (int idx = threadIdx.x; idx < n_out * nb; idx += blockDim.x) {
        const int i = idx / nb;
        const int b = idx - i * nb;
        if (b < ncv) ob[i * out_si + b] = s[lay.at(i, b)];
    }
}

template <typename R, bool PBC>
__global__ void __launch_bounds__(kMaxFftThreads) k_conv(cplx_t<R>* S, const R* __restrict__ Nred, FFTPlan fplan, FFTPlan iplan,
                                               int n_in, int64_t si, int64_t comp_stride, int64_t other_stride,
                                               int ncols, int nb, int axis_is_z, int ny, int nz, int nxh, PbcOp pop) {
    conv_tile<R, PBC>(S, Nred, fplan, iplan, n_in, si, comp_stride, other_stride, ncols, nb, axis_is_z, ny, nz, nxh,
                      pop, blockIdx.x, blockIdx.y);
}

template <typename R, int EPI>
__global__ void __launch_bounds__(kMaxFftThreads) k_xinv_epi(const cplx_t<R>* __restrict__ S1, int pitch, FFTPlan plan,
                                                   const cplx_t<R>* __restrict__ twP, Geom g, R scale,
                                                   const R* __restrict__ m, MsInfo ms, TermList tl, EpilogueArgs ep,
                                                   int nbr) {
    xinv_tile<R, EPI>(S1, pitch, plan, twP, g, scale, m, ms, tl, ep, nbr, blockIdx.x, 0);
}

// Local terms only (no demag in the term list).
template <typename R, int EPI>
__global__ void __launch_bounds__(256) k_local_epi(Geom g, const R* __restrict__ m, MsInfo ms, TermList tl,
                                                   EpilogueArgs ep) {
    double eacc = 0;
    const R hd[3] = {0, 0, 0};
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < g.N;
         cell += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(cell % g.nx);
        const int64_t r = cell / g.nx;
        const int y = (int)(r % g.ny);
        const int z = (int)(r / g.ny);
        epilogue_cell<R, EPI>(g, x, y, z, cell, m, ms, tl, ep, hd, eacc);
    }
    if constexpr (EPI == EPI_EDENS || EPI == EPI_EGRAD) block_sum_store(eacc, ep.partials);
}

// Local terms only, in runs of RN consecutive cells along x: the x-inverse's
// run epilogue with a zero demag contribution (eligibility: run4_eligible).
// Thread q takes run q of the flattened (row, run) index (fewer than 2^31 runs).
// FP32: capped for two CTAs per SM (128 registers); FP64 uncapped (it would spill).
template <typename R, int EPI, int RN>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 2 : 1) k_local_run(Geom g, const R* __restrict__ m, TermList tl, EpilogueArgs ep,
                                                   int nruns) {
    const int runs_row = g.nx / RN;
    R hd[RN][3];
#pragma unroll
    for (int i = 0; i < RN; ++i) hd[i][0] = hd[i][1] = hd[i][2] = (R)0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nruns; q += gridDim.x * blockDim.x) {
        const int row = q / runs_row;
        const int x0 = (q - row * runs_row) * RN;
        const int z = row / g.ny;
        const int y = row - z * g.ny;
        const int64_t cell0 = (int64_t)row * g.nx + x0;
        RunN<R, RN> r;
        runN_load<R, RN>(m, g, x0, y, z, cell0, r);
        runN_epilogue<R, EPI, RN>(tl, g, r, cell0, hd, ep);
    }
}

__global__ void k_sum_partials(const double* __restrict__ p, int n, double* out) {
    double v = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

__global__ void k_stage32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

__global__ void k_widen(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

void widen_m(const float* m32, double* m64, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_widen<<<(unsigned)blocks, 256, 0, st>>>(m32, m64, n);
    MAF_LAUNCH_CHECK();
}

void stage_m32(const double* m64, float* m32, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16);
    k_stage32<<<(unsigned)blocks, 256, 0, st>>>(m64, m32, n);
    MAF_LAUNCH_CHECK();
}

// Extract the real part of the spectral tensor on the stored quadrant.
__global__ void k_reduce_tensor(const double2* __restrict__ spec, double* __restrict__ dst, int nxh, int pitch, int Py,
                                int Kz, int Ky) {
    const int64_t total = (int64_t)Kz * Ky * nxh;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i % nxh);
        const int ky = (int)((i / nxh) % Ky);
        const int kz = (int)(i / ((int64_t)nxh * Ky));
        dst[i] = spec[((int64_t)kz * Py + ky) * pitch + kx].x;
    }
}

__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <typename K> static void set_smem(K kernel, size_t bytes) {
    // opt in above 32 KB: the 48 KB default also has to hold the static shared memory
    if (bytes > 32 * 1024) MAF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}


template <typename R>
static void launch_xfwd(const R* in, int n_in, int64_t rows, int64_t rows_pc, const R* msf, R ms, cplx_t<R>* out,
                        int pitch, int Px, Twiddles& tw, cudaStream_t st, bool try_ct = true) {
    if (try_ct && ct_xfwd<R>(in, n_in, rows, rows_pc, msf, ms, out, pitch, Px, tw, st)) return;
    const bool f64 = sizeof(R) == 8;
    const int Lc = Px / 2;
    FFTPlan plan = make_fft_plan(Lc, tw.get(Lc, f64));
    int nb = pick_nb(Lc, tile_target<R>(), (int)std::min<int64_t>(rows, 1 << 20), 64);
    int threads;
    while (true) {
        threads = fft_threads_needed(plan, nb);
        threads = std::max(threads, std::min(256, nb * Lc));
        if (threads <= kMaxFftThreads || nb == 1) break;
        nb = std::max(1, nb / 2);
    }
    threads = round_threads(threads);
    const size_t smem = sizeof(cplx_t<R>) * (size_t)nb * spad_len(Lc);
    set_smem(k_xfwd<R>, smem);
    const int64_t blocks = ceil_div(rows, nb);
    k_xfwd<R><<<(unsigned)blocks, threads, smem, st>>>(in, n_in, rows, rows_pc, msf, ms, out, pitch, plan,
                                                       static_cast<const cplx_t<R>*>(tw.get(Px, f64)), nb);
    MAF_LAUNCH_CHECK();
}

template <typename R, int DIR>
static void launch_cols(const cplx_t<R>* in, cplx_t<R>* out, int L, int n_in, int n_out, int ncols, int64_t in_si,
                        int64_t out_si, int64_t in_sbat, int64_t out_sbat, int nbat, Twiddles& tw,
                        const TuneChoice& tc, cudaStream_t st, bool try_ct = true) {
    if (try_ct && ct_cols<R, DIR>(in, out, L, n_in, n_out, ncols, in_si, out_si, in_sbat, out_sbat, nbat, tw, tc, st))
        return;
    const bool f64 = sizeof(R) == 8;
    FFTPlan plan = make_fft_plan(L, tw.get(L, f64));
    int nb = pick_nb(L, tile_target<R>(), ncols, 32);
    int threads;
    while (true) {
        threads = fft_threads_needed(plan, nb);
        threads = std::max(threads, std::min(256, nb * L));
        if (threads <= kMaxFftThreads || nb == 1) break;
        nb = std::max(1, nb / 2);
    }
    threads = round_threads(threads);
    const size_t smem = sizeof(cplx_t<R>) * (size_t)nb * spad_len(L);
    set_smem(k_fft_cols<R, DIR>, smem);
    dim3 grid((unsigned)ceil_div(ncols, nb), (unsigned)nbat);
    k_fft_cols<R, DIR><<<grid, threads, smem, st>>>(in, out, plan, n_in, n_out, ncols, in_si, out_si, in_sbat,
                                                    out_sbat, nb);
    MAF_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Demag
// ---------------------------------------------------------------------------
Demag::Demag(const MeshDims& md, cudaStream_t st, const double* tensor_host, bool pbc) : md_(md), pbc_(pbc) {
    if (md.nx < 1 || md.ny < 1 || md.nz < 1) throw Error(1, "DemagField: empty mesh");
    if (pbc) {
        // the reference's inverse fftC2R(h, is_odd = false) returns 2*(nx/2) columns,
        // i.e. the field only has the mesh's shape for even nx (demag_field_pbc.cpp:70)
        if (md.nx % 2 != 0) throw Error(6, "DemagFieldPBC: nx must be even");
        pitch_ = (nxh() + 3) / 4 * 4;
        make_fft_plan(Px() / 2, nullptr);
        make_fft_plan(Py(), nullptr);
        make_fft_plan(Pz(), nullptr);
        return;
    }
    // complex pitch: multiple of 4 so that tiles of 4 complex values start on 32 B
    pitch_ = (nxh() + 3) / 4 * 4;
    // validate all FFT lengths early
    make_fft_plan(Px() / 2, nullptr);
    make_fft_plan(Py(), nullptr);
    make_fft_plan(Pz(), nullptr);
    if (tensor_host) {
        Nred64_.alloc(sizeof(double) * tensor_elems());
        MAF_CUDA(cudaMemcpyAsync(Nred64_.p, tensor_host, sizeof(double) * tensor_elems(), cudaMemcpyHostToDevice, st));
        MAF_CUDA(cudaStreamSynchronize(st));
    } else {
        build_tensor(st);
    }
}

void Demag::build_tensor(cudaStream_t st) {
    const int Px_ = Px(), Py_ = Py(), Pz_ = Pz();
    const int64_t nreal = (int64_t)Px_ * Py_ * Pz_;
    const int Ky = md_.ny + 1;
    const int Kz = md_.nz == 1 ? 1 : md_.nz + 1;
    const int64_t cstride = (int64_t)Kz * Ky * nxh();
    Nred64_.alloc(sizeof(double) * cstride * ncomp());
    DevBuf real(sizeof(double) * nreal);
    DevBuf spec(sizeof(double2) * (int64_t)Pz_ * Py_ * pitch_);
    const int comps6[6] = {0, 1, 2, 3, 4, 5};
    const int comps4[4] = {0, 1, 3, 5};
    const int* comps = md_.nz == 1 ? comps4 : comps6;
    for (int ci = 0; ci < ncomp(); ++ci) {
        newell_component(real.as<double>(), comps[ci], md_, Px_, Py_, Pz_, true, st);
        // 3-D R2C of the real tensor component
        launch_xfwd<double>(real.as<double>(), Px_, (int64_t)Py_ * Pz_, (int64_t)Py_ * Pz_, nullptr, 1.0,
                            spec.as<double2>(), pitch_, Px_, tw_, st);
        launch_cols<double, -1>(spec.as<double2>(), spec.as<double2>(), Py_, Py_, Py_, nxh(), pitch_, pitch_,
                                (int64_t)Py_ * pitch_, (int64_t)Py_ * pitch_, Pz_, tw_, tune, st);
        if (Pz_ > 1)
            launch_cols<double, -1>(spec.as<double2>(), spec.as<double2>(), Pz_, Pz_, Pz_, nxh(),
                                    (int64_t)Py_ * pitch_, (int64_t)Py_ * pitch_, pitch_, pitch_, Py_, tw_, tune,
                                    st);
        const int64_t total = cstride;
        const int64_t blocks = std::min<int64_t>(ceil_div(total, 256), (int64_t)sm_count() * 16);
        k_reduce_tensor<<<(unsigned)blocks, 256, 0, st>>>(spec.as<double2>(), Nred64_.as<double>() + ci * cstride,
                                                           nxh(), pitch_, Py_, Kz, Ky);
        MAF_LAUNCH_CHECK();
    }
    MAF_CUDA(cudaStreamSynchronize(st));
}

void Demag::download_tensor(double* host, cudaStream_t st) const {
    MAF_CUDA(cudaMemcpyAsync(host, Nred64_.p, sizeof(double) * tensor_elems(), cudaMemcpyDeviceToHost, st));
    MAF_CUDA(cudaStreamSynchronize(st));
}

void Demag::download_real_tensor(double* host, bool symmetric, cudaStream_t st) {
    const int64_t nreal = (int64_t)Px() * Py() * Pz();
    DevBuf real(sizeof(double) * nreal);
    for (int c = 0; c < 6; ++c) {
        newell_component(real.as<double>(), c, md_, Px(), Py(), Pz(), symmetric, st);
        MAF_CUDA(cudaMemcpyAsync(host + c * nreal, real.p, sizeof(double) * nreal, cudaMemcpyDeviceToHost, st));
    }
    MAF_CUDA(cudaStreamSynchronize(st));
}

template <> const double* Demag::tensor<double>() { return Nred64_.as<double>(); }
template <> const float* Demag::tensor<float>() {
    if (!Nred32_.p) {
        const int64_t n = (int64_t)tensor_elems();
        Nred32_.alloc(sizeof(float) * n);
        k_d2f<<<(unsigned)std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16), 256>>>(Nred64_.as<double>(),
                                                                                   Nred32_.as<float>(), n);
        MAF_LAUNCH_CHECK();
        MAF_CUDA(cudaDeviceSynchronize());
    }
    return Nred32_.as<float>();
}

template <> cplx_t<double>* Demag::S1<double>() {
    S1_64_.ensure(sizeof(double2) * 3 * md_.N() / md_.nx * pitch_);
    return S1_64_.as<double2>();
}
template <> cplx_t<float>* Demag::S1<float>() {
    S1_32_.ensure(sizeof(float2) * 3 * md_.N() / md_.nx * pitch_);
    return S1_32_.as<float2>();
}
template <> cplx_t<double>* Demag::S2<double>() {
    S2_64_.ensure(sizeof(double2) * 3 * (int64_t)md_.nz * Py() * pitch_);
    return S2_64_.as<double2>();
}
template <> cplx_t<float>* Demag::S2<float>() {
    S2_32_.ensure(sizeof(float2) * 3 * (int64_t)md_.nz * Py() * pitch_);
    return S2_32_.as<float2>();
}

template <typename R> void Demag::forward_conv(const R* m, const MsInfo& ms, cudaStream_t st, PassMarks* marks) {
    using C = cplx_t<R>;
    const bool f64 = sizeof(R) == 8;
    const int nx = md_.nx, ny = md_.ny, nz = md_.nz;
    const int64_t rows_pc = (int64_t)ny * nz;
    const R* msf = nullptr;
    if (ms.field64) {
        if constexpr (sizeof(R) == 4) msf = reinterpret_cast<const R*>(ms.field32);
        else msf = reinterpret_cast<const R*>(ms.field64);
    }
    C* s1 = S1<R>();
    // the periodic form has no tensor and runs the run-time plans only
    const R* Nr = pbc_ ? nullptr : tensor<R>();
    const bool ct = !pbc_ && !tune.generic;
    const PbcOp pop{nx, ny, nz, md_.dx, md_.dy, md_.dz};
    // pass 1: x forward (zero pad fused)
    launch_xfwd<R>(m, nx, 3 * rows_pc, rows_pc, msf, (R)ms.Ms, s1, pitch_, Px(), tw_, st, ct);
    if (marks) marks->mark(st, "x_fwd");
    if (nz > 1) {
        C* s2 = S2<R>();
        // pass 2: y forward, S1 [3*nz][ny][pitch] -> S2 [3*nz][Py][pitch]
        launch_cols<R, -1>(s1, s2, Py(), ny, Py(), nxh(), pitch_, pitch_, (int64_t)ny * pitch_,
                           (int64_t)Py() * pitch_, 3 * nz, tw_, tune, st, ct);
        if (marks) marks->mark(st, "y_fwd");
        // pass 3: z forward . tensor . z inverse, in place on S2
        if (!ct || !ct_convz<R>(s2, Nr, nz, ny, nxh(), pitch_, tw_, tune, st)) {
            const int L = Pz();
            FFTPlan fp = make_fft_plan(L, tw_.get(L, f64));
            FFTPlan ip = fp;
            int nb = pick_nb(3 * L, tile_target<R>(), nxh(), 64);
            int threads;
            while (true) {
                threads = std::max(fft_threads_needed(fp, 3 * nb), std::min(256, 3 * nb * L));
                if (threads <= kMaxFftThreads || nb == 1) break;
                nb = std::max(1, nb / 2);
            }
            threads = round_threads(threads);
            const size_t smem = sizeof(C) * (size_t)3 * nb * spad_len(L);
            dim3 grid((unsigned)ceil_div(nxh(), nb), (unsigned)Py());
            if (pbc_) {
                set_smem(k_conv<R, true>, smem);
                k_conv<R, true><<<grid, threads, smem, st>>>(s2, Nr, fp, ip, nz, (int64_t)Py() * pitch_,
                                                             (int64_t)nz * Py() * pitch_, pitch_, nxh(), nb, 1, ny,
                                                             nz, nxh(), pop);
            } else {
                set_smem(k_conv<R, false>, smem);
                k_conv<R, false><<<grid, threads, smem, st>>>(s2, Nr, fp, ip, nz, (int64_t)Py() * pitch_,
                                                              (int64_t)nz * Py() * pitch_, pitch_, nxh(), nb, 1, ny,
                                                              nz, nxh(), pop);
            }
            MAF_LAUNCH_CHECK();
        }
        if (marks) marks->mark(st, "z_conv");
        // pass 4: y inverse, S2 -> S1, keep ky rows [0, ny)
        launch_cols<R, 1>(s2, s1, Py(), Py(), ny, nxh(), pitch_, pitch_, (int64_t)Py() * pitch_,
                          (int64_t)ny * pitch_, 3 * nz, tw_, tune, st, ct);
        if (marks) marks->mark(st, "y_inv");
    } else {
        // pass 2 (2-D): y forward . tensor . y inverse, in place on S1
        if (ct && ct_convy<R>(s1, Nr, ny, nxh(), pitch_, tw_, st)) {
            if (marks) marks->mark(st, "y_conv");
            return;
        }
        const int L = Py();
        FFTPlan fp = make_fft_plan(L, tw_.get(L, f64));
        int nb = pick_nb(3 * L, tile_target<R>(), nxh(), 64);
        int threads;
        while (true) {
            threads = std::max(fft_threads_needed(fp, 3 * nb), std::min(256, 3 * nb * L));
            if (threads <= kMaxFftThreads || nb == 1) break;
            nb = std::max(1, nb / 2);
        }
        threads = round_threads(threads);
        const size_t smem = sizeof(C) * (size_t)3 * nb * spad_len(L);
        dim3 grid((unsigned)ceil_div(nxh(), nb), 1);
        if (pbc_) {
            set_smem(k_conv<R, true>, smem);
            k_conv<R, true><<<grid, threads, smem, st>>>(s1, Nr, fp, fp, ny, pitch_, (int64_t)ny * pitch_, 0, nxh(),
                                                         nb, 0, ny, nz, nxh(), pop);
        } else {
            set_smem(k_conv<R, false>, smem);
            k_conv<R, false><<<grid, threads, smem, st>>>(s1, Nr, fp, fp, ny, pitch_, (int64_t)ny * pitch_, 0, nxh(),
                                                          nb, 0, ny, nz, nxh(), pop);
        }
        MAF_LAUNCH_CHECK();
        if (marks) marks->mark(st, "y_conv");
    }
}

template <typename R> int Demag::edens_blocks() const { return 0; }

template <typename R>
void Demag::inverse_x_epilogue(const R* m, const MsInfo& ms, const TermList& tl, const EpilogueArgs& ep,
                               cudaStream_t st, int* nblocks_out, PassMarks* marks) {
    const bool f64 = sizeof(R) == 8;
    const int Lc = Px() / 2;
    if (!pbc_ && !tune.generic) {
        const R scale = (R)(1.0 / ((double)Px() * Py() * Pz()));
        if (ct_xinv<R>(S1<R>(), pitch_, Px(), tw_, md_.geom(), scale, m, ms, tl, ep, tune, st, nblocks_out)) {
            if (marks) marks->mark(st, "x_inv_local");
            return;
        }
    }
    FFTPlan plan = make_fft_plan(Lc, tw_.get(Lc, f64));
    const int64_t rows_pc = (int64_t)md_.ny * md_.nz;
    int nbr = pick_nb(3 * Lc, tile_target<R>(), (int)std::min<int64_t>(rows_pc, 1 << 20), 32);
    int threads;
    while (true) {
        threads = std::max(fft_threads_needed(plan, 3 * nbr), std::min(256, 3 * nbr * Lc));
        if (threads <= kMaxFftThreads || nbr == 1) break;
        nbr = std::max(1, nbr / 2);
    }
    threads = round_threads(threads);
    const size_t smem = sizeof(cplx_t<R>) * (size_t)3 * nbr * spad_len(Lc);
    const int64_t blocks = ceil_div(rows_pc, nbr);
    if (nblocks_out) *nblocks_out = (int)blocks;
    const R scale = (R)(1.0 / ((double)Px() * Py() * Pz()));
    const cplx_t<R>* tP = static_cast<const cplx_t<R>*>(tw_.get(Px(), f64));
    const Geom g = md_.geom();
    switch (ep.kind) {
        case EPI_H:
            set_smem(k_xinv_epi<R, EPI_H>, smem);
            k_xinv_epi<R, EPI_H><<<(unsigned)blocks, threads, smem, st>>>(S1<R>(), pitch_, plan, tP, g, scale, m, ms,
                                                                          tl, ep, nbr);
            break;
        case EPI_LLG:
            set_smem(k_xinv_epi<R, EPI_LLG>, smem);
            k_xinv_epi<R, EPI_LLG><<<(unsigned)blocks, threads, smem, st>>>(S1<R>(), pitch_, plan, tP, g, scale, m,
                                                                            ms, tl, ep, nbr);
            break;
        case EPI_EGRAD:
            set_smem(k_xinv_epi<R, EPI_EGRAD>, smem);
            k_xinv_epi<R, EPI_EGRAD><<<(unsigned)blocks, threads, smem, st>>>(S1<R>(), pitch_, plan, tP, g, scale, m,
                                                                              ms, tl, ep, nbr);
            break;
        default:
            set_smem(k_xinv_epi<R, EPI_EDENS>, smem);
            k_xinv_epi<R, EPI_EDENS><<<(unsigned)blocks, threads, smem, st>>>(S1<R>(), pitch_, plan, tP, g, scale, m,
                                                                              ms, tl, ep, nbr);
            break;
    }
    MAF_LAUNCH_CHECK();
    if (marks) marks->mark(st, "x_inv_local");
}

template void Demag::forward_conv<float>(const float*, const MsInfo&, cudaStream_t, PassMarks*);
template void Demag::forward_conv<double>(const double*, const MsInfo&, cudaStream_t, PassMarks*);
template void Demag::inverse_x_epilogue<float>(const float*, const MsInfo&, const TermList&, const EpilogueArgs&,
                                               cudaStream_t, int*, PassMarks*);
template void Demag::inverse_x_epilogue<double>(const double*, const MsInfo&, const TermList&, const EpilogueArgs&,
                                                cudaStream_t, int*, PassMarks*);

// ---------------------------------------------------------------------------
// field evaluation of a term list
// ---------------------------------------------------------------------------
template <typename R>
void eval_terms(const std::vector<Term*>& terms, const MeshDims& md, const R* m, const MsInfo& ms,
                const EpilogueArgs& ep_in, cudaStream_t st, DevBuf& scratch, double* energy_out,
                PassMarks* marks) {
    if (terms.empty()) throw Error(1, "no field terms");
    if ((int)terms.size() > kMaxTerms) throw Error(1, "too many field terms (max 8)");
    TermList tl;
    Demag* demag = nullptr;
    for (Term* t : terms) {
        if (t->kind == TK_DEMAG) {
            if (demag) throw Error(1, "at most one DemagField per term list");
            if (t->demag_pbc() && !(t->demag && t->demag_mesh == md)) {
                // DemagFieldPBC takes its mesh from the state: plan it on first use
                t->demag = std::make_unique<Demag>(md, st, nullptr, true);
                t->demag_mesh = md;
            }
            if (!(t->demag_mesh == md)) throw Error(1, "DemagField mesh differs from the state's mesh");
            demag = t->demag.get();
        }
        if (t->field_cells && t->field_cells != md.N())
            throw Error(1, "field-term parameter array does not match the state's mesh");
        if (t->kind == TK_BULKDMI && (md.nx < 2 || md.ny < 2 || md.nz < 2))
            throw Error(1, "BulkDMIExchangeField needs at least 2 cells along x, y and z");
        tl.t[tl.n++] = t->desc();
    }
    EpilogueArgs ep = ep_in;
    int nblocks = 0;
    if (ep.kind == EPI_EDENS || ep.kind == EPI_EGRAD) {
        // upper bound of CTAs for the partial sums
        const int64_t maxb = std::max<int64_t>(md.N(), (int64_t)sm_count() * 8) + 1;
        scratch.ensure(sizeof(double) * (maxb + 1));
        ep.partials = scratch.as<double>();
    }
    if (demag) {
        if (marks) marks->mark(st, "start");
        demag->forward_conv<R>(m, ms, st, marks);
        demag->inverse_x_epilogue<R>(m, ms, tl, ep, st, &nblocks, marks);
    } else if (run4_eligible(md.geom(), m, ms, tl, ep) && md.N() / 4 < (int64_t)INT32_MAX) {
        // scalar parameters, no Ms field, nx % 4 == 0: runs of four cells with
        // per-launch term constants (no division in the cell loop)
        constexpr int RN = 4;
        const Geom g = md.geom();
        prepare_run4(tl, g, ms.Ms);
        const int nruns = (int)(md.N() / RN);
        const int threads = 256;
        const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nruns, threads), (int64_t)sm_count() * 16);
        if (marks) marks->mark(st, "start");
        if (ep.kind == EPI_H)
            k_local_run<R, EPI_H, RN><<<blocks, threads, 0, st>>>(g, m, tl, ep, nruns);
        else
            k_local_run<R, EPI_LLG, RN><<<blocks, threads, 0, st>>>(g, m, tl, ep, nruns);
        MAF_LAUNCH_CHECK();
        if (marks) marks->mark(st, "local");
    } else {
        const int threads = 256;
        const int64_t blocks = std::min<int64_t>(ceil_div(md.N(), threads), (int64_t)sm_count() * 8);
        nblocks = (int)blocks;
        const Geom g = md.geom();
        if (marks) marks->mark(st, "start");
        switch (ep.kind) {
            case EPI_H: k_local_epi<R, EPI_H><<<(unsigned)blocks, threads, 0, st>>>(g, m, ms, tl, ep); break;
            case EPI_LLG: k_local_epi<R, EPI_LLG><<<(unsigned)blocks, threads, 0, st>>>(g, m, ms, tl, ep); break;
            case EPI_EGRAD: k_local_epi<R, EPI_EGRAD><<<(unsigned)blocks, threads, 0, st>>>(g, m, ms, tl, ep); break;
            default: k_local_epi<R, EPI_EDENS><<<(unsigned)blocks, threads, 0, st>>>(g, m, ms, tl, ep); break;
        }
        MAF_LAUNCH_CHECK();
        if (marks) marks->mark(st, "local");
    }
    if (ep.kind == EPI_EDENS || ep.kind == EPI_EGRAD) {
        double* dst = ep_in.energy_dev ? ep_in.energy_dev : ep.partials + nblocks;
        k_sum_partials<<<1, 256, 0, st>>>(ep.partials, nblocks, dst);
        MAF_LAUNCH_CHECK();
        if (ep_in.energy_dev) return;  // the caller reads it back
        double e = 0;
        MAF_CUDA(cudaMemcpyAsync(&e, dst, sizeof(double), cudaMemcpyDeviceToHost, st));
        MAF_CUDA(cudaStreamSynchronize(st));
        if (energy_out) *energy_out = e * md.dx * md.dy * md.dz;
    }
}

template void eval_terms<float>(const std::vector<Term*>&, const MeshDims&, const float*, const MsInfo&,
                                const EpilogueArgs&, cudaStream_t, DevBuf&, double*, PassMarks*);
template void eval_terms<double>(const std::vector<Term*>&, const MeshDims&, const double*, const MsInfo&,
                                 const EpilogueArgs&, cudaStream_t, DevBuf&, double*, PassMarks*);

}  // namespace mafb
