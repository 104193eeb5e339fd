// Batched passes of an ensemble of 2-D states (batch.hpp): every pass of a
// fixed-step stochastic / RK4 step is one launch over a device work table of
// (member, tile) pairs.  The tile bodies are the generic kernels' (run-time
// FFT plans, passes_generic.cuh) and the element-wise kernels repeat the
// arithmetic of llg.cu's, so a member's trajectory is bit-identical to the one
// the per-state path computes with its generic kernels.
#include <algorithm>
#include <cstring>

#include "batch.hpp"
#include "passes_generic.cuh"

namespace mafb {

namespace {

constexpr int kElemThreads = 256;
constexpr int kElemPerThread = 4;
constexpr int kElemChunk = kElemThreads * kElemPerThread;  // values per work item of the element-wise kernels

template <typename R> struct XfwdA {
    const R* in;
    int n_in;
    int64_t rows, rows_pc;
    R ms;
    cplx_t<R>* out;
    int pitch;
    FFTPlan plan;
    const cplx_t<R>* twP;
    int nb;
};

template <typename R> struct ConvA {
    cplx_t<R>* S;
    const R* Nred;
    FFTPlan plan;
    int n_in;
    int64_t si, comp_stride;
    int ncols, nb, ny, nz, nxh;
};

template <typename R> struct XinvA {
    const cplx_t<R>* S1;
    int pitch;
    FFTPlan plan;
    const cplx_t<R>* twP;
    Geom g;
    R scale;
    const R* m;
    MsInfo ms;
    TermList tl;
    EpilogueArgs ep;
    int nbr;
};

struct StageA {  // FP32 copy of the stage-0 m
    const double* m;
    float* o;
    int64_t n;
};

struct CombA {  // m_s = m + sum_t c[t] k[t]
    const double* m;
    const double* k[6];
    double c[6];
    int n;
    double* o64;
    float* o32;
    int64_t len;
};

struct FinA {  // out = normalise0(m + sum_t c[t] k[t]) per cell
    const double* m;
    const double* k[6];
    double c[6];
    int n;
    double* out;
    int64_t N;
};

template <typename R>
__global__ void __launch_bounds__(kMaxFftThreads) kb_xfwd(const XfwdA<R>* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const XfwdA<R>& d = a[t.x];
    xfwd_tile<R>(d.in, d.n_in, d.rows, d.rows_pc, nullptr, d.ms, d.out, d.pitch, d.plan, d.twP, d.nb, t.y);
}

template <typename R>
__global__ void __launch_bounds__(kMaxFftThreads) kb_conv(const ConvA<R>* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const ConvA<R>& d = a[t.x];
    const PbcOp none{1, 1, 1, 1.0, 1.0, 1.0};
    conv_tile<R, false>(d.S, d.Nred, d.plan, d.plan, d.n_in, d.si, d.comp_stride, 0, d.ncols, d.nb, 0, d.ny, d.nz,
                        d.nxh, none, t.y, 0);
}

template <typename R>
__global__ void __launch_bounds__(kMaxFftThreads) kb_xinv(const XinvA<R>* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const XinvA<R>& d = a[t.x];
    xinv_tile<R, EPI_LLG>(d.S1, d.pitch, d.plan, d.twP, d.g, d.scale, d.m, d.ms, d.tl, d.ep, d.nbr, t.y, 0);
}

__global__ void __launch_bounds__(kElemThreads) kb_stage32(const StageA* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const StageA& d = a[t.x];
    const int64_t i0 = (int64_t)t.y * kElemChunk;
#pragma unroll
    for (int u = 0; u < kElemPerThread; ++u) {
        const int64_t i = i0 + u * kElemThreads + threadIdx.x;
        if (i < d.n) d.o[i] = (float)d.m[i];
    }
}

__global__ void __launch_bounds__(kElemThreads) kb_combine(const CombA* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const CombA& d = a[t.x];
    const int64_t i0 = (int64_t)t.y * kElemChunk;
#pragma unroll
    for (int u = 0; u < kElemPerThread; ++u) {
        const int64_t i = i0 + u * kElemThreads + threadIdx.x;
        if (i < d.len) {
            double acc = d.m[i];
            for (int j = 0; j < d.n; ++j) acc = acc + d.c[j] * d.k[j][i];
            d.o64[i] = acc;
            if (d.o32) d.o32[i] = (float)acc;
        }
    }
}

__global__ void __launch_bounds__(kElemThreads) kb_finalize(const FinA* __restrict__ a, const int2* __restrict__ w) {
    const int2 t = w[blockIdx.x];
    const FinA& d = a[t.x];
    const int64_t c0 = (int64_t)t.y * kElemChunk;
#pragma unroll
    for (int u = 0; u < kElemPerThread; ++u) {
        const int64_t cell = c0 + u * kElemThreads + threadIdx.x;
        if (cell >= d.N) continue;
        double o[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * d.N + cell;
            double sumbk = 0.0;
            for (int j = 0; j < d.n; ++j) sumbk = sumbk + d.c[j] * d.k[j][i];
            o[c] = d.m[i] + sumbk;
        }
        // the zero-safe normalisation (util.cpp:52), as rk_finalize's mode 2
        const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        if (nrm != 0) {
            o[0] /= nrm; o[1] /= nrm; o[2] /= nrm;
        } else {
            o[0] = 0; o[1] = 0; o[2] = 0;
        }
        d.out[cell] = o[0];
        d.out[d.N + cell] = o[1];
        d.out[2 * d.N + cell] = o[2];
    }
}

__global__ void kb_inc(unsigned long long* const* __restrict__ q, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i][0] += 1ull;
}

template <typename T> void upload(DevBuf& buf, const std::vector<T>& v, cudaStream_t st) {
    buf.alloc(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) MAF_CUDA(cudaMemcpyAsync(buf.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
}

void add_items(std::vector<int2>& w, int member, int64_t tiles) {
    for (int64_t t = 0; t < tiles; ++t) w.push_back(make_int2(member, (int)t));
}

// threads of a generic FFT tile, as the per-state launches choose them
int tile_threads(const FFTPlan& p, int ncols, int elems) {
    return round_threads(std::max(fft_threads_needed(p, ncols), std::min(256, elems)));
}

}  // namespace

struct FusedBatch::Impl {
    bool f32 = false;
    int M = 0, S = 0;
    FusedScheme scheme;
    std::vector<FusedMember> mem;
    // argument arrays: [parity][stage][member] (x passes), [member] (conv)
    DevBuf xfwd, conv, xinv, comb, fin, stage32, qptr;
    DevBuf w_xfwd, w_conv, w_xinv, w_el3, w_cell;
    int n_xfwd = 0, n_conv = 0, n_xinv = 0, n_el3 = 0, n_cell = 0;
    int t_xfwd = 32, t_conv = 32, t_xinv = 32;
    size_t s_xfwd = 0, s_conv = 0, s_xinv = 0;

    template <typename R> void build(cudaStream_t st);
    template <typename R> void record(cudaStream_t st, int p);
};

template <typename R> void FusedBatch::Impl::build(cudaStream_t st) {
    using C = cplx_t<R>;
    const bool f64 = sizeof(R) == 8;
    std::vector<XfwdA<R>> xf((size_t)2 * S * M);
    std::vector<XinvA<R>> xi((size_t)2 * S * M);
    std::vector<ConvA<R>> cv(M);
    std::vector<CombA> cb((size_t)2 * S * M);
    std::vector<FinA> fn((size_t)2 * M);
    std::vector<StageA> sg((size_t)2 * M);
    std::vector<unsigned long long*> qs(M);
    std::vector<int2> wx, wc, wi, we, wn;
    for (int i = 0; i < M; ++i) {
        const FusedMember& f = mem[i];
        Demag* dm = f.demag;
        const int nx = f.md.nx, ny = f.md.ny;
        const int64_t N = f.md.N(), rows_pc = (int64_t)ny * f.md.nz;
        const int Px = dm->Px(), Py = dm->Py(), Lc = Px / 2, nxh = dm->nxh(), pitch = dm->pitch();
        C* s1 = dm->spectrum<R>();
        // x forward (launch_xfwd's generic shape)
        const FFTPlan px = make_fft_plan(Lc, dm->twiddles(Lc, f64));
        int nbx = pick_nb(Lc, tile_target<R>(), (int)std::min<int64_t>(3 * rows_pc, 1 << 20), 64);
        while (true) {
            const int th = std::max(fft_threads_needed(px, nbx), std::min(256, nbx * Lc));
            if (th <= kMaxFftThreads || nbx == 1) break;
            nbx = std::max(1, nbx / 2);
        }
        t_xfwd = std::max(t_xfwd, tile_threads(px, nbx, nbx * Lc));
        s_xfwd = std::max(s_xfwd, sizeof(C) * (size_t)nbx * spad_len(Lc));
        add_items(wx, i, ceil_div(3 * rows_pc, nbx));
        // y convolution (forward_conv's generic nz == 1 shape)
        const FFTPlan py = make_fft_plan(Py, dm->twiddles(Py, f64));
        int nbc = pick_nb(3 * Py, tile_target<R>(), nxh, 64);
        while (true) {
            const int th = std::max(fft_threads_needed(py, 3 * nbc), std::min(256, 3 * nbc * Py));
            if (th <= kMaxFftThreads || nbc == 1) break;
            nbc = std::max(1, nbc / 2);
        }
        t_conv = std::max(t_conv, tile_threads(py, 3 * nbc, 3 * nbc * Py));
        s_conv = std::max(s_conv, sizeof(C) * (size_t)3 * nbc * spad_len(Py));
        add_items(wc, i, ceil_div(nxh, nbc));
        cv[i] = ConvA<R>{s1, dm->tensor_data<R>(), py, ny, (int64_t)pitch, (int64_t)ny * pitch, nxh, nbc, ny, 1, nxh};
        // x inverse + LLG epilogue (inverse_x_epilogue's generic shape)
        int nbr = pick_nb(3 * Lc, tile_target<R>(), (int)std::min<int64_t>(rows_pc, 1 << 20), 32);
        while (true) {
            const int th = std::max(fft_threads_needed(px, 3 * nbr), std::min(256, 3 * nbr * Lc));
            if (th <= kMaxFftThreads || nbr == 1) break;
            nbr = std::max(1, nbr / 2);
        }
        t_xinv = std::max(t_xinv, tile_threads(px, 3 * nbr, 3 * nbr * Lc));
        s_xinv = std::max(s_xinv, sizeof(C) * (size_t)3 * nbr * spad_len(Lc));
        add_items(wi, i, ceil_div(rows_pc, nbr));
        add_items(we, i, ceil_div(3 * N, kElemChunk));
        add_items(wn, i, ceil_div(N, kElemChunk));
        TermList tl;
        for (const TermDesc& t : f.terms) tl.t[tl.n++] = t;
        MsInfo ms;
        ms.Ms = f.Ms;
        const C* twP = static_cast<const C*>(dm->twiddles(Px, f64));
        const R scale = (R)(1.0 / ((double)Px * Py * dm->Pz()));
        for (int p = 0; p < 2; ++p) {
            const double* mp = f.m[p];
            double* mo = f.m[1 - p];
            sg[(size_t)p * M + i] = StageA{mp, f.m32, 3 * N};
            for (int s = 0; s < S; ++s) {
                const FusedStage& fs = scheme.stages[s];
                const size_t a = ((size_t)p * S + s) * M + i;
                const R* in;
                if constexpr (sizeof(R) == 4) in = s == 0 ? f.m32 : f.mstage32;
                else in = s == 0 ? mp : f.mstage64;
                xf[a] = XfwdA<R>{in, nx, 3 * rows_pc, rows_pc, (R)f.Ms, s1, pitch, px, twP, nbx};
                EpilogueArgs ep;
                ep.kind = EPI_LLG;
                ep.out = f.k[s];
                ep.llg.c_prec = f.c_prec;
                ep.llg.c_damp = f.c_damp;
                ep.llg.scale = fs.scale;
                ep.llg.m64 = s == 0 ? mp : f.mstage64;
                if (fs.noise) {
                    ep.llg.sigma = f.sigma;
                    ep.llg.seed = f.seed;
                    ep.llg.member = f.member;
                    ep.llg.noise_base = f.q;
                    ep.llg.noise_mul = scheme.noise_mul;
                    ep.llg.noise_index = fs.offset;
                }
                xi[a] = XinvA<R>{s1, pitch, px, twP, f.md.geom(), scale, in, ms, tl, ep, nbr};
                CombA c{};
                c.m = mp;
                c.n = fs.n;
                for (int t = 0; t < fs.n; ++t) {
                    c.k[t] = f.k[fs.j[t]];
                    c.c[t] = fs.c[t];
                }
                c.o64 = f.mstage64;
                c.o32 = sizeof(R) == 4 ? f.mstage32 : nullptr;
                c.len = 3 * N;
                cb[a] = c;
            }
            FinA z{};
            z.m = mp;
            z.n = scheme.nfin;
            for (int t = 0; t < scheme.nfin; ++t) {
                z.k[t] = f.k[scheme.fin_base + t];
                z.c[t] = scheme.fin_c[t];
            }
            z.out = mo;
            z.N = N;
            fn[(size_t)p * M + i] = z;
        }
        qs[i] = f.q;
    }
    upload(xfwd, xf, st);
    upload(xinv, xi, st);
    upload(conv, cv, st);
    upload(comb, cb, st);
    upload(fin, fn, st);
    upload(stage32, sg, st);
    upload(qptr, qs, st);
    upload(w_xfwd, wx, st);
    upload(w_conv, wc, st);
    upload(w_xinv, wi, st);
    upload(w_el3, we, st);
    upload(w_cell, wn, st);
    n_xfwd = (int)wx.size();
    n_conv = (int)wc.size();
    n_xinv = (int)wi.size();
    n_el3 = (int)we.size();
    n_cell = (int)wn.size();
    auto smem_attr = [](auto k, size_t bytes) {
        if (bytes > 32 * 1024) MAF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    };
    smem_attr(kb_xfwd<R>, s_xfwd);
    smem_attr(kb_conv<R>, s_conv);
    smem_attr(kb_xinv<R>, s_xinv);
    MAF_CUDA(cudaStreamSynchronize(st));
}

template <typename R> void FusedBatch::Impl::record(cudaStream_t st, int p) {
    const size_t psm = (size_t)p * S * M;
    if (f32) {
        kb_stage32<<<n_el3, kElemThreads, 0, st>>>(stage32.as<StageA>() + (size_t)p * M, w_el3.as<int2>());
        MAF_LAUNCH_CHECK();
    }
    for (int s = 0; s < S; ++s) {
        const size_t a = psm + (size_t)s * M;
        if (s > 0) {
            kb_combine<<<n_el3, kElemThreads, 0, st>>>(comb.as<CombA>() + a, w_el3.as<int2>());
            MAF_LAUNCH_CHECK();
        }
        kb_xfwd<R><<<n_xfwd, t_xfwd, s_xfwd, st>>>(xfwd.as<XfwdA<R>>() + a, w_xfwd.as<int2>());
        MAF_LAUNCH_CHECK();
        kb_conv<R><<<n_conv, t_conv, s_conv, st>>>(conv.as<ConvA<R>>(), w_conv.as<int2>());
        MAF_LAUNCH_CHECK();
        kb_xinv<R><<<n_xinv, t_xinv, s_xinv, st>>>(xinv.as<XinvA<R>>() + a, w_xinv.as<int2>());
        MAF_LAUNCH_CHECK();
    }
    kb_finalize<<<n_cell, kElemThreads, 0, st>>>(fin.as<FinA>() + (size_t)p * M, w_cell.as<int2>());
    MAF_LAUNCH_CHECK();
    kb_inc<<<1, 256, 0, st>>>(qptr.as<unsigned long long*>(), M);
    MAF_LAUNCH_CHECK();
}

FusedBatch::FusedBatch(std::vector<FusedMember> members, FusedScheme scheme, bool f32, cudaStream_t st)
    : impl_(new Impl) {
    impl_->f32 = f32;
    impl_->M = (int)members.size();
    impl_->S = (int)scheme.stages.size();
    impl_->scheme = scheme;
    impl_->mem = std::move(members);
    try {
        if (f32)
            impl_->build<float>(st);
        else
            impl_->build<double>(st);
    } catch (...) {
        delete impl_;
        throw;
    }
}

FusedBatch::~FusedBatch() { delete impl_; }

void FusedBatch::record_step(cudaStream_t st, int parity) {
    if (impl_->f32)
        impl_->record<float>(st, parity & 1);
    else
        impl_->record<double>(st, parity & 1);
}

int FusedBatch::launches_per_step() const { return (impl_->f32 ? 1 : 0) + 4 * impl_->S - 1 + 2; }

bool fused_supported(const std::vector<FusedMember>& members, const FusedScheme& scheme) {
    if (members.empty() || scheme.stages.empty() || scheme.stages.size() > 6 || scheme.nfin < 1) return false;
    for (const FusedMember& f : members) {
        if (!f.demag || f.demag->pbc() || f.md.nz != 1 || f.terms.size() > (size_t)kMaxTerms) return false;
        int ndemag = 0;
        for (const TermDesc& t : f.terms) {
            if (t.kind == TK_DEMAG) ++ndemag;
            if (t.f0 || t.f1) return false;  // parameter fields: the per-state path
        }
        if (ndemag != 1) return false;
    }
    return true;
}

}  // namespace mafb
