// Batched passes of an ensemble of 2-D states (batch.hpp): every pass of a
// fixed-step stochastic / RK4 step is one launch per transform length over a
// device work table of (member, tile) pairs, the launches of a pass on
// parallel graph branches.  Members whose lengths have compile-time kernels run
// those kernels' tile bodies (fields_ct.cu), the others the generic kernels'
// (run-time FFT plans, passes_generic.cuh); members of a DemagField set to the
// run-time-plan kernels run those.  The element-wise kernels repeat the
// arithmetic of llg.cu's, so a member's trajectory is bit-identical to the one
// the per-state path computes with the same kernels.
#include <algorithm>
#include <cstring>

#include "batch.hpp"
#include "ct_dispatch.hpp"
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

// The members of one compile-time kernel of a pass (same transform length L and,
// for the x inverse, run length): their argument items, [parity][stage][member
// of the class] for the x passes and [member of the class] for the convolution,
// and the work table of (member of the class, tile).
struct CtClass {
    int L = 0, run = 0;
    std::vector<int> members;
    DevBuf items, work;
    int nwork = 0;
    const void* tw = nullptr;
    const void* twP = nullptr;
};

// The members of a pass on the generic kernels with one transform length: their
// work table of (member, tile) and the CTA shape the per-state launch uses.
struct GenClass {
    int L = 0;
    std::vector<int2> w;
    DevBuf work;
    int nwork = 0, threads = 32;
    size_t smem = 0;
};

struct FusedBatch::Impl {
    bool f32 = false;
    int M = 0, S = 0;
    FusedScheme scheme;
    std::vector<FusedMember> mem;
    // generic-kernel argument arrays: [parity][stage][member] (x passes), [member] (conv)
    DevBuf xfwd, conv, xinv, comb, fin, stage32, qptr;
    DevBuf w_el3, w_cell;
    int n_el3 = 0, n_cell = 0;
    // the launches of a pass: one per transform length (generic and compile-time)
    std::vector<GenClass> gx, gc, gi;
    std::vector<CtClass> cx, cc, ci;
    // the launches of a pass run on parallel branches: side streams and fork/join events
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;
    cudaEvent_t fork_ev = nullptr;

    ~Impl() {
        for (cudaStream_t q : side) cudaStreamDestroy(q);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        if (fork_ev) cudaEventDestroy(fork_ev);
    }
    template <typename R> void build(cudaStream_t st);
    template <typename R> void record(cudaStream_t st, int p);
    // runs launch(b, stream) for b < n, branch 0 on st and the others on side streams
    template <typename F> void branches(cudaStream_t st, int n, F&& launch);
};

template <typename F> void FusedBatch::Impl::branches(cudaStream_t st, int n, F&& launch) {
    if (n <= 1) {
        if (n == 1) launch(0, st);
        return;
    }
    MAF_CUDA(cudaEventRecord(fork_ev, st));
    for (int b = 1; b < n; ++b) MAF_CUDA(cudaStreamWaitEvent(side[b - 1], fork_ev, 0));
    launch(0, st);
    for (int b = 1; b < n; ++b) {
        launch(b, side[b - 1]);
        MAF_CUDA(cudaEventRecord(ev[b - 1], side[b - 1]));
        MAF_CUDA(cudaStreamWaitEvent(st, ev[b - 1], 0));
    }
}

// the class of cls with length L (and run), created on first use
static CtClass& ct_class(std::vector<CtClass>& cls, int L, int run) {
    for (CtClass& c : cls)
        if (c.L == L && c.run == run) return c;
    cls.emplace_back();
    cls.back().L = L;
    cls.back().run = run;
    return cls.back();
}

static GenClass& gen_class(std::vector<GenClass>& cls, int L) {
    for (GenClass& c : cls)
        if (c.L == L) return c;
    cls.emplace_back();
    cls.back().L = L;
    return cls.back();
}

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
    std::vector<int2> we, wn;
    // compile-time kernel per pass and member (the per-state path's choice: ct_xfwd,
    // ct_convy and ct_xinv run for these lengths unless the DemagField is set to the
    // run-time-plan kernels); cx_of[i] etc.: the member's class, -1 for generic
    std::vector<int> cx_of(M, -1), cc_of(M, -1), ci_of(M, -1), pos_x(M), pos_c(M), pos_i(M);
    for (int i = 0; i < M; ++i) {
        Demag* dm = mem[i].demag;
        if (dm->tune.generic) continue;
        const int Lc = dm->Px() / 2, Py = dm->Py();
        const int run = dm->tune.xinv_run ? dm->tune.xinv_run : 2;
        if (ct_batch_tile<R>(0, Lc) > 0) {
            CtClass& c = ct_class(cx, Lc, 0);
            cx_of[i] = (int)(&c - cx.data());
            pos_x[i] = (int)c.members.size();
            c.members.push_back(i);
        }
        if (ct_batch_tile<R>(1, Py) > 0) {
            CtClass& c = ct_class(cc, Py, 0);
            cc_of[i] = (int)(&c - cc.data());
            pos_c[i] = (int)c.members.size();
            c.members.push_back(i);
        }
        if (ct_batch_tile<R>(2, Lc) > 0 && mem[i].md.nx == Lc) {
            CtClass& c = ct_class(ci, Lc, run);
            ci_of[i] = (int)(&c - ci.data());
            pos_i[i] = (int)c.members.size();
            c.members.push_back(i);
        }
    }
    std::vector<std::vector<CtXfwdItem<R>>> ixf(cx.size());
    std::vector<std::vector<CtConvyItem<R>>> icv(cc.size());
    std::vector<std::vector<CtXinvItem<R>>> ixi(ci.size());
    std::vector<std::vector<int2>> wcx(cx.size()), wcc(cc.size()), wci(ci.size());
    for (size_t c = 0; c < cx.size(); ++c) ixf[c].resize((size_t)2 * S * cx[c].members.size());
    for (size_t c = 0; c < cc.size(); ++c) icv[c].resize(cc[c].members.size());
    for (size_t c = 0; c < ci.size(); ++c) ixi[c].resize((size_t)2 * S * ci[c].members.size());
    for (int i = 0; i < M; ++i) {
        const FusedMember& f = mem[i];
        Demag* dm = f.demag;
        const int nx = f.md.nx, ny = f.md.ny;
        const int64_t N = f.md.N(), rows_pc = (int64_t)ny * f.md.nz;
        const int Px = dm->Px(), Py = dm->Py(), Lc = Px / 2, nxh = dm->nxh(), pitch = dm->pitch();
        C* s1 = dm->spectrum<R>();
        if (cx_of[i] >= 0) {
            CtClass& c = cx[cx_of[i]];
            if (!c.tw) {
                c.tw = ct_batch_twiddles<R>(0, Lc, dm->twiddle_tables());
                c.twP = dm->twiddles(Px, f64);
            }
            add_items(wcx[cx_of[i]], pos_x[i], ceil_div(3 * rows_pc, ct_batch_tile<R>(0, Lc)));
        }
        if (cc_of[i] >= 0) {
            CtClass& c = cc[cc_of[i]];
            if (!c.tw) c.tw = ct_batch_twiddles<R>(1, Py, dm->twiddle_tables());
            add_items(wcc[cc_of[i]], pos_c[i], ceil_div(nxh, ct_batch_tile<R>(1, Py)));
            icv[cc_of[i]][pos_c[i]] = CtConvyItem<R>{s1, dm->tensor_data<R>(), nxh, pitch};
        }
        if (ci_of[i] >= 0) {
            CtClass& c = ci[ci_of[i]];
            if (!c.tw) {
                c.tw = ct_batch_twiddles<R>(2, Lc, dm->twiddle_tables());
                c.twP = dm->twiddles(Px, f64);
            }
            add_items(wci[ci_of[i]], pos_i[i], ceil_div(rows_pc, ct_batch_tile<R>(2, Lc)));
        }
        // x forward (launch_xfwd's generic shape)
        const FFTPlan px = make_fft_plan(Lc, dm->twiddles(Lc, f64));
        int nbx = pick_nb(Lc, tile_target<R>(), (int)std::min<int64_t>(3 * rows_pc, 1 << 20), 64);
        while (true) {
            const int th = std::max(fft_threads_needed(px, nbx), std::min(256, nbx * Lc));
            if (th <= kMaxFftThreads || nbx == 1) break;
            nbx = std::max(1, nbx / 2);
        }
        if (cx_of[i] < 0) {
            GenClass& g = gen_class(gx, Lc);
            g.threads = std::max(g.threads, tile_threads(px, nbx, nbx * Lc));
            g.smem = std::max(g.smem, sizeof(C) * (size_t)nbx * spad_len(Lc));
            add_items(g.w, i, ceil_div(3 * rows_pc, nbx));
        }
        // y convolution (forward_conv's generic nz == 1 shape)
        const FFTPlan py = make_fft_plan(Py, dm->twiddles(Py, f64));
        int nbc = pick_nb(3 * Py, tile_target<R>(), nxh, 64);
        while (true) {
            const int th = std::max(fft_threads_needed(py, 3 * nbc), std::min(256, 3 * nbc * Py));
            if (th <= kMaxFftThreads || nbc == 1) break;
            nbc = std::max(1, nbc / 2);
        }
        if (cc_of[i] < 0) {
            GenClass& g = gen_class(gc, Py);
            g.threads = std::max(g.threads, tile_threads(py, 3 * nbc, 3 * nbc * Py));
            g.smem = std::max(g.smem, sizeof(C) * (size_t)3 * nbc * spad_len(Py));
            add_items(g.w, i, ceil_div(nxh, nbc));
        }
        cv[i] = ConvA<R>{s1, dm->tensor_data<R>(), py, ny, (int64_t)pitch, (int64_t)ny * pitch, nxh, nbc, ny, 1, nxh};
        // x inverse + LLG epilogue (inverse_x_epilogue's generic shape)
        int nbr = pick_nb(3 * Lc, tile_target<R>(), (int)std::min<int64_t>(rows_pc, 1 << 20), 32);
        while (true) {
            const int th = std::max(fft_threads_needed(px, 3 * nbr), std::min(256, 3 * nbr * Lc));
            if (th <= kMaxFftThreads || nbr == 1) break;
            nbr = std::max(1, nbr / 2);
        }
        if (ci_of[i] < 0) {
            GenClass& g = gen_class(gi, Lc);
            g.threads = std::max(g.threads, tile_threads(px, 3 * nbr, 3 * nbr * Lc));
            g.smem = std::max(g.smem, sizeof(C) * (size_t)3 * nbr * spad_len(Lc));
            add_items(g.w, i, ceil_div(rows_pc, nbr));
        }
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
                if (cx_of[i] >= 0) {
                    const size_t nc = cx[cx_of[i]].members.size();
                    ixf[cx_of[i]][((size_t)p * S + s) * nc + pos_x[i]] =
                        CtXfwdItem<R>{in, nx, 3 * rows_pc, (R)f.Ms, s1, pitch};
                }
                if (ci_of[i] >= 0) {
                    const size_t nc = ci[ci_of[i]].members.size();
                    CtXinvItem<R> it{s1, pitch, f.md.geom(), scale, in, ms, tl, ep, 0};
                    ct_batch_xinv_prepare<R>(it);
                    ixi[ci_of[i]][((size_t)p * S + s) * nc + pos_i[i]] = it;
                }
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
    size_t s_xfwd = 0, s_conv = 0, s_xinv = 0;
    for (std::vector<GenClass>* v : {&gx, &gc, &gi})
        for (GenClass& g : *v) {
            upload(g.work, g.w, st);
            g.nwork = (int)g.w.size();
        }
    for (const GenClass& g : gx) s_xfwd = std::max(s_xfwd, g.smem);
    for (const GenClass& g : gc) s_conv = std::max(s_conv, g.smem);
    for (const GenClass& g : gi) s_xinv = std::max(s_xinv, g.smem);
    for (size_t c = 0; c < cx.size(); ++c) {
        upload(cx[c].items, ixf[c], st);
        upload(cx[c].work, wcx[c], st);
        cx[c].nwork = (int)wcx[c].size();
    }
    for (size_t c = 0; c < cc.size(); ++c) {
        upload(cc[c].items, icv[c], st);
        upload(cc[c].work, wcc[c], st);
        cc[c].nwork = (int)wcc[c].size();
    }
    for (size_t c = 0; c < ci.size(); ++c) {
        upload(ci[c].items, ixi[c], st);
        upload(ci[c].work, wci[c], st);
        ci[c].nwork = (int)wci[c].size();
    }
    upload(w_el3, we, st);
    upload(w_cell, wn, st);
    const size_t nbr_max = std::max({gx.size() + cx.size(), gc.size() + cc.size(), gi.size() + ci.size(), (size_t)1});
    for (size_t b = 1; b < nbr_max; ++b) {
        cudaStream_t q;
        MAF_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        side.push_back(q);
        cudaEvent_t e;
        MAF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
    }
    MAF_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
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
        const int ngx = (int)gx.size(), ngc = (int)gc.size(), ngi = (int)gi.size();
        branches(st, ngx + (int)cx.size(), [&](int b, cudaStream_t q) {
            if (b < ngx) {
                const GenClass& g = gx[b];
                kb_xfwd<R><<<g.nwork, g.threads, g.smem, q>>>(xfwd.as<XfwdA<R>>() + a, g.work.as<int2>());
                MAF_LAUNCH_CHECK();
            } else {
                const CtClass& c = cx[b - ngx];
                ct_batch_xfwd<R>(c.items.as<CtXfwdItem<R>>() + ((size_t)p * S + s) * c.members.size(),
                                 c.work.as<int2>(), c.nwork, c.L, c.tw, c.twP, q);
            }
        });
        branches(st, ngc + (int)cc.size(), [&](int b, cudaStream_t q) {
            if (b < ngc) {
                const GenClass& g = gc[b];
                kb_conv<R><<<g.nwork, g.threads, g.smem, q>>>(conv.as<ConvA<R>>(), g.work.as<int2>());
                MAF_LAUNCH_CHECK();
            } else {
                const CtClass& c = cc[b - ngc];
                ct_batch_convy<R>(c.items.as<CtConvyItem<R>>(), c.work.as<int2>(), c.nwork, c.L, c.tw, q);
            }
        });
        branches(st, ngi + (int)ci.size(), [&](int b, cudaStream_t q) {
            if (b < ngi) {
                const GenClass& g = gi[b];
                kb_xinv<R><<<g.nwork, g.threads, g.smem, q>>>(xinv.as<XinvA<R>>() + a, g.work.as<int2>());
                MAF_LAUNCH_CHECK();
            } else {
                const CtClass& c = ci[b - ngi];
                ct_batch_xinv<R>(c.items.as<CtXinvItem<R>>() + ((size_t)p * S + s) * c.members.size(),
                                 c.work.as<int2>(), c.nwork, c.L, c.run, c.tw, c.twP, q);
            }
        });
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

int FusedBatch::launches_per_step() const {
    const Impl& b = *impl_;
    const int per_stage = (int)(b.gx.size() + b.gc.size() + b.gi.size() + b.cx.size() + b.cc.size() + b.ci.size());
    return (b.f32 ? 1 : 0) + b.S * (per_stage + 1) - 1 + 2;
}

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
