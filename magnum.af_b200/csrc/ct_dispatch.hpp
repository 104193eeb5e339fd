// Compile-time specialised demag passes (fields_ct.cu).  Each returns false when
// no specialisation exists for the transform length; the caller then runs the
// generic kernel of fields.cu.
#pragma once
#include "engine.hpp"

namespace mafb {

template <typename R>
bool ct_xfwd(const R* in, int n_in, int64_t rows, int64_t rows_pc, const R* msf, R ms, cplx_t<R>* out, int pitch,
             int Px, Twiddles& tw, cudaStream_t st);
template <typename R, int DIR>
bool ct_cols(const cplx_t<R>* in, cplx_t<R>* out, int L, int n_in, int n_out, int ncols, int64_t in_si, int64_t out_si,
             int64_t in_sbat, int64_t out_sbat, int nbat, Twiddles& tw, const TuneChoice& tc, cudaStream_t st);
template <typename R>
bool ct_convz(cplx_t<R>* S, const R* Nred, int nz, int ny, int nxh, int pitch, Twiddles& tw, const TuneChoice& tc,
              cudaStream_t st);
template <typename R>
bool ct_convy(cplx_t<R>* S, const R* Nred, int ny, int nxh, int pitch, Twiddles& tw, cudaStream_t st);
template <typename R>
bool ct_xinv(const cplx_t<R>* S1, int pitch, int Px, Twiddles& tw, const Geom& g, R scale, const R* m,
             const MsInfo& ms, const TermList& tl, const EpilogueArgs& ep, const TuneChoice& tc, cudaStream_t st,
             int* nblocks);

// Batched compile-time passes: one launch runs the (item, tile) pairs of a
// device work table, every item of a launch with the same transform length
// (the ensembles' batched steps; the tile bodies are those of the per-state
// kernels, so an item's results equal its per-state pass bit for bit).
template <typename R> struct CtXfwdItem {
    const R* in;
    int n_in;
    int64_t rows;
    R ms;
    cplx_t<R>* out;
    int pitch;
};
template <typename R> struct CtConvyItem {
    cplx_t<R>* S;
    const R* Nred;
    int nxh, pitch;
};
template <typename R> struct CtXinvItem {
    const cplx_t<R>* S1;
    int pitch;
    Geom g;
    R scale;
    const R* m;
    MsInfo ms;
    TermList tl;
    EpilogueArgs ep;  // EPI_LLG
    int run4;
};
// pass: 0 x forward (L = Px / 2), 1 y convolution (L = Py), 2 x inverse (L = Px / 2).
// Rows (x passes) or kx columns (y convolution) per tile; 0: no compile-time kernel.
template <typename R> int ct_batch_tile(int pass, int L);
// The twiddle table the pass's kernel of length L reads (created on first use).
template <typename R> const void* ct_batch_twiddles(int pass, int L, Twiddles& tw);
// The run-epilogue flag and constants of an x-inverse item (as the per-state launch prepares them).
template <typename R> void ct_batch_xinv_prepare(CtXinvItem<R>& it);
// Launches; tw from ct_batch_twiddles, twP the length-Px table (Twiddles::get).
template <typename R>
void ct_batch_xfwd(const CtXfwdItem<R>* items, const int2* work, int nwork, int L, const void* tw, const void* twP,
                   cudaStream_t st);
template <typename R>
void ct_batch_convy(const CtConvyItem<R>* items, const int2* work, int nwork, int L, const void* tw, cudaStream_t st);
template <typename R>
void ct_batch_xinv(const CtXinvItem<R>* items, const int2* work, int nwork, int L, int run, const void* tw,
                   const void* twP, cudaStream_t st);

}  // namespace mafb
