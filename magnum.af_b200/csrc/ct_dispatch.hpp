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

}  // namespace mafb
