// Tile bodies of the generic (run-time plan) demag passes, shared by the
// per-state kernels of fields.cu and the batched kernels of batch.cu, which
// map each CTA to a (member, tile) pair.  See fields.cu for the data layout.
#pragma once
#include "engine.hpp"
#include "epilogue.cuh"

namespace mafb {

// Launch shapes of the generic passes (host).
inline int round_threads(int t) {
    t = t > 32 ? t : 32;
    t = (t + 31) / 32 * 32;
    if (t > kMaxFftThreads) throw Error(6, "FFT tile needs more threads than one CTA has (transform length too large)");
    return t;
}

// columns per tile so that the tile holds about `target` complex values
inline int pick_nb(int L, int target, int ncols, int nbmax) {
    int nb = target / (L > 1 ? L : 1);
    nb = nb > 1 ? nb : 1;
    nb = nb < nbmax ? nb : nbmax;
    const int nc = ncols > 1 ? ncols : 1;
    return nb < nc ? nb : nc;
}

template <typename R> inline int tile_target() { return sizeof(R) == 4 ? 8192 : 4096; }

// x-forward: rows of n_in reals (times Ms) zero-padded to Px = 2*Lc, real FFT by
// packing even/odd samples into Lc complex values; writes kx in [0, Lc].
// Tile `tile` (rows [tile*nb, tile*nb + nb)) of the pass; the plan may sit in
// global memory (batched launches).
template <typename R>
__device__ __forceinline__ void xfwd_tile(const R* __restrict__ in, int n_in, int64_t rows, int64_t rows_pc,
                                          const R* __restrict__ msf, R ms, cplx_t<R>* __restrict__ out, int pitch,
                                          const FFTPlan& plan, const cplx_t<R>* __restrict__ twP, int nb, int64_t tile) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int Lc = plan.L;
    const SLay<false> lay{nb, spad_len(Lc)};
    const int64_t r0 = tile * nb;
    for (int idx = threadIdx.x; idx < nb * Lc; idx += blockDim.x) {
        const int b = idx / Lc;
        const int k = idx - b * Lc;
        const int64_t row = r0 + b;
        R a = 0, c = 0;
        if (row < rows) {
            const R* rp = in + row * n_in;
            const int x0 = 2 * k, x1 = 2 * k + 1;
            if (msf) {
                const R* mp = msf + (row % rows_pc) * n_in;
                if (x0 < n_in) a = mp[x0] * rp[x0];
                if (x1 < n_in) c = mp[x1] * rp[x1];
            } else {
                if (x0 < n_in) a = ms * rp[x0];
                if (x1 < n_in) c = ms * rp[x1];
            }
        }
        s[lay.at(k, b)] = mk(a, c);
    }
    __syncthreads();
    run_fft<R, -1, false>(s, lay, plan);
    const R half = (R)0.5;
    for (int idx = threadIdx.x; idx < nb * (Lc + 1); idx += blockDim.x) {
        const int b = idx / (Lc + 1);
        const int k = idx - b * (Lc + 1);
        const int64_t row = r0 + b;
        if (row >= rows) continue;
        const C Zk = s[lay.at(k == Lc ? 0 : k, b)];
        const C Zm = s[lay.at(k == 0 ? 0 : Lc - k, b)];
        const C E = cscale(cadd(Zk, cconj(Zm)), half);
        const C O = cscale(cmul_i<-1>(csub(Zk, cconj(Zm))), half);
        const C w = twP[k];  // W_Px^k, k <= Lc < Px
        out[row * pitch + k] = cadd(E, cmul(w, O));
    }
}

// Mesh lengths and spacings of the periodic Poisson operator.
struct PbcOp {
    int nx, ny, nz;
    double dx, dy, dz;
};

// DemagFieldPBC in k space (demag_field_pbc.cpp:44-68), for the three
// components M of the transform of Ms*m at (kx, ky, kz):
//   K_a = 2 pi k_a / n_a,  d_a = 1 - exp(-i K_a) = (1 - cos K_a) + i sin K_a
//   u = -(sum_a d_a M_a / h_a) / (sum_a 4/h_a^2 sin^2(K_a/2)),  u(0,0,0) = 0
//   H_a = (1 - exp(i K_a)) u / h_a = conj(d_a) u / h_a
// Evaluated in FP64 for either transform precision.
template <typename C>
__device__ __forceinline__ void pbc_poisson(const PbcOp& op, int kx, int ky, int kz, C& mx, C& my, C& mz) {
    const double K[3] = {2.0 * kPi * kx / op.nx, 2.0 * kPi * ky / op.ny, 2.0 * kPi * kz / op.nz};
    const double h[3] = {op.dx, op.dy, op.dz};
    double dre[3], dim[3], den = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double sn, cs;
        sincos(K[a], &sn, &cs);
        dre[a] = 1.0 - cs;
        dim[a] = sn;
        const double s2 = sin(K[a] / 2.0);
        den += 4.0 / (h[a] * h[a]) * (s2 * s2);
    }
    const double M[3][2] = {{(double)mx.x, (double)mx.y}, {(double)my.x, (double)my.y}, {(double)mz.x, (double)mz.y}};
    double divr = 0.0, divi = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        divr += (dre[a] * M[a][0] - dim[a] * M[a][1]) / h[a];
        divi += (dre[a] * M[a][1] + dim[a] * M[a][0]) / h[a];
    }
    double ur = 0.0, ui = 0.0;
    if (kx != 0 || ky != 0 || kz != 0) {
        ur = -divr / den;
        ui = -divi / den;
    }
    double H[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        H[a][0] = (dre[a] * ur + dim[a] * ui) / h[a];
        H[a][1] = (dre[a] * ui - dim[a] * ur) / h[a];
    }
    using R = decltype(mx.x);
    mx = mk((R)H[0][0], (R)H[0][1]);
    my = mk((R)H[1][0], (R)H[1][1]);
    mz = mk((R)H[2][0], (R)H[2][1]);
}

// Spectral convolution along the last transform axis (z for 3-D meshes, y for
// nz == 1), in place: forward FFT of the three components (zero pad fused),
// multiply by the symmetric tensor (or, PBC, apply the periodic Poisson
// operator), inverse FFT, keep the first n_in values.
// Tile (tile_x, other) of the pass: columns [tile_x*nb, tile_x*nb + nb) at
// other = ky for the z convolution.
template <typename R, bool PBC>
__device__ __forceinline__ void conv_tile(cplx_t<R>* S, const R* __restrict__ Nred, const FFTPlan& fplan,
                                          const FFTPlan& iplan, int n_in, int64_t si, int64_t comp_stride,
                                          int64_t other_stride, int ncols, int nb, int axis_is_z, int ny, int nz,
                                          int nxh, const PbcOp& pop, int tile_x, int other) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int L = fplan.L;
    const int nb3 = 3 * nb;
    const SLay<true> lay{nb3, 0};
    const int c0 = tile_x * nb;
    C* base = S + (int64_t)other * other_stride + c0;
    const int ncv = min(nb, ncols - c0);
    for (int idx = threadIdx.x; idx < L * nb3; idx += blockDim.x) {
        const int i = idx / nb3;
        const int cb = idx - i * nb3;
        const int comp = cb / nb;
        const int b = cb - comp * nb;
        C v = mk((R)0, (R)0);
        if (i < n_in && b < ncv) v = base[comp * comp_stride + i * si + b];
        s[lay.at(i, cb)] = v;
    }
    __syncthreads();
    run_fft<R, -1, true>(s, lay, fplan);
    // tensor multiply
    const int Py = 2 * ny;
    const int Pz = (nz == 1) ? 1 : 2 * nz;
    const int Kz = (nz == 1) ? 1 : nz + 1;
    const int64_t cs = (int64_t)Kz * (ny + 1) * nxh;  // component stride of Nred
    for (int idx = threadIdx.x; idx < L * nb; idx += blockDim.x) {
        const int kf = idx / nb;
        const int b = idx - kf * nb;
        if (b >= ncv) continue;
        const int kx = c0 + b;
        int ky, kz;
        if (axis_is_z) { ky = other; kz = kf; } else { ky = kf; kz = 0; }
        if constexpr (PBC) {
            C px = s[lay.at(kf, b)], py = s[lay.at(kf, nb + b)], pz = s[lay.at(kf, 2 * nb + b)];
            pbc_poisson(pop, kx, ky, kz, px, py, pz);
            s[lay.at(kf, b)] = px;
            s[lay.at(kf, nb + b)] = py;
            s[lay.at(kf, 2 * nb + b)] = pz;
            continue;
        }
        const int kyr = ky <= ny ? ky : Py - ky;
        const R sy = ky <= ny ? (R)1 : (R)-1;
        int kzr = 0;
        R sz = (R)1;
        if (nz > 1) { kzr = kz <= nz ? kz : Pz - kz; sz = kz <= nz ? (R)1 : (R)-1; }
        const int64_t o = ((int64_t)kzr * (ny + 1) + kyr) * nxh + kx;
        const C mx = s[lay.at(kf, b)];
        const C my = s[lay.at(kf, nb + b)];
        const C mz = s[lay.at(kf, 2 * nb + b)];
        R Nxx, Nxy, Nxz, Nyy, Nyz, Nzz;
        if (nz > 1) {
            Nxx = Nred[o];
            Nxy = sy * Nred[cs + o];
            Nxz = sz * Nred[2 * cs + o];
            Nyy = Nred[3 * cs + o];
            Nyz = sy * sz * Nred[4 * cs + o];
            Nzz = Nred[5 * cs + o];
        } else {
            Nxx = Nred[o];
            Nxy = sy * Nred[cs + o];
            Nxz = 0;
            Nyy = Nred[2 * cs + o];
            Nyz = 0;
            Nzz = Nred[3 * cs + o];
        }
        const C hx = cadd(cadd(cscale(mx, Nxx), cscale(my, Nxy)), cscale(mz, Nxz));
        const C hy = cadd(cadd(cscale(mx, Nxy), cscale(my, Nyy)), cscale(mz, Nyz));
        const C hz = cadd(cadd(cscale(mx, Nxz), cscale(my, Nyz)), cscale(mz, Nzz));
        s[lay.at(kf, b)] = hx;
        s[lay.at(kf, nb + b)] = hy;
        s[lay.at(kf, 2 * nb + b)] = hz;
    }
    __syncthreads();
    run_fft<R, 1, true>(s, lay, iplan);
    for (int idx = threadIdx.x; idx < n_in * nb3; idx += blockDim.x) {
        const int i = idx / nb3;
        const int cb = idx - i * nb3;
        const int comp = cb / nb;
        const int b = cb - comp * nb;
        if (b < ncv) base[comp * comp_stride + i * si + b] = s[lay.at(i, cb)];
    }
}

// x-inverse C2R of the half spectrum (3 components of nbr rows), scale, then
// the per-cell epilogue with the local terms.
// Tile `tile` (rows [tile*nbr, tile*nbr + nbr) of every component); the energy
// partial of the tile goes to ep.partials[part_index].
template <typename R, int EPI>
__device__ __forceinline__ void xinv_tile(const cplx_t<R>* __restrict__ S1, int pitch, const FFTPlan& plan,
                                          const cplx_t<R>* __restrict__ twP, const Geom& g, R scale,
                                          const R* __restrict__ m, const MsInfo& ms, const TermList& tl,
                                          const EpilogueArgs& ep, int nbr, int64_t tile, int part_index) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int Lc = plan.L;
    const int nb3 = 3 * nbr;
    const SLay<false> lay{nb3, spad_len(Lc)};
    const int64_t rows_pc = (int64_t)g.ny * g.nz;
    const int64_t ry0 = tile * nbr;
    for (int idx = threadIdx.x; idx < nb3 * Lc; idx += blockDim.x) {
        const int cb = idx / Lc;
        const int k = idx - cb * Lc;
        const int comp = cb / nbr;
        const int b = cb - comp * nbr;
        const int64_t ry = ry0 + b;
        C Z = mk((R)0, (R)0);
        if (ry < rows_pc) {
            const C* rp = S1 + (comp * rows_pc + ry) * pitch;
            const C Xk = rp[k];
            const C Xm = rp[Lc - k];
            const C E = cadd(Xk, cconj(Xm));
            const C O = cmulc(csub(Xk, cconj(Xm)), twP[k]);  // times W_Px^{-k}
            Z = cadd(E, cmul_i<1>(O));
        }
        s[lay.at(k, cb)] = Z;
    }
    __syncthreads();
    run_fft<R, 1, false>(s, lay, plan);
    double eacc = 0;
    for (int idx = threadIdx.x; idx < nbr * g.nx; idx += blockDim.x) {
        const int b = idx / g.nx;
        const int x = idx - b * g.nx;
        const int64_t ry = ry0 + b;
        if (ry >= rows_pc) continue;
        const int z = (int)(ry / g.ny);
        const int y = (int)(ry - (int64_t)z * g.ny);
        const int64_t cell = ry * g.nx + x;
        R hd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const C v = s[lay.at(x >> 1, c * nbr + b)];
            hd[c] = scale * ((x & 1) ? v.y : v.x);
        }
        epilogue_cell<R, EPI>(g, x, y, z, cell, m, ms, tl, ep, hd, eacc);
    }
    if constexpr (EPI == EPI_EDENS || EPI == EPI_EGRAD) block_sum_store(eacc, ep.partials + part_index);
}

}  // namespace mafb
