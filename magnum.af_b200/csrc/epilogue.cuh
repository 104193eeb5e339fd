// Per-cell epilogue shared by every kernel that ends a field evaluation: sum of
// the terms in list order (demag value supplied by the caller), then write H,
// or dt * LLG right-hand side in FP64, or accumulate the energy density.
#pragma once
#include "engine.hpp"

namespace mafb {

template <typename R>
__device__ __forceinline__ R cell_Ms(const MsInfo& ms, int64_t cell) {
    if (ms.field64) {
        if constexpr (sizeof(R) == 4) return ms.field32[cell];
        else return (R)ms.field64[cell];
    }
    return (R)ms.Ms;
}

template <typename R, int EPI>
__device__ __forceinline__ void epilogue_cell(const Geom& g, int x, int y, int z, int64_t cell,
                                              const R* __restrict__ m, const MsInfo& ms, const TermList& tl,
                                              const EpilogueArgs& ep, const R hd[3], double& eacc) {
    R mc[3];
    mvec(m, g, cell, mc);
    const bool msf = ms.field64 != nullptr;
    const R Ms = cell_Ms<R>(ms, cell);
    if constexpr (EPI == EPI_EDENS) {
        const double Msd = msf ? ms.field64[cell] : ms.Ms;
        for (int it = 0; it < tl.n; ++it) {
            const TermDesc& t = tl.t[it];
            R ht[3] = {0, 0, 0};
            double w = -kMu0 / 2.0;
            if (t.kind == TK_DEMAG) {
                ht[0] = hd[0]; ht[1] = hd[1]; ht[2] = hd[2];
            } else if (t.kind == TK_CUBIC) {
                R h1[3], h2[3], h3[3];
                cubic_h123(t, mc, Ms, h1, h2, h3);
                double e = 0;
                for (int c = 0; c < 3; ++c)
                    e += (-1.0 / 4.0 * (double)h1[c] - 1.0 / 6.0 * (double)h2[c] - 1.0 / 8.0 * (double)h3[c]) *
                         (double)mc[c];
                eacc += kMu0 * Msd * e;
                continue;
            } else if (t.kind == TK_EXCHANGE && ep.edge_exchange) {
                // h_withedges (exchange_field.cpp:28-60): the zero-padded stencil plus
                // m/d^2 on each boundary face, i.e. the Neumann Laplacian
                if (!(msf && Ms == (R)0)) {
                    const R coef = (R)(2.0 * t.p[0]) / ((R)kMu0 * Ms);
                    h_exchange_add(m, g, x, y, z, mc, coef, (R)(1.0 / (g.dx * g.dx)), (R)(1.0 / (g.dy * g.dy)),
                                   (R)(1.0 / (g.dz * g.dz)), true, ht);
                }
            } else {
                add_local_term(t, m, g, x, y, z, cell, mc, Ms, msf, ht);
                if (t.kind == TK_ZEEMAN) w = -kMu0;
            }
            const double hm = (double)ht[0] * (double)mc[0] + (double)ht[1] * (double)mc[1] + (double)ht[2] * (double)mc[2];
            eacc += w * Msd * hm;
        }
    } else {
        R h[3] = {0, 0, 0};
        for (int it = 0; it < tl.n; ++it) {
            const TermDesc& t = tl.t[it];
            if (t.kind == TK_DEMAG) {
                h[0] += hd[0]; h[1] += hd[1]; h[2] += hd[2];
            } else {
                add_local_term(t, m, g, x, y, z, cell, mc, Ms, msf, h);
            }
        }
        if constexpr (EPI == EPI_H) {
            R* o = static_cast<R*>(ep.out);
            o[cell] = h[0];
            o[g.N + cell] = h[1];
            o[2 * g.N + cell] = h[2];
        } else {
            const double* m64 = ep.llg.m64;
            const double M0 = m64[cell], M1 = m64[g.N + cell], M2 = m64[2 * g.N + cell];
            const double H0 = h[0], H1 = h[1], H2 = h[2];
            const double x0 = M1 * H2 - M2 * H1;
            const double x1 = M2 * H0 - M0 * H2;
            const double x2 = M0 * H1 - M1 * H0;
            const double d0 = M1 * x2 - M2 * x1;
            const double d1 = M2 * x0 - M0 * x2;
            const double d2 = M0 * x1 - M1 * x0;
            double cp = ep.llg.c_prec, cd = ep.llg.c_damp;
            if (ep.llg.alpha) {
                const double a = ep.llg.alpha[cell];
                cp = -kGamma / (1. + a * a);
                cd = -a * kGamma / (1. + a * a);
            }
            double k0, k1, k2;
            if (ep.llg.dissipation_only) {
                k0 = cd * d0; k1 = cd * d1; k2 = cd * d2;
            } else {
                k0 = cp * x0 + cd * d0; k1 = cp * x1 + cd * d1; k2 = cp * x2 + cd * d2;
            }
            double* o = static_cast<double*>(ep.out);
            const double sc = ep.llg.scale;
            o[cell] = sc * k0;
            o[g.N + cell] = sc * k1;
            o[2 * g.N + cell] = sc * k2;
        }
    }
}

__device__ __forceinline__ void block_sum_store(double v, double* partials) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) partials[blockIdx.x] = s;
    }
}

}  // namespace mafb
