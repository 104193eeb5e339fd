// Per-cell epilogue shared by every kernel that ends a field evaluation: sum of
// the terms in list order (demag value supplied by the caller), then write H,
// or dt * LLG right-hand side in FP64, or accumulate the energy density.
#pragma once
#include "engine.hpp"
#include "rng.cuh"

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
    if constexpr (EPI == EPI_EDENS || EPI == EPI_EGRAD) {
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
    }
    if constexpr (EPI != EPI_EDENS) {
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
        } else if constexpr (EPI == EPI_EGRAD) {
            // LBFGS gradient m x (m x Heff) (lbfgs_minimizer.cpp:33-36), FP64
            const double* m64 = ep.llg.m64;
            const double M0 = m64[cell], M1 = m64[g.N + cell], M2 = m64[2 * g.N + cell];
            const double H0 = h[0], H1 = h[1], H2 = h[2];
            const double x0 = M1 * H2 - M2 * H1;
            const double x1 = M2 * H0 - M0 * H2;
            const double x2 = M0 * H1 - M1 * H0;
            double* o = static_cast<double*>(ep.out);
            o[cell] = M1 * x2 - M2 * x1;
            o[g.N + cell] = M2 * x0 - M0 * x2;
            o[2 * g.N + cell] = M0 * x1 - M1 * x0;
        } else {
            const double* m64 = ep.llg.m64;
            const double M0 = m64[cell], M1 = m64[g.N + cell], M2 = m64[2 * g.N + cell];
            double H0 = h[0], H1 = h[1], H2 = h[2];
            if (ep.llg.sigma != 0.0) {
                // Heff + h_th (stochastic_llg.cpp:19-22), h_th = sqrt(2D/dt) N(0,1)
                double xi[3];
                normal3(ep.llg.seed, ep.llg.member, ep.llg.stream_index(), (uint64_t)cell, xi);
                H0 += ep.llg.sigma * xi[0];
                H1 += ep.llg.sigma * xi[1];
                H2 += ep.llg.sigma * xi[2];
            }
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

// ---------------------------------------------------------------------------
// Fast epilogue for a run of N = 2 or 4 consecutive cells along x (x0 % N == 0): all
// m values the stencils need (the run, its two x neighbours, and the runs at
// y-1, y+1, z-1, z+1) are fetched first with vector loads, then the terms are
// evaluated.  Valid when the term list holds only demag, exchange, interface
// DMI, uniaxial and cubic anisotropy with scalar parameters and a uniform
// Zeeman field, the state has no Ms_field and nx % 4 == 0 (run4_eligible on the host).
// Same arithmetic per cell as add_local_term / epilogue_cell.
// ---------------------------------------------------------------------------
template <typename R, int N> struct RunN {
    R c[3][N];            // the run
    R xl[3], xr[3];       // x neighbours of the first and the last cell
    R ym[3][N], yp[3][N], zm[3][N], zp[3][N];
    bool hxl, hxr, hym, hyp, hzm, hzp;
};

template <typename R, int N> __device__ __forceinline__ void loadN(const R* __restrict__ p, R out[N]) {
    if constexpr (sizeof(R) == 4 && N == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
    } else if constexpr (sizeof(R) == 4) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        out[0] = v.x; out[1] = v.y;
    } else {
#pragma unroll
        for (int h = 0; h < N / 2; ++h) {
            const double2 a = reinterpret_cast<const double2*>(p)[h];
            out[2 * h] = a.x; out[2 * h + 1] = a.y;
        }
    }
}

template <typename R, int N> __device__ __forceinline__ void storeN(R* p, const R v[N]) {
    if constexpr (sizeof(R) == 4 && N == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (sizeof(R) == 4) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    } else {
#pragma unroll
        for (int h = 0; h < N / 2; ++h) reinterpret_cast<double2*>(p)[h] = make_double2(v[2 * h], v[2 * h + 1]);
    }
}

template <typename R, int N>
__device__ __forceinline__ void runN_load(const R* __restrict__ m, const Geom& g, int x0, int y, int z, int64_t cell0,
                                          RunN<R, N>& r) {
    const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
    r.hxl = x0 > 0;
    r.hxr = x0 + N < g.nx;
    r.hym = y > 0;
    r.hyp = y < g.ny - 1;
    r.hzm = z > 0;
    r.hzp = z < g.nz - 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R* p = m + c * g.N + cell0;
        loadN<R, N>(p, r.c[c]);
        r.xl[c] = r.hxl ? p[-1] : (R)0;
        r.xr[c] = r.hxr ? p[N] : (R)0;
#pragma unroll
        for (int i = 0; i < N; ++i) { r.ym[c][i] = 0; r.yp[c][i] = 0; r.zm[c][i] = 0; r.zp[c][i] = 0; }
        if (r.hym) loadN<R, N>(p - sy, r.ym[c]);
        if (r.hyp) loadN<R, N>(p + sy, r.yp[c]);
        if (r.hzm) loadN<R, N>(p - sz, r.zm[c]);
        if (r.hzp) loadN<R, N>(p + sz, r.zp[c]);
    }
}

// H of the N cells of the run (hd = demag contribution).  Terms outer,
// cells inner; the per-term constants come from TermDesc::q, prepared once per
// launch on the host (prepare_run4), so no division is left in the cell loop:
//   exchange  q = 2A/(mu0 Ms) / (dx^2, dy^2, dz^2)
//   DMI       q = 2D/(mu0 Ms), 1/(2dx), 1/(2dy), 1/(2dz)
//   uniaxial  q = 2Ku/(mu0 Ms)
//   cubic     q = -2Kc1/(mu0 Ms), -2Kc2/(mu0 Ms), -4Kc3/(mu0 Ms)
template <typename R, int N>
__device__ __forceinline__ void runN_fields(const TermList& tl, const RunN<R, N>& r, const R hd[N][3], R h[N][3]) {
    // FP32: the constants come pre-rounded (TermDesc::qf), the same values as a device-side rounding
    constexpr bool kF32 = sizeof(R) == 4;
#pragma unroll
    for (int i = 0; i < N; ++i) h[i][0] = h[i][1] = h[i][2] = 0;
    for (int it = 0; it < tl.n; ++it) {
        const TermDesc& t = tl.t[it];
        switch (t.kind) {
            case TK_DEMAG:
#pragma unroll
                for (int i = 0; i < N; ++i) { h[i][0] += hd[i][0]; h[i][1] += hd[i][1]; h[i][2] += hd[i][2]; }
                break;
            case TK_EXCHANGE: {
                const R qx = kF32 ? (R)t.qf[0] : (R)t.q[0], qy = kF32 ? (R)t.qf[1] : (R)t.q[1];
                const R qz = kF32 ? (R)t.qf[2] : (R)t.q[2];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        const R v = r.c[c][i];
                        const R left = i > 0 ? r.c[c][i - 1] - v : (r.hxl ? r.xl[c] - v : -v);
                        const R right = i < N - 1 ? r.c[c][i + 1] - v : (r.hxr ? r.xr[c] - v : -v);
                        const R ay = (r.hym ? r.ym[c][i] - v : -v) + (r.hyp ? r.yp[c][i] - v : -v);
                        const R az = (r.hzm ? r.zm[c][i] - v : -v) + (r.hzp ? r.zp[c][i] - v : -v);
                        h[i][c] += (left + right) * qx + ay * qy + az * qz;
                    }
                }
                break;
            }
            case TK_DMI: {
                const R coef = kF32 ? (R)t.qf[0] : (R)t.q[0], hx = kF32 ? (R)t.qf[1] : (R)t.q[1];
                const R hy = kF32 ? (R)t.qf[2] : (R)t.q[2], hz = kF32 ? (R)t.qf[3] : (R)t.q[3];
                const R n0 = kF32 ? (R)t.qf[4] : (R)t.p[1], n1 = kF32 ? (R)t.qf[5] : (R)t.p[2];
                const R n2 = kF32 ? (R)t.qf[6] : (R)t.p[3];
                auto nm = [&](const R v0, const R v1, const R v2) { return n0 * v0 + n1 * v1 + n2 * v2; };
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    R lm[3], rm[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        lm[c] = i > 0 ? r.c[c][i - 1] : r.xl[c];
                        rm[c] = i < N - 1 ? r.c[c][i + 1] : r.xr[c];
                    }
                    const R div = (rm[0] - lm[0]) * hx + (r.yp[1][i] - r.ym[1][i]) * hy + (r.zp[2][i] - r.zm[2][i]) * hz;
                    const R g0 = (nm(rm[0], rm[1], rm[2]) - nm(lm[0], lm[1], lm[2])) * hx;
                    const R g1 = (nm(r.yp[0][i], r.yp[1][i], r.yp[2][i]) - nm(r.ym[0][i], r.ym[1][i], r.ym[2][i])) * hy;
                    const R g2 = (nm(r.zp[0][i], r.zp[1][i], r.zp[2][i]) - nm(r.zm[0][i], r.zm[1][i], r.zm[2][i])) * hz;
                    h[i][0] += coef * (n0 * div - g0);
                    h[i][1] += coef * (n1 * div - g1);
                    h[i][2] += coef * (n2 * div - g2);
                }
                break;
            }
            case TK_UNIAXIAL: {
                const R e0 = kF32 ? (R)t.qf[1] : (R)t.p[1], e1 = kF32 ? (R)t.qf[2] : (R)t.p[2];
                const R e2 = kF32 ? (R)t.qf[3] : (R)t.p[3];
                const R coef = kF32 ? (R)t.qf[0] : (R)t.q[0];
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const R em = coef * (e0 * r.c[0][i] + e1 * r.c[1][i] + e2 * r.c[2][i]);
                    h[i][0] += e0 * em;
                    h[i][1] += e1 * em;
                    h[i][2] += e2 * em;
                }
                break;
            }
            case TK_CUBIC: {
                R c1[3], c2[3], c3[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    c1[c] = kF32 ? (R)t.qf[3 + c] : (R)t.p[3 + c];
                    c2[c] = kF32 ? (R)t.qf[6 + c] : (R)t.p[6 + c];
                    c3[c] = kF32 ? (R)t.qf[9 + c] : (R)t.p[9 + c];
                }
                const R k1 = kF32 ? (R)t.qf[0] : (R)t.q[0], k2 = kF32 ? (R)t.qf[1] : (R)t.q[1];
                const R k3 = kF32 ? (R)t.qf[2] : (R)t.q[2];
                if (t.qf[12] != 0.0f) {
                    // axes x, y, z and K2 = K3 = 0 (flag set on the host): the same values
                    // without the products by the axes' zeros and ones and the zero terms
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        const R m0 = r.c[0][i], m1 = r.c[1][i], m2 = r.c[2][i];
                        const R s1 = m0 * m0, s2 = m1 * m1, s3 = m2 * m2;
                        h[i][0] += k1 * (s2 + s3) * m0;
                        h[i][1] += k1 * (s1 + s3) * m1;
                        h[i][2] += k1 * (s1 + s2) * m2;
                    }
                    break;
                }
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const R m0 = r.c[0][i], m1 = r.c[1][i], m2 = r.c[2][i];
                    const R c1m = c1[0] * m0 + c1[1] * m1 + c1[2] * m2;
                    const R c2m = c2[0] * m0 + c2[1] * m1 + c2[2] * m2;
                    const R c3m = c3[0] * m0 + c3[1] * m1 + c3[2] * m2;
                    const R s1 = c1m * c1m, s2 = c2m * c2m, s3 = c3m * c3m;
                    // h1 + h2 + h3 of cubic_h123 with the prefactors folded in
                    const R w1 = k1 * (s2 + s3) * c1m + k2 * (s2 * s3) * c1m + k3 * (s2 * s2 + s3 * s3) * (s1 * c1m);
                    const R w2 = k1 * (s1 + s3) * c2m + k2 * (s1 * s3) * c2m + k3 * (s1 * s1 + s3 * s3) * (s2 * c2m);
                    const R w3 = k1 * (s1 + s2) * c3m + k2 * (s1 * s2) * c3m + k3 * (s1 * s1 + s2 * s2) * (s3 * c3m);
#pragma unroll
                    for (int c = 0; c < 3; ++c) h[i][c] += w1 * c1[c] + w2 * c2[c] + w3 * c3[c];
                }
                break;
            }
            case TK_ZEEMAN: {
                const R z0 = kF32 ? (R)t.qf[0] : (R)t.p[0], z1 = kF32 ? (R)t.qf[1] : (R)t.p[1];
                const R z2 = kF32 ? (R)t.qf[2] : (R)t.p[2];
#pragma unroll
                for (int i = 0; i < N; ++i) { h[i][0] += z0; h[i][1] += z1; h[i][2] += z2; }
                break;
            }
            default: break;
        }
    }
}

// Writes the epilogue output (H, dt*LLG or the LBFGS gradient) of the run.
template <typename R, int EPI, int N>
__device__ __forceinline__ void runN_epilogue(const TermList& tl, const Geom& g, const RunN<R, N>& r, int64_t cell0,
                                              const R hd[N][3], const EpilogueArgs& ep) {
    R h[N][3];
    runN_fields<R, N>(tl, r, hd, h);
    if constexpr (EPI == EPI_H) {
        R* o = static_cast<R*>(ep.out);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R v[N];
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = h[i][c];
            storeN<R, N>(o + c * g.N + cell0, v);
        }
    } else {
        const double* m64 = ep.llg.m64;
        double* o = static_cast<double*>(ep.out);
        double M[3][N], out[3][N];
#pragma unroll
        for (int c = 0; c < 3; ++c) loadN<double, N>(m64 + c * g.N + cell0, M[c]);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double H0 = h[i][0], H1 = h[i][1], H2 = h[i][2];
            if constexpr (EPI == EPI_LLG) {
                if (ep.llg.sigma != 0.0) {
                    double xi[3];
                    normal3(ep.llg.seed, ep.llg.member, ep.llg.stream_index(), (uint64_t)(cell0 + i), xi);
                    H0 += ep.llg.sigma * xi[0];
                    H1 += ep.llg.sigma * xi[1];
                    H2 += ep.llg.sigma * xi[2];
                }
            }
            const double M0 = M[0][i], M1 = M[1][i], M2 = M[2][i];
            const double x0 = M1 * H2 - M2 * H1;
            const double x1 = M2 * H0 - M0 * H2;
            const double x2 = M0 * H1 - M1 * H0;
            const double d0 = M1 * x2 - M2 * x1;
            const double d1 = M2 * x0 - M0 * x2;
            const double d2 = M0 * x1 - M1 * x0;
            if constexpr (EPI == EPI_EGRAD) {
                out[0][i] = d0; out[1][i] = d1; out[2][i] = d2;
            } else {
                double cp = ep.llg.c_prec, cd = ep.llg.c_damp;
                if (ep.llg.alpha) {
                    const double a = ep.llg.alpha[cell0 + i];
                    cp = -kGamma / (1. + a * a);
                    cd = -a * kGamma / (1. + a * a);
                }
                const double sc = ep.llg.scale;
                if (ep.llg.dissipation_only) {
                    out[0][i] = sc * (cd * d0); out[1][i] = sc * (cd * d1); out[2][i] = sc * (cd * d2);
                } else {
                    out[0][i] = sc * (cp * x0 + cd * d0);
                    out[1][i] = sc * (cp * x1 + cd * d1);
                    out[2][i] = sc * (cp * x2 + cd * d2);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) storeN<double, N>(o + c * g.N + cell0, out[c]);
    }
}

// ---------------------------------------------------------------------------
// Host side of the run epilogue: eligibility and per-launch term constants.
// ---------------------------------------------------------------------------
// The 4-cell epilogue (epilogue.cuh) needs nx % 4 == 0, 16-byte aligned m and
// output, a scalar Ms and only terms with scalar parameters.
template <typename R>
inline bool run4_eligible(const Geom& g, const R* m, const MsInfo& ms, const TermList& tl, const EpilogueArgs& ep) {
    if (g.nx % 4 != 0 || ms.field64) return false;
    if (ep.kind != EPI_H && ep.kind != EPI_LLG) return false;
    if (((uintptr_t)m | (uintptr_t)ep.out) % 16 != 0) return false;
    if (ep.kind == EPI_LLG && ((uintptr_t)ep.llg.m64 % 16 != 0)) return false;
    for (int i = 0; i < tl.n; ++i) {
        const TermDesc& t = tl.t[i];
        switch (t.kind) {
            case TK_DEMAG: case TK_EXCHANGE: case TK_CUBIC: break;
            case TK_DMI: case TK_UNIAXIAL: case TK_ZEEMAN:
                if (t.f0 || t.f1) return false;
                break;
            default: return false;
        }
    }
    return true;
}

// Per-launch constants of the 4-cell epilogue (TermDesc::q); the scalar Ms is
// known because run4 excludes an Ms_field.
inline void prepare_run4(TermList& tl, const Geom& g, double Ms) {
    const double mu0Ms = kMu0 * Ms;
    for (int i = 0; i < tl.n; ++i) {
        TermDesc& t = tl.t[i];
        switch (t.kind) {
            case TK_EXCHANGE: {
                const double c = 2.0 * t.p[0] / mu0Ms;
                t.q[0] = c / (g.dx * g.dx);
                t.q[1] = c / (g.dy * g.dy);
                t.q[2] = c / (g.dz * g.dz);
                break;
            }
            case TK_DMI:
                t.q[0] = 2.0 * t.p[0] / mu0Ms;
                t.q[1] = 0.5 / g.dx;
                t.q[2] = 0.5 / g.dy;
                t.q[3] = 0.5 / g.dz;
                break;
            case TK_UNIAXIAL: t.q[0] = 2.0 * t.p[0] / mu0Ms; break;
            case TK_CUBIC:
                t.q[0] = -2.0 * t.p[0] / mu0Ms;
                t.q[1] = -2.0 * t.p[1] / mu0Ms;
                t.q[2] = -4.0 * t.p[2] / mu0Ms;
                break;
            default: break;
        }
        // FP32 copies in the order runN_fields reads them
        auto f = [](double v) { return (float)v; };
        switch (t.kind) {
            case TK_EXCHANGE:
                for (int k = 0; k < 3; ++k) t.qf[k] = f(t.q[k]);
                break;
            case TK_DMI:
                for (int k = 0; k < 4; ++k) t.qf[k] = f(t.q[k]);
                for (int k = 0; k < 3; ++k) t.qf[4 + k] = f(t.p[1 + k]);
                break;
            case TK_UNIAXIAL:
                t.qf[0] = f(t.q[0]);
                for (int k = 0; k < 3; ++k) t.qf[1 + k] = f(t.p[1 + k]);
                break;
            case TK_CUBIC: {
                for (int k = 0; k < 3; ++k) t.qf[k] = f(t.q[k]);
                for (int k = 3; k < 12; ++k) t.qf[k] = f(t.p[k]);
                // axes exactly x, y, z and only K1: the epilogue's short form
                const double id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
                bool fast = t.p[1] == 0.0 && t.p[2] == 0.0;
                for (int k = 0; k < 9; ++k) fast = fast && t.p[3 + k] == id[k];
                t.qf[12] = fast ? 1.0f : 0.0f;
                break;
            }
            case TK_ZEEMAN:
                for (int k = 0; k < 3; ++k) t.qf[k] = f(t.p[k]);
                break;
            default: break;
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
