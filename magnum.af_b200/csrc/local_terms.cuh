// Per-cell evaluation of the local field terms, fused into the epilogue of the
// last demag pass (or run standalone when no demag term is present).
//
// Reference semantics (paths relative to the magnum.af project root):
//  exchange      magnumaf/src/field_terms/micro/exchange_field.cpp:115-134
//                7-point Laplacian with the -2/dx^2-2/dy^2-2/dz^2 self term,
//                neighbours outside the mesh are zero; Ms_field==0 -> 0.
//  interface DMI magnumaf/src/field_terms/micro/dmi_field.cpp:41-110
//                2D/(mu0 Ms) [n div m - grad(n.m)], zero-padded central
//                differences, no DMI boundary condition.
//  bulk DMI+ex   magnumaf/src/field_terms/micro/bulk_dmi_exchange_field.cpp:11-119
//                ghost cells m_in +/- (d D/A) (n x m) on the six faces, then
//                (2D curl m - 2A lap m)/(-mu0 Ms).
//  uniaxial      magnumaf/src/field_terms/micro/uniaxial_anisotropy_field.cpp:58-89
//  cubic         magnumaf/src/field_terms/micro/cubic_anisotropy_field.cpp:61-96
//  Zeeman        magnumaf/src/field_terms/micro/external_field.cpp:28-37
#pragma once
#include "common.cuh"

namespace mafb {

enum TermKind : int {
    TK_DEMAG = 0,
    TK_EXCHANGE = 1,
    TK_DMI = 2,
    TK_BULKDMI = 3,
    TK_UNIAXIAL = 4,
    TK_CUBIC = 5,
    TK_ZEEMAN = 6,
    TK_STT = 7,
    TK_SPARSE_EXCH = 8,
};

constexpr int kMaxTerms = 8;

struct TermDesc {
    int kind = TK_DEMAG;
    double p[12] = {};          // kind-specific parameters (see make_* in field.cu)
    double q[4] = {};           // per-launch constants of the fast run epilogue (prepare_run4)
    float qf[16] = {};          // the run epilogue's constants rounded to FP32 once on the host (prepare_run4)
    const double* f0 = nullptr;  // optional per-cell scalar field (Ku1, D) or vector field (Zeeman) [3][N]
    const double* f1 = nullptr;  // optional per-cell axis field [3][N]
};

struct TermList {
    int n = 0;
    TermDesc t[kMaxTerms];
};

struct Geom {
    int nx, ny, nz;
    int64_t N;
    double dx, dy, dz;
};

// Read component c of m at (x, y, z), zero outside the mesh.
template <typename R>
__device__ __forceinline__ R mget(const R* __restrict__ m, const Geom& g, int c, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) return (R)0;
    return m[c * g.N + ((int64_t)z * g.ny + y) * g.nx + x];
}

// 3-vector of m at a cell that is known to be inside.
template <typename R>
__device__ __forceinline__ void mvec(const R* __restrict__ m, const Geom& g, int64_t cell, R v[3]) {
    v[0] = m[cell];
    v[1] = m[g.N + cell];
    v[2] = m[2 * g.N + cell];
}

// Neighbour of the bulk-DMI ghost-cell array along `axis` (0,1,2) in direction
// `dir` (-1, +1); ghost values follow bulk_dmi_exchange_field.cpp:27-81.
template <typename R>
__device__ __forceinline__ void bulk_neighbour(const R* __restrict__ m, const Geom& g, int x, int y, int z, int axis,
                                               int dir, R coef, R out[3]) {
    int p[3] = {x, y, z};
    int n[3] = {g.nx, g.ny, g.nz};
    p[axis] += dir;
    if (p[axis] >= 0 && p[axis] < n[axis]) {
        const int64_t c = ((int64_t)p[2] * g.ny + p[1]) * g.nx + p[0];
        mvec(m, g, c, out);
        return;
    }
    // ghost: boundary cell i (the current cell) and one cell inward io
    int q[3] = {x, y, z};
    q[axis] -= dir;  // one cell inward from the boundary cell
    const int64_t ci = ((int64_t)z * g.ny + y) * g.nx + x;
    const int64_t co = ((int64_t)q[2] * g.ny + q[1]) * g.nx + q[0];
    R mi[3], mo[3];
    mvec(m, g, ci, mi);
    mvec(m, g, co, mo);
    const R sign = dir > 0 ? (R)1 : (R)-1;
    if (axis == 0) {
        out[0] = mo[0];
        out[1] = mo[1] + coef * (sign * (R)-1 * mi[2]);
        out[2] = mo[2] + coef * (sign * mi[1]);
    } else if (axis == 1) {
        out[0] = mo[0] + coef * (sign * mi[2]);
        out[1] = mo[1];
        out[2] = mo[2] + coef * (sign * (R)-1 * mi[0]);
    } else {
        out[0] = mo[0] + coef * (sign * (R)-1 * mi[1]);
        out[1] = mo[1] + coef * (sign * mi[0]);
        out[2] = mo[2];
    }
}

// Exchange Laplacian of one cell, added as coef * lap to h.  neumann = false:
// neighbours outside the mesh are zero (exchange_field.cpp:115-126);
// neumann = true: they are absent, i.e. the h_withedges field of the exchange
// energy (exchange_field.cpp:28-51, which adds m/d^2 back on each boundary face).
template <typename R>
__device__ __forceinline__ void h_exchange_add(const R* __restrict__ m, const Geom& g, int x, int y, int z,
                                               const R mc[3], R coef, R idx2, R idy2, R idz2, bool neumann, R h[3]) {
    const int64_t cell = ((int64_t)z * g.ny + y) * g.nx + x;
    const bool xm = x > 0, xp = x < g.nx - 1, ym = y > 0, yp = y < g.ny - 1, zm = z > 0, zp = z < g.nz - 1;
    const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const R* mcmp = m + c * g.N + cell;
        const R v = mc[c];
        const R ab = neumann ? (R)0 : -v;  // contribution of a neighbour outside the mesh
        const R ax = (xm ? mcmp[-1] - v : ab) + (xp ? mcmp[1] - v : ab);
        const R ay = (ym ? mcmp[-sy] - v : ab) + (yp ? mcmp[sy] - v : ab);
        const R az = (zm ? mcmp[-sz] - v : ab) + (zp ? mcmp[sz] - v : ab);
        h[c] += coef * (ax * idx2 + ay * idy2 + az * idz2);
    }
}

// Cubic anisotropy h1, h2, h3 (cubic_anisotropy_field.cpp:61-91) for one cell.
template <typename R>
__device__ __forceinline__ void cubic_h123(const TermDesc& t, const R mc[3], R Ms, R h1[3], R h2[3], R h3[3]) {
    const R c1[3] = {(R)t.p[3], (R)t.p[4], (R)t.p[5]};
    const R c2[3] = {(R)t.p[6], (R)t.p[7], (R)t.p[8]};
    const R c3[3] = {(R)t.p[9], (R)t.p[10], (R)t.p[11]};
    const R c1m = c1[0] * mc[0] + c1[1] * mc[1] + c1[2] * mc[2];
    const R c2m = c2[0] * mc[0] + c2[1] * mc[1] + c2[2] * mc[2];
    const R c3m = c3[0] * mc[0] + c3[1] * mc[1] + c3[2] * mc[2];
    const R c1m2 = c1m * c1m, c2m2 = c2m * c2m, c3m2 = c3m * c3m;
    const R c1m3 = c1m2 * c1m, c2m3 = c2m2 * c2m, c3m3 = c3m2 * c3m;
    const R c1m4 = c1m2 * c1m2, c2m4 = c2m2 * c2m2, c3m4 = c3m2 * c3m2;
    const R pre2 = (R)-2 / ((R)kMu0 * Ms);
    const R pre4 = (R)-4 / ((R)kMu0 * Ms);
    const R K1 = (R)t.p[0], K2 = (R)t.p[1], K3 = (R)t.p[2];
    const R a1 = (c2m2 + c3m2) * c1m, a2 = (c1m2 + c3m2) * c2m, a3 = (c1m2 + c2m2) * c3m;
    const R b1 = c2m2 * c3m2 * c1m, b2 = c1m2 * c3m2 * c2m, b3 = c1m2 * c2m2 * c3m;
    const R d1 = (c2m4 + c3m4) * c1m3, d2 = (c1m4 + c3m4) * c2m3, d3 = (c1m4 + c2m4) * c3m3;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        h1[i] = pre2 * K1 * (a1 * c1[i] + a2 * c2[i] + a3 * c3[i]);
        h2[i] = pre2 * K2 * (b1 * c1[i] + b2 * c2[i] + b3 * c3[i]);
        h3[i] = pre4 * K3 * (d1 * c1[i] + d2 * c2[i] + d3 * c3[i]);
    }
}

template <typename R>
__device__ __forceinline__ void cubic_h123_sum(const TermDesc& t, const R mc[3], R Ms, R h[3]) {
    R h1[3], h2[3], h3[3];
    cubic_h123(t, mc, Ms, h1, h2, h3);
#pragma unroll
    for (int i = 0; i < 3; ++i) h[i] = h1[i] + h2[i] + h3[i];
}

// SparseExchangeField / ExchangeFieldPBC for one cell: H = (M m)_cell / Ms with
// the 7-point matrix M those terms assemble (sparse_exchange_field.cpp:8-18,
// exchange_field_pbc.cpp:9-19).  p[0] = scalar A, p[1] != 0 for periodic
// neighbours, f0 = optional A field [N].
//   scalar A, open boundary: each neighbour inside the mesh weighs 2A/mu0/d^2
//     and the row has no diagonal (sparse_exchange_field.cpp:25-101);
//   A field or periodic: neighbour weight lapA = 2A_i/(mu0 d^2) * 2A_nb/(A_nb + A_i)
//     (sparse_exchange_field.cpp:183-185), diagonal = minus their sum, rows of
//     cells with A_i = 0 empty (:189-270; periodic wrap exchange_field_pbc.cpp:60-80).
// A row with a diagonal is evaluated as sum_nb w (m_nb - m_c): the same value,
// exactly zero for a uniform m.  The weights are formed in FP64 as assembled.
template <typename R>
__device__ __forceinline__ void sparse_exchange_add(const TermDesc& t, const R* __restrict__ m, const Geom& g, int x,
                                                    int y, int z, int64_t cell, const R mc[3], R Ms, R h[3]) {
    const bool periodic = t.p[1] != 0.0;
    const bool diag = periodic || t.f0 != nullptr;
    const double Ai = t.f0 ? t.f0[cell] : t.p[0];
    if (diag && Ai == 0.0) return;
    R acc[3] = {0, 0, 0};
    auto nb = [&](int xx, int yy, int zz, double d) {
        const int64_t j = ((int64_t)zz * g.ny + yy) * g.nx + xx;
        double w;
        if (diag) {
            const double Aj = t.f0 ? t.f0[j] : t.p[0];
            w = 2.0 * Ai / (kMu0 * (d * d)) * 2.0 * Aj / (Aj + Ai);
        } else {
            w = 2.0 * Ai / kMu0 / (d * d);
        }
        const R wr = (R)w;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const R v = m[c * g.N + j];
            acc[c] += diag ? wr * (v - mc[c]) : wr * v;
        }
    };
    if (periodic) {
        nb(x + 1 == g.nx ? 0 : x + 1, y, z, g.dx);
        nb(x == 0 ? g.nx - 1 : x - 1, y, z, g.dx);
        nb(x, y + 1 == g.ny ? 0 : y + 1, z, g.dy);
        nb(x, y == 0 ? g.ny - 1 : y - 1, z, g.dy);
        nb(x, y, z + 1 == g.nz ? 0 : z + 1, g.dz);
        nb(x, y, z == 0 ? g.nz - 1 : z - 1, g.dz);
    } else {
        if (x < g.nx - 1) nb(x + 1, y, z, g.dx);
        if (x > 0) nb(x - 1, y, z, g.dx);
        if (y < g.ny - 1) nb(x, y + 1, z, g.dy);
        if (y > 0) nb(x, y - 1, z, g.dy);
        if (z < g.nz - 1) nb(x, y, z + 1, g.dz);
        if (z > 0) nb(x, y, z - 1, g.dz);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) h[c] += acc[c] / Ms;
}

// Adds the field of local term `t` at cell (x,y,z) to h.  Ms is the cell's
// saturation magnetisation (the scalar Ms or Ms_field[cell]).
template <typename R>
__device__ __forceinline__ void add_local_term(const TermDesc& t, const R* __restrict__ m, const Geom& g, int x, int y,
                                               int z, int64_t cell, const R mc[3], R Ms, bool ms_is_field, R h[3]) {
    switch (t.kind) {
        case TK_EXCHANGE: {
            // p[0]=A.  The reference filter (centre -2/dx^2-2/dy^2-2/dz^2, neighbours
            // 1/d^2, zero outside) is evaluated as sum over the six neighbours of
            // (m_nb - m_c)/d^2, with m_nb = 0 outside the mesh: the same value,
            // without cancelling the ~1e7 A/m self term against the neighbour sum
            // (which would cost the FP32-field form five digits).
            if (ms_is_field && Ms == (R)0) return;
            const R idx2 = (R)(1.0 / (g.dx * g.dx)), idy2 = (R)(1.0 / (g.dy * g.dy)), idz2 = (R)(1.0 / (g.dz * g.dz));
            const R coef = (R)(2.0 * t.p[0]) / ((R)kMu0 * Ms);
            h_exchange_add(m, g, x, y, z, mc, coef, idx2, idy2, idz2, false, h);
            break;
        }
        case TK_DMI: {
            // p[0]=D, p[1..3]=unit axis n; f0: optional D field [N]
            if (ms_is_field && Ms == (R)0) return;
            const R n0 = (R)t.p[1], n1 = (R)t.p[2], n2 = (R)t.p[3];
            const R hx = (R)(0.5 / g.dx), hy = (R)(0.5 / g.dy), hz = (R)(0.5 / g.dz);
            const R div = (mget(m, g, 0, x + 1, y, z) - mget(m, g, 0, x - 1, y, z)) * hx +
                          (mget(m, g, 1, x, y + 1, z) - mget(m, g, 1, x, y - 1, z)) * hy +
                          (mget(m, g, 2, x, y, z + 1) - mget(m, g, 2, x, y, z - 1)) * hz;
            auto nm = [&](int xx, int yy, int zz) -> R {
                return n0 * mget(m, g, 0, xx, yy, zz) + n1 * mget(m, g, 1, xx, yy, zz) +
                       n2 * mget(m, g, 2, xx, yy, zz);
            };
            const R g0 = (nm(x + 1, y, z) - nm(x - 1, y, z)) * hx;
            const R g1 = (nm(x, y + 1, z) - nm(x, y - 1, z)) * hy;
            const R g2 = (nm(x, y, z + 1) - nm(x, y, z - 1)) * hz;
            const R D = t.f0 ? (R)t.f0[cell] : (R)t.p[0];
            const R coef = (R)2 * D / ((R)kMu0 * Ms);
            h[0] += coef * (n0 * div - g0);
            h[1] += coef * (n1 * div - g1);
            h[2] += coef * (n2 * div - g2);
            break;
        }
        case TK_BULKDMI: {
            // p[0]=D, p[1]=A
            const R D = (R)t.p[0], A = (R)t.p[1];
            const R cx = (R)(2.0 * g.dx * t.p[0] / (2.0 * t.p[1]));
            const R cy = (R)(2.0 * g.dy * t.p[0] / (2.0 * t.p[1]));
            const R cz = (R)(2.0 * g.dz * t.p[0] / (2.0 * t.p[1]));
            R xm[3], xp[3], ym[3], yp[3], zm[3], zp[3];
            bulk_neighbour(m, g, x, y, z, 0, -1, cx, xm);
            bulk_neighbour(m, g, x, y, z, 0, +1, cx, xp);
            bulk_neighbour(m, g, x, y, z, 1, -1, cy, ym);
            bulk_neighbour(m, g, x, y, z, 1, +1, cy, yp);
            bulk_neighbour(m, g, x, y, z, 2, -1, cz, zm);
            bulk_neighbour(m, g, x, y, z, 2, +1, cz, zp);
            const R hx = (R)(0.5 / g.dx), hy = (R)(0.5 / g.dy), hz = (R)(0.5 / g.dz);
            const R curl0 = (yp[2] - ym[2]) * hy - (zp[1] - zm[1]) * hz;
            const R curl1 = (zp[0] - zm[0]) * hz - (xp[2] - xm[2]) * hx;
            const R curl2 = (xp[1] - xm[1]) * hx - (yp[0] - ym[0]) * hy;
            const R idx2 = (R)(1.0 / (g.dx * g.dx)), idy2 = (R)(1.0 / (g.dy * g.dy)), idz2 = (R)(1.0 / (g.dz * g.dz));
            const R curl[3] = {curl0, curl1, curl2};
            const R den = (R)-kMu0 * Ms;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                // laplace_3D (math.cpp:107-122) as a sum of neighbour differences
                const R lap = ((xm[c] - mc[c]) + (xp[c] - mc[c])) * idx2 + ((ym[c] - mc[c]) + (yp[c] - mc[c])) * idy2 +
                              ((zm[c] - mc[c]) + (zp[c] - mc[c])) * idz2;
                h[c] += ((R)2 * D * curl[c] + (R)-2 * A * lap) / den;
            }
            break;
        }
        case TK_UNIAXIAL: {
            // p[0]=Ku1, p[1..3]=unit axis; f0: optional Ku1 field [N]; f1: optional axis field [3][N]
            if (ms_is_field && Ms == (R)0) return;
            R e0, e1, e2;
            if (t.f1) {
                e0 = (R)t.f1[cell];
                e1 = (R)t.f1[g.N + cell];
                e2 = (R)t.f1[2 * g.N + cell];
            } else {
                e0 = (R)t.p[1];
                e1 = (R)t.p[2];
                e2 = (R)t.p[3];
            }
            const R Ku = t.f0 ? (R)t.f0[cell] : (R)t.p[0];
            const R em = e0 * mc[0] + e1 * mc[1] + e2 * mc[2];
            const R coef = (R)2 * Ku / ((R)kMu0 * Ms);
            h[0] += coef * (e0 * em);
            h[1] += coef * (e1 * em);
            h[2] += coef * (e2 * em);
            break;
        }
        case TK_CUBIC: {
            // p[0..2]=Kc1..3, p[3..5]=c1, p[6..8]=c2, p[9..11]=c3
            R hc[3];
            cubic_h123_sum(t, mc, Ms, hc);
            h[0] += hc[0];
            h[1] += hc[1];
            h[2] += hc[2];
            break;
        }
        case TK_STT: {
            // spin-transfer (spin-orbit) torque field (spin_transfer_torque_field.cpp:17-28):
            // p[0] = -j_e hbar / (2 e mu0 d), p[1] = eta_damping, p[2] = eta_field,
            // f1 = unit polarisation [3][N]; H = p[0]/Ms (eta_d m x p + eta_f p), 0 where Ms = 0
            if (ms_is_field && Ms == (R)0) return;
            const R p0 = (R)t.f1[cell], p1 = (R)t.f1[g.N + cell], p2 = (R)t.f1[2 * g.N + cell];
            const R coef = (R)t.p[0] / Ms, ed = (R)t.p[1], ef = (R)t.p[2];
            h[0] += coef * (ed * (mc[1] * p2 - mc[2] * p1) + ef * p0);
            h[1] += coef * (ed * (mc[2] * p0 - mc[0] * p2) + ef * p1);
            h[2] += coef * (ed * (mc[0] * p1 - mc[1] * p0) + ef * p2);
            break;
        }
        case TK_SPARSE_EXCH: {
            // zero where Ms = 0 (the af::replace of sparse_exchange_field.cpp:15)
            if (ms_is_field && Ms == (R)0) return;
            sparse_exchange_add(t, m, g, x, y, z, cell, mc, Ms, h);
            break;
        }
        case TK_ZEEMAN: {
            // p[0..2]=uniform field; f0: optional field [3][N]
            if (t.f0) {
                h[0] += (R)t.f0[cell];
                h[1] += (R)t.f0[g.N + cell];
                h[2] += (R)t.f0[2 * g.N + cell];
            } else {
                h[0] += (R)t.p[0];
                h[1] += (R)t.p[1];
                h[2] += (R)t.p[2];
            }
            break;
        }
        default: break;
    }
}

}  // namespace mafb
