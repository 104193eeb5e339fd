// Newell demag tensor on the zero-padded grid, FP64.
//
// Follows magnumaf/src/field_terms/micro/demag_field.cpp:20-121 term for term:
// f() and g() keep the reference's expression order, Nxx/Nxy sum the 27
// stencil values in the reference's order, and the index wrap
// j = (i + P/2) % P - P/2 and the component mapping are the same.  This file
// is compiled with -fmad=false so that no multiply-add is contracted, which
// keeps the rounding of the (cancellation-prone) 27-point sums close to the
// reference's host build.  Only the elementary functions differ (CUDA's
// asinh/atan instead of the host libm), which perturbs far-field entries at
// the level of their own cancellation noise.
#include "engine.hpp"

namespace mafb {

__device__ double newell_f(double x, double y, double z) {
    x = fabs(x);
    y = fabs(y);
    z = fabs(z);
    const double R = sqrt(x * x + y * y + z * z);
    const double xx = x * x;
    const double yy = y * y;
    const double zz = z * z;
    double result = 1.0 / 6.0 * (2.0 * xx - yy - zz) * R;
    if (xx + zz > 0) result += y / 2.0 * (zz - xx) * asinh(y / (sqrt(xx + zz)));
    if (xx + yy > 0) result += z / 2.0 * (yy - xx) * asinh(z / (sqrt(xx + yy)));
    if (x * R > 0) result += -x * y * z * atan(y * z / (x * R));
    return result;
}

__device__ double newell_g(const double x, const double y, double z) {
    z = fabs(z);
    const double R = sqrt(x * x + y * y + z * z);
    const double xx = x * x;
    const double yy = y * y;
    const double zz = z * z;
    double result = -x * y * R / 3.0;
    if (xx + yy > 0) result += x * y * z * asinh(z / (sqrt(xx + yy)));
    if (yy + zz > 0) result += y / 6.0 * (3.0 * zz - yy) * asinh(x / (sqrt(yy + zz)));
    if (xx + zz > 0) result += x / 6.0 * (3.0 * zz - xx) * asinh(y / (sqrt(xx + zz)));
    if (z * R > 0) result += -(z * z * z) / 6.0 * atan(x * y / (z * R));
    if (y * R != 0) result += -z * yy / 2.0 * atan(x * z / (y * R));
    if (x * R != 0) result += -z * xx / 2.0 * atan(y * z / (x * R));
    return result;
}

template <bool IS_F>
__device__ double newell_27(int ix, int iy, int iz, double dx, double dy, double dz) {
    const double x = dx * ix;
    const double y = dy * iy;
    const double z = dz * iz;
    auto F = [](double a, double b, double c) { return IS_F ? newell_f(a, b, c) : newell_g(a, b, c); };
    double result = 8.0 * F(x, y, z) - 4.0 * F(x + dx, y, z) - 4.0 * F(x - dx, y, z) - 4.0 * F(x, y + dy, z) -
                    4.0 * F(x, y - dy, z) - 4.0 * F(x, y, z + dz) - 4.0 * F(x, y, z - dz) + 2.0 * F(x + dx, y + dy, z) +
                    2.0 * F(x + dx, y - dy, z) + 2.0 * F(x - dx, y + dy, z) + 2.0 * F(x - dx, y - dy, z) +
                    2.0 * F(x + dx, y, z + dz) + 2.0 * F(x + dx, y, z - dz) + 2.0 * F(x - dx, y, z + dz) +
                    2.0 * F(x - dx, y, z - dz) + 2.0 * F(x, y + dy, z + dz) + 2.0 * F(x, y + dy, z - dz) +
                    2.0 * F(x, y - dy, z + dz) + 2.0 * F(x, y - dy, z - dz) - 1.0 * F(x + dx, y + dy, z + dz) -
                    1.0 * F(x + dx, y + dy, z - dz) - 1.0 * F(x + dx, y - dy, z + dz) -
                    1.0 * F(x + dx, y - dy, z - dz) - 1.0 * F(x - dx, y + dy, z + dz) -
                    1.0 * F(x - dx, y + dy, z - dz) - 1.0 * F(x - dx, y - dy, z + dz) - 1.0 * F(x - dx, y - dy, z - dz);
    return -result / (4.0 * 3.14159265358979323846 * dx * dy * dz);
}

__device__ __forceinline__ double newell_comp(int comp, int j0, int j1, int j2, double dx, double dy, double dz) {
    switch (comp) {
        case 0: return newell_27<true>(j0, j1, j2, dx, dy, dz);    // xx
        case 1: return newell_27<false>(j0, j1, j2, dx, dy, dz);   // xy
        case 2: return newell_27<false>(j0, j2, j1, dx, dz, dy);   // xz
        case 3: return newell_27<true>(j1, j2, j0, dy, dz, dx);    // yy
        case 4: return newell_27<false>(j1, j2, j0, dy, dz, dx);   // yz
        default: return newell_27<true>(j2, j0, j1, dz, dx, dy);   // zz
    }
}

// sym == 0: the reference's setup_N value at every padded index.
// sym == 1: the parity-exact tensor that the spectral pipeline transforms: the
//   value at (|j0|,|j1|,|j2|) times the component's parity sign (xy odd in x,y;
//   xz odd in x,z; yz odd in y,z), and zero for an odd component where it
//   vanishes in exact arithmetic (j = 0 along an odd axis) and on its Nyquist
//   plane j = -P/2, which never reaches the truncated output.  The field on the
//   mesh is the reference's up to the rounding noise of its 27-point sums; the
//   exact symmetry makes the spectral tensor real with exact even/odd symmetry
//   in ky and kz (and Nxz = Nyz = 0 for a single layer).
__global__ void k_newell(double* __restrict__ out, int comp, int Px, int Py, int Pz, double dx, double dy, double dz,
                         int sym) {
    const int64_t total = (int64_t)Px * Py * Pz;
    const bool ox = comp == 1 || comp == 2, oy = comp == 1 || comp == 4, oz = comp == 2 || comp == 4;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % Px);
        const int i1 = (int)((idx / Px) % Py);
        const int i2 = (int)(idx / ((int64_t)Px * Py));
        const int j0 = (i0 + Px / 2) % Px - Px / 2;
        const int j1 = (i1 + Py / 2) % Py - Py / 2;
        const int j2 = (i2 + Pz / 2) % Pz - Pz / 2;
        double v;
        if (!sym) {
            v = newell_comp(comp, j0, j1, j2, dx, dy, dz);
        } else {
            // an odd function vanishes at j = 0 and, on the periodic grid, at j = -P/2
            const bool zero = (ox && (j0 == 0 || i0 == Px / 2)) || (oy && (j1 == 0 || i1 == Py / 2)) ||
                              (oz && (j2 == 0 || i2 == Pz / 2));
            if (zero) {
                v = 0.0;
            } else {
                v = newell_comp(comp, abs(j0), abs(j1), abs(j2), dx, dy, dz);
                const bool neg = (ox && j0 < 0) ^ (oy && j1 < 0) ^ (oz && j2 < 0);
                if (neg) v = -v;
            }
        }
        out[idx] = v;
    }
}

void newell_component(double* out, int comp, const MeshDims& md, int Px, int Py, int Pz, bool symmetric,
                      cudaStream_t st) {
    const int64_t total = (int64_t)Px * Py * Pz;
    const int threads = 128;
    const int64_t blocks = std::min<int64_t>(ceil_div(total, threads), (int64_t)sm_count() * 64);
    k_newell<<<(unsigned)blocks, threads, 0, st>>>(out, comp, Px, Py, Pz, md.dx, md.dy, md.dz, symmetric ? 1 : 0);
    MAF_LAUNCH_CHECK();
}

}  // namespace mafb
