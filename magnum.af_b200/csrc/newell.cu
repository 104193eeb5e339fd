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

__global__ void k_newell(double* __restrict__ out, int comp, int Px, int Py, int Pz, double dx, double dy, double dz) {
    const int64_t total = (int64_t)Px * Py * Pz;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % Px);
        const int i1 = (int)((idx / Px) % Py);
        const int i2 = (int)(idx / ((int64_t)Px * Py));
        const int j0 = (i0 + Px / 2) % Px - Px / 2;
        const int j1 = (i1 + Py / 2) % Py - Py / 2;
        const int j2 = (i2 + Pz / 2) % Pz - Pz / 2;
        double v = 0;
        switch (comp) {
            case 0: v = newell_27<true>(j0, j1, j2, dx, dy, dz); break;
            case 1: v = newell_27<false>(j0, j1, j2, dx, dy, dz); break;
            case 2: v = newell_27<false>(j0, j2, j1, dx, dz, dy); break;
            case 3: v = newell_27<true>(j1, j2, j0, dy, dz, dx); break;
            case 4: v = newell_27<false>(j1, j2, j0, dy, dz, dx); break;
            default: v = newell_27<true>(j2, j0, j1, dz, dx, dy); break;
        }
        out[idx] = v;
    }
}

void newell_component(double* out, int comp, const MeshDims& md, int Px, int Py, int Pz, cudaStream_t st) {
    const int64_t total = (int64_t)Px * Py * Pz;
    const int threads = 128;
    const int64_t blocks = std::min<int64_t>(ceil_div(total, threads), 148LL * 64);
    k_newell<<<(unsigned)blocks, threads, 0, st>>>(out, comp, Px, Py, Pz, md.dx, md.dy, md.dz);
    MAF_LAUNCH_CHECK();
}

}  // namespace mafb
