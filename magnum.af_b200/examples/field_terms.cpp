// The further field terms through the C++ host API (reference constructors):
// DemagFieldPBC(), SparseExchangeField(A_field, mesh), ExchangeFieldPBC(A, mesh)
// and SpinTransferTorqueField(...), evaluated on a uniform and on a two-domain m.
// Prints "<name> <max |H| uniform> <max |H| two-domain> <energy two-domain>" per term.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "magnumaf_b200.hpp"

using namespace magnumaf;

static double max_abs(const HostArray& h) {
    double v = 0;
    for (double x : h) v = std::max(v, std::fabs(x));
    return v;
}

int main() {
    const int nx = 16, ny = 8, nz = 4;
    Mesh mesh(nx, ny, nz, 2e-9, 2e-9, 2e-9);
    HostArray uniform(3 * mesh.n(), 0.0), walls(3 * mesh.n(), 0.0);
    for (size_t c = 0; c < mesh.n(); ++c) {
        uniform[2 * mesh.n() + c] = 1.0;
        const int iz = (int)(c / ((size_t)nx * ny));
        walls[2 * mesh.n() + c] = iz < nz / 2 ? -1.0 : 1.0;
    }
    State s_uniform(mesh, 8e5, uniform);
    State s_walls(mesh, 8e5, walls);

    HostArray A_field(mesh.n(), 1.3e-11);
    HostArray pol(3 * mesh.n(), 0.0);
    for (size_t c = 0; c < mesh.n(); ++c) pol[c] = 1.0;  // polarisation along x

    DemagFieldPBC demag;
    SparseExchangeField sparse(A_field, mesh);
    ExchangeFieldPBC pbc(1.3e-11, mesh);
    SpinTransferTorqueField stt(mesh, pol, 0.3, 0.1, 2e10, 1e-9);

    const FieldTerm* terms[] = {&demag, &sparse, &pbc, &stt};
    const char* names[] = {"DemagFieldPBC", "SparseExchangeField", "ExchangeFieldPBC", "SpinTransferTorqueField"};
    for (int i = 0; i < 4; ++i)
        std::printf("%s %.17g %.17g %.17g\n", names[i], max_abs(terms[i]->H_in_Apm(s_uniform)),
                    max_abs(terms[i]->H_in_Apm(s_walls)), terms[i]->Energy_in_J(s_walls));
    return 0;
}
