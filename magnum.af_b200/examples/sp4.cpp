// muMAG standard problem 4 with the reference's C++ host API shape
// (magnumaf/examples/sp4.cpp), on the B200 library: relax for 1 ns with
// alpha = 1, then switch in (-24.6, 4.3, 0) mT with alpha = 0.02 until 2 ns.
// Prints the time integrals of <m> over both phases (the quantities checked by
// python/test/sp4.py:34-36,60-62) and writes "t <mx> <my> <mz>" rows to argv[1].
#include <cstdio>
#include <fstream>

#include "magnumaf_b200.hpp"

using namespace magnumaf;

int main(int argc, char** argv) {
    const double x = 5.e-7, y = 1.25e-7, z = 3.e-9;
    const int nx = 100, ny = 25, nz = 1;
    const double A = 1.3e-11;
    const double Ms = 8e5;

    Mesh mesh(nx, ny, nz, x / nx, y / ny, z / nz);

    // initial m: +x inside, +y on the two x faces ([3][nz][ny][nx], x fastest)
    HostArray m(3 * mesh.n(), 0.0);
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
            const size_t cell = (size_t)iy * nx + ix;
            if (ix == 0 || ix == nx - 1)
                m[mesh.n() + cell] = 1;
            else
                m[cell] = 1;
        }

    State state(mesh, Ms, m);
    DemagField dmag(mesh, true, true, 0);
    ExchangeField exch(A);
    LLGIntegrator llg(1.0, fieldterm::to_vec(std::move(dmag), std::move(exch)));

    std::ofstream stream(argc > 1 ? argv[1] : "m.dat");
    stream.precision(12);

    double ix = 0, iy = 0, iz = 0;
    while (state.t < 1e-9) {
        const double t1 = state.t;
        llg.step(state);
        const double dt = state.t - t1;
        const auto mm = state.mean_m();
        ix += mm[0] * dt;
        iy += mm[1] * dt;
        iz += mm[2] * dt;
        stream << state << '\n';
    }
    std::printf("relax %.12e %.12e %.12e\n", ix, iy, iz);

    HostArray external(3 * mesh.n(), 0.0);
    for (size_t i = 0; i < mesh.n(); ++i) {
        external[i] = -24.6e-3 / constants::mu0;
        external[mesh.n() + i] = +4.3e-3 / constants::mu0;
    }
    llg.llgterms.push_back(fieldterm::to_uptr<ExternalField>(mesh, external));
    llg.alpha = 0.02;

    ix = iy = iz = 0;
    while (state.t < 2e-9) {
        const double t1 = state.t;
        llg.step(state);
        const double dt = state.t - t1;
        const auto mm = state.mean_m();
        ix += mm[0] * dt;
        iy += mm[1] * dt;
        iz += mm[2] * dt;
        stream << state << '\n';
    }
    std::printf("switch %.12e %.12e %.12e\n", ix, iy, iz);
    return 0;
}
