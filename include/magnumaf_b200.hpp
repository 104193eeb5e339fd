// C++ host interface with magnum.af's class names over the B200 C ABI
// (include/maf_b200.h).  Reference-style host code
//
//     Mesh mesh(nx, ny, nz, dx, dy, dz);
//     State state(mesh, Ms, m);
//     LLGIntegrator llg(1.0, fieldterm::to_vec(DemagField(mesh), ExchangeField(A)));
//     while (state.t < 1e-9) llg.step(state);
//
// compiles against this header with ArrayFire arrays replaced by host vectors
// (magnumaf::HostArray, x fastest: [3][nz][ny][nx] for vector fields, the same
// bytes as the reference's column-major af::array [nx, ny, nz, 3]).
// Interfaces mirrored (paths relative to the magnum.af project root):
//   Mesh                 magnumaf/include/magnumaf/mesh.hpp:11-20
//   State                magnumaf/include/magnumaf/state.hpp:11-78
//   FieldTerm + terms    magnumaf/include/magnumaf/field_terms/field_term.hpp:12-51
//   Controller           magnumaf/include/magnumaf/integrators/controller.hpp:11-61
//   LLGIntegrator        magnumaf/include/magnumaf/integrators/llg_integrator.hpp:26-82
// Errors that the reference reports by exit() or exceptions raise
// std::runtime_error carrying the C ABI's message.
#pragma once
#include <array>
#include <cmath>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "maf_b200.h"

namespace magnumaf {

namespace constants {
constexpr double mu0 = 4e-7 * M_PI;
constexpr double gamma = 1.760859644e11 * mu0;
constexpr double mu_b = 9.274009994e-24;
constexpr double e_abs = 1.6021766208e-19;
constexpr double kb = 1.38064852e-23;
constexpr double hbar = 1.0545718e-34;
}  // namespace constants

using HostArray = std::vector<double>;

inline void maf_check(int rc) {
    if (rc != MAF_OK) throw std::runtime_error(std::string("magnum.af B200: ") + maf_last_error());
}

struct Mesh {
    size_t nx, ny, nz;
    double dx, dy, dz;
    Mesh(size_t nx_, size_t ny_, size_t nz_, double dx_, double dy_, double dz_)
        : nx(nx_), ny(ny_), nz(nz_), dx(dx_), dy(dy_), dz(dz_) {}
    size_t n() const { return nx * ny * nz; }
};

enum class Precision { FP64 = MAF_FP64, FP32_FIELD = MAF_FP32_FIELD };

class State {
  public:
    // Time proxy: `state.t` reads and writes the device state's time like the
    // reference's public member.
    class TimeRef {
      public:
        explicit TimeRef(State* s) : s_(s) {}
        operator double() const {
            double t = 0;
            maf_check(maf_state_get_t(s_->h_.get(), &t));
            return t;
        }
        TimeRef& operator=(double v) {
            maf_check(maf_state_set_t(s_->h_.get(), v));
            return *this;
        }
        TimeRef& operator+=(double v) { return *this = double(*this) + v; }
        TimeRef(const TimeRef&) = delete;
        TimeRef& operator=(const TimeRef& o) { return *this = double(o); }

      private:
        State* s_;
    };

    State(Mesh mesh_in, double Ms, const HostArray& m_in, Precision p = Precision::FP64)
        : mesh(mesh_in), t(this), h_(create(mesh_in, Ms, nullptr, m_in, p)) {}
    State(Mesh mesh_in, const HostArray& Ms_field, const HostArray& m_in, Precision p = Precision::FP64)
        : mesh(mesh_in), t(this), h_(create(mesh_in, std::nan(""), &Ms_field, m_in, p)) {}
    State(const State&) = delete;
    State& operator=(const State&) = delete;

    Mesh mesh;
    TimeRef t;

    HostArray m() const {
        HostArray out(3 * mesh.n());
        maf_check(maf_state_get_m(h_.get(), out.data()));
        return out;
    }
    void set_m(const HostArray& m_in) {
        check_size(m_in, 3 * mesh.n());
        maf_check(maf_state_set_m(h_.get(), m_in.data()));
    }
    unsigned long long steps() const {
        unsigned long long s = 0;
        maf_check(maf_state_get_steps(h_.get(), &s));
        return s;
    }
    std::array<double, 3> mean_m() const {
        std::array<double, 3> out{};
        maf_check(maf_state_mean_m(h_.get(), out.data()));
        return out;
    }
    double meani(int i) const { return mean_m()[i]; }
    double mean_mx() const { return mean_m()[0]; }
    double mean_my() const { return mean_m()[1]; }
    double mean_mz() const { return mean_m()[2]; }
    maf_state handle() const { return h_.get(); }

    friend std::ostream& operator<<(std::ostream& os, const State& s) {
        const auto mm = s.mean_m();
        double t = 0;
        maf_check(maf_state_get_t(s.h_.get(), &t));
        return os << t << '\t' << mm[0] << '\t' << mm[1] << '\t' << mm[2];
    }

  private:
    struct Del {
        void operator()(maf_state s) const { maf_state_destroy(s); }
    };
    static void check_size(const HostArray& a, size_t n) {
        if (a.size() != n) throw std::invalid_argument("array size does not match the mesh");
    }
    static maf_state create(const Mesh& mesh, double Ms, const HostArray* Msf, const HostArray& m, Precision p) {
        check_size(m, 3 * mesh.n());
        if (Msf) check_size(*Msf, mesh.n());
        maf_state s = nullptr;
        maf_check(maf_state_create(&s, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, mesh.dx, mesh.dy, mesh.dz, Ms,
                                   Msf ? Msf->data() : nullptr, m.data(), static_cast<int>(p)));
        return s;
    }
    std::unique_ptr<maf_state_s, Del> h_;
};

class FieldTerm {
  public:
    virtual ~FieldTerm() = default;
    HostArray H_in_Apm(const State& state) const {
        HostArray out(3 * state.mesh.n());
        maf_check(maf_term_H(h_.get(), state.handle(), out.data()));
        return out;
    }
    HostArray H_in_T(const State& state) const {
        HostArray h = H_in_Apm(state);
        for (auto& v : h) v *= constants::mu0;
        return h;
    }
    double Energy_in_J(const State& state) const {
        double e = 0;
        maf_check(maf_term_E(h_.get(), state.handle(), &e));
        return e;
    }
    double Energy_in_eV(const State& state) const { return Energy_in_J(state) / constants::e_abs; }
    maf_term handle() const { return h_.get(); }

  protected:
    struct Del {
        void operator()(maf_term t) const { maf_term_destroy(t); }
    };
    void reset(maf_term t) { h_ = std::shared_ptr<maf_term_s>(t, Del()); }
    std::shared_ptr<maf_term_s> h_;
};

class DemagField : public FieldTerm {
  public:
    // verbose/caching/nthreads are accepted for source compatibility: the tensor
    // is assembled on the GPU (demag_field.cpp:211-213 computes it on host threads)
    explicit DemagField(Mesh mesh, bool /*verbose*/ = false, bool /*caching*/ = false, unsigned /*nthreads*/ = 0) {
        maf_term t = nullptr;
        maf_check(maf_term_demag_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, mesh.dx, mesh.dy, mesh.dz));
        reset(t);
    }
};

class ExchangeField : public FieldTerm {
  public:
    explicit ExchangeField(double A) {
        maf_term t = nullptr;
        maf_check(maf_term_exchange_create(&t, A));
        reset(t);
    }
};

class DmiField : public FieldTerm {
  public:
    DmiField(double D, std::array<double, 3> D_axis = {0, 0, 1}) {
        maf_term t = nullptr;
        maf_check(maf_term_dmi_create(&t, D, D_axis[0], D_axis[1], D_axis[2]));
        reset(t);
    }
};

class BulkDMIExchangeField : public FieldTerm {
  public:
    BulkDMIExchangeField(double D, double A) {
        maf_term t = nullptr;
        maf_check(maf_term_bulkdmi_exchange_create(&t, D, A));
        reset(t);
    }
};

class UniaxialAnisotropyField : public FieldTerm {
  public:
    UniaxialAnisotropyField(double Ku1, std::array<double, 3> Ku1_axis = {0, 0, 1}) {
        maf_term t = nullptr;
        maf_check(maf_term_uniaxial_create(&t, Ku1, Ku1_axis[0], Ku1_axis[1], Ku1_axis[2]));
        reset(t);
    }
};

class CubicAnisotropyField : public FieldTerm {
  public:
    CubicAnisotropyField(double Kc1, double Kc2 = 0, double Kc3 = 0, std::array<double, 3> c1 = {1, 0, 0},
                         std::array<double, 3> c2 = {0, 1, 0}) {
        maf_term t = nullptr;
        maf_check(maf_term_cubic_create(&t, Kc1, Kc2, Kc3, c1.data(), c2.data()));
        reset(t);
    }
};

class ExternalField : public FieldTerm {
  public:
    ExternalField(const Mesh& mesh, const HostArray& zee) {
        if (zee.size() != 3 * mesh.n()) throw std::invalid_argument("ExternalField: size does not match the mesh");
        maf_term t = nullptr;
        maf_check(maf_term_external_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, zee.data()));
        reset(t);
    }
};

// DemagFieldPBC() (demag_field_pbc.cpp): the mesh is the evaluated state's
class DemagFieldPBC : public FieldTerm {
  public:
    DemagFieldPBC() {
        maf_term t = nullptr;
        maf_check(maf_term_demag_pbc_create(&t));
        reset(t);
    }
};

// SparseExchangeField(A, mesh) / (A_field, mesh) (sparse_exchange_field.cpp); A_field is [nz][ny][nx]
class SparseExchangeField : public FieldTerm {
  public:
    SparseExchangeField(double A, Mesh mesh, bool /*verbose*/ = true) {
        maf_term t = nullptr;
        maf_check(maf_term_sparse_exchange_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, nullptr, A));
        reset(t);
    }
    SparseExchangeField(const HostArray& A_field, Mesh mesh, bool /*verbose*/ = true) {
        if (A_field.size() != mesh.n())
            throw std::invalid_argument("SparseExchangeField: size does not match the mesh");
        maf_term t = nullptr;
        maf_check(maf_term_sparse_exchange_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, A_field.data(), 0.0));
        reset(t);
    }
};

// ExchangeFieldPBC(A, mesh) / (A_field, mesh) (exchange_field_pbc.cpp)
class ExchangeFieldPBC : public FieldTerm {
  public:
    ExchangeFieldPBC(double A, Mesh mesh, bool /*verbose*/ = true) {
        maf_term t = nullptr;
        maf_check(maf_term_exchange_pbc_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, nullptr, A));
        reset(t);
    }
    ExchangeFieldPBC(const HostArray& A_field, Mesh mesh, bool /*verbose*/ = true) {
        if (A_field.size() != mesh.n()) throw std::invalid_argument("ExchangeFieldPBC: size does not match the mesh");
        maf_term t = nullptr;
        maf_check(maf_term_exchange_pbc_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, A_field.data(), 0.0));
        reset(t);
    }
};

// SpinTransferTorqueField(polarization, eta_damping, eta_field, j_e, fl_thickness)
// (spin_transfer_torque_field.cpp); polarization is [3][nz][ny][nx]
class SpinTransferTorqueField : public FieldTerm {
  public:
    SpinTransferTorqueField(const Mesh& mesh, const HostArray& polarization, double eta_damping, double eta_field,
                            double j_e, double fl_thickness) {
        if (polarization.size() != 3 * mesh.n())
            throw std::invalid_argument("SpinTransferTorqueField: size does not match the mesh");
        maf_term t = nullptr;
        maf_check(maf_term_stt_create(&t, (int)mesh.nx, (int)mesh.ny, (int)mesh.nz, polarization.data(), eta_damping,
                                      eta_field, j_e, fl_thickness));
        reset(t);
    }
};

using uptr_FieldTerm = std::unique_ptr<FieldTerm>;
using vec_uptr_FieldTerm = std::vector<uptr_FieldTerm>;

namespace fieldterm {
template <typename T, class... Args> uptr_FieldTerm to_uptr(Args&&... args) {
    return uptr_FieldTerm(new T(std::forward<Args>(args)...));
}
template <typename... Args> vec_uptr_FieldTerm to_vec(Args... args) {
    vec_uptr_FieldTerm v;
    (v.push_back(uptr_FieldTerm(new Args(std::move(args)))), ...);
    return v;
}
}  // namespace fieldterm

struct Controller {
    double hmin, hmax, atol, rtol;
    Controller(double hmin_ = 1e-15, double hmax_ = 3.5e-10, double atol_ = 1e-6, double rtol_ = 1e-6)
        : hmin(hmin_), hmax(hmax_), atol(atol_), rtol(rtol_) {}
};

class LLGIntegrator {
  public:
    // `llg.llgterms.push_back(...)` appends a term to the device integrator
    class Terms {
      public:
        explicit Terms(LLGIntegrator* l) : l_(l) {}
        void push_back(uptr_FieldTerm t) {
            maf_check(maf_llg_add_term(l_->h_.get(), t->handle()));
            l_->owned_.push_back(std::move(t));
        }
        size_t size() const { return l_->owned_.size(); }

      private:
        LLGIntegrator* l_;
    };
    class AlphaRef {
      public:
        explicit AlphaRef(LLGIntegrator* l) : l_(l) {}
        AlphaRef& operator=(double a) {
            l_->alpha_ = a;
            maf_check(maf_llg_set_alpha(l_->h_.get(), a));
            return *this;
        }
        operator double() const { return l_->alpha_; }

      private:
        LLGIntegrator* l_;
    };

    LLGIntegrator(double alpha_in, vec_uptr_FieldTerm terms, const std::string& scheme = "RKF45",
                  Controller c = Controller(), bool dissipation_term_only = false)
        : llgterms(this), alpha(this), alpha_(alpha_in), owned_(std::move(terms)) {
        std::vector<maf_term> hs;
        for (auto& t : owned_) hs.push_back(t->handle());
        maf_llg l = nullptr;
        maf_check(maf_llg_create(&l, alpha_in, nullptr, 0, 0, 0, hs.data(), (int)hs.size(), scheme.c_str(), c.hmin,
                                 c.hmax, c.atol, c.rtol, dissipation_term_only ? 1 : 0));
        h_.reset(l);
    }
    LLGIntegrator(const LLGIntegrator&) = delete;
    LLGIntegrator& operator=(const LLGIntegrator&) = delete;

    Terms llgterms;
    AlphaRef alpha;

    void step(State& state) { maf_check(maf_llg_step(h_.get(), state.handle())); }
    double E(const State& state) const {
        double e = 0;
        maf_check(maf_llg_E(h_.get(), state.handle(), &e));
        return e;
    }
    HostArray h(const State& state) const {
        HostArray out(3 * state.mesh.n());
        maf_check(maf_llg_heff(h_.get(), state.handle(), out.data()));
        return out;
    }
    void relax(State& state, double precision = 1e-10, unsigned eval_E = 100) {
        maf_check(maf_llg_relax(h_.get(), state.handle(), precision, (int)eval_E));
    }
    // llg_integrator.cpp:68-104; rows "t <mx> <my> <mz>" like `os << state`
    void integrate_dense(State& state, double time_in_s, double write_every_dt_in_s, std::ostream& os) {
        const int max_rows = (int)std::ceil(time_in_s / write_every_dt_in_s) + 4;
        std::vector<double> rows(4 * (size_t)max_rows);
        int n = 0;
        maf_check(maf_llg_integrate_dense(h_.get(), state.handle(), time_in_s, write_every_dt_in_s, rows.data(),
                                          max_rows, &n));
        for (int i = 0; i < n; ++i)
            os << rows[4 * i] << '\t' << rows[4 * i + 1] << '\t' << rows[4 * i + 2] << '\t' << rows[4 * i + 3] << '\n';
    }
    unsigned long long accumulated_steps() const {
        unsigned long long c[4] = {0, 0, 0, 0};
        maf_check(maf_llg_counters(h_.get(), c));
        return c[0];
    }

  private:
    struct Del {
        void operator()(maf_llg l) const { maf_llg_destroy(l); }
    };
    double alpha_;
    vec_uptr_FieldTerm owned_;
    std::unique_ptr<maf_llg_s, Del> h_;
};

}  // namespace magnumaf
