// C ABI of the magnum.af B200 library (declared in include/maf_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/maf_b200.h"
#include "capi_internal.hpp"
#include "batch.hpp"
#include "engine.hpp"
#include "rk.hpp"

using namespace mafb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

template <typename F> int guarded(F&& f) {
    try {
        g_last_error.clear();
        f();
        return MAF_OK;
    } catch (const Error& e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return fail(MAF_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(MAF_ERR_CUDA, e.what());
    }
}

void require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw Error(MAF_ERR_NODEVICE, "no CUDA device available: the magnum.af B200 library has no CPU path");
    }
}

void check(bool ok, const std::string& msg) {
    if (!ok) throw Error(MAF_ERR_BADARG, msg);
}

// ---------------------------------------------------------------------------
// Controller (magnumaf/include/magnumaf/integrators/controller.hpp:11-61,
//             magnumaf/src/integrators/controller.cpp:36-95)
// ---------------------------------------------------------------------------
struct Controller {
    double hmin = 1e-15, hmax = 3.5e-10, atol = 1e-6, rtol = 1e-6;
    const double beta = 0.4 / 5.0;
    const double alpha = 0.2 - 0.75 * beta;
    const double headroom = 0.9;
    const double minscale = 0.2;
    const double maxscale = 10.;
    bool reject = false;
    double errold = 1.0e-4;
    double hnext = 0.0;
    unsigned long long n_reject = 0, n_accepted = 0, n_hmax = 0, n_hmin = 0;

    bool success(double err, double& h) {
        double scale;
        if (err <= 1.0) {
            if (err == 0.0) {
                scale = maxscale;
            } else {
                scale = headroom * std::pow(err, -alpha) * std::pow(errold, beta);
                if (scale < minscale) scale = minscale;
                if (scale > maxscale) scale = maxscale;
            }
            hnext = reject ? h * std::min(scale, 1.0) : h * scale;
            if (hnext <= hmin) {
                hnext = hmin;
                ++n_hmin;
            } else if (hnext >= hmax) {
                hnext = hmax;
                ++n_hmax;
            }
            errold = std::max(err, 1.0e-4);
            reject = false;
            ++n_accepted;
            return true;
        }
        scale = std::max(headroom * std::pow(err, -alpha), minscale);
        h *= scale;
        if (h <= hmin) {
            h = hmin;
            ++n_hmin;
            return true;
        }
        if (h >= hmax) {
            h = hmax;
            ++n_hmax;
            return true;
        }
        reject = true;
        ++n_reject;
        return false;
    }
};

// Butcher tableaus (adaptive_runge_kutta.cpp:75-173, 496-529); coefficients
// with dt_in_k == false are multiplied by dt at run time (BS23 keeps k = f).
struct Scheme {
    int stages = 0;
    double a[8][8] = {};
    double b[8] = {};
    double e[8] = {};
    int form = 0;  // 0: err = sum e_j k_j ; 1: err = sumbk - sum e_j k_j
    bool dt_in_k = true;
};

Scheme make_scheme(const std::string& name) {
    Scheme s;
    if (name == "RKF45") {
        s.stages = 6;
        s.a[1][0] = 1. / 4.;
        s.a[2][0] = 3. / 32.; s.a[2][1] = 9 / 32.;
        s.a[3][0] = 1932. / 2197.; s.a[3][1] = -7200. / 2197.; s.a[3][2] = 7296. / 2197.;
        s.a[4][0] = 439. / 216.; s.a[4][1] = -8.; s.a[4][2] = 3680. / 513.; s.a[4][3] = -845. / 4104.;
        s.a[5][0] = -8. / 27.; s.a[5][1] = 2.; s.a[5][2] = -3544. / 2565.; s.a[5][3] = 1859. / 4104.;
        s.a[5][4] = -11. / 40.;
        const double b[6] = {16. / 135., 0, 6656. / 12825., 28561. / 56430., -9. / 50., 2. / 55.};
        const double bh[6] = {25. / 216., 0, 1408. / 2565., 2197. / 4104., -1. / 5., 0};
        for (int i = 0; i < 6; ++i) { s.b[i] = b[i]; s.e[i] = bh[i]; }
        s.form = 1;
    } else if (name == "DP45") {
        s.stages = 7;
        s.a[1][0] = 0.2;
        s.a[2][0] = 3.0 / 40.0; s.a[2][1] = 9.0 / 40.0;
        s.a[3][0] = 44.0 / 45.0; s.a[3][1] = -56.0 / 15.0; s.a[3][2] = 32.0 / 9.0;
        s.a[4][0] = 19372.0 / 6561.0; s.a[4][1] = -25360.0 / 2187.0; s.a[4][2] = 64448.0 / 6561.0;
        s.a[4][3] = -212.0 / 729.0;
        s.a[5][0] = 9017.0 / 3168.0; s.a[5][1] = -355.0 / 33.0; s.a[5][2] = 46732.0 / 5247.0;
        s.a[5][3] = 49.0 / 176.0; s.a[5][4] = -5103.0 / 18656.0;
        s.a[6][0] = 35.0 / 384.0; s.a[6][2] = 500.0 / 1113.0; s.a[6][3] = 125.0 / 192.0;
        s.a[6][4] = -2187.0 / 6784.0; s.a[6][5] = 11.0 / 84.0;
        for (int j = 0; j < 6; ++j) s.b[j] = s.a[6][j];
        const double e[7] = {71.0 / 57600.0, 0, -71.0 / 16695.0, 71.0 / 1920.0, -17253.0 / 339200.0, 22.0 / 525.0,
                             -1.0 / 40.0};
        for (int j = 0; j < 7; ++j) s.e[j] = e[j];
        s.form = 0;
    } else if (name == "BS23") {
        s.stages = 4;
        s.dt_in_k = false;
        s.a[1][0] = 1. / 2.;
        s.a[2][1] = 3. / 4.;
        s.a[3][0] = 2. / 9.; s.a[3][1] = 1. / 3.; s.a[3][2] = 4. / 9.;
        s.b[0] = 2. / 9.; s.b[1] = 1. / 3.; s.b[2] = 4. / 9.;
        s.e[0] = 7. / 24.; s.e[1] = 1. / 4.; s.e[2] = 1. / 3.; s.e[3] = 1. / 8.;
        s.form = 1;
    } else {
        throw Error(MAF_ERR_BADARG, "Integration method not found. Valid arguments are 'RKF45', 'DP45', 'BS23'");
    }
    return s;
}

}  // namespace

// Error handling shared with entry points defined in other translation units:
// runs f after the device check and maps exceptions to status codes and
// maf_last_error() exactly like the entry points in this file.
int mafb::capi_run(const std::function<void()>& f) {
    return guarded([&] {
        require_device();
        f();
    });
}

// ---------------------------------------------------------------------------
// handle structs
// ---------------------------------------------------------------------------
// Buffers and streams of the pipelined evaluation (maf_llg_heff_pipeline).
struct HeffPipe {
    DevBuf m[2], h[2], m32, m_in32[2];  // m_in32: FP32 host inputs (maf_llg_heff_pipeline_m32)
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t up_done[2] = {}, comp_done[2] = {}, down_done[2] = {};
    ~HeffPipe() {
        for (int b = 0; b < 2; ++b) {
            if (up_done[b]) cudaEventDestroy(up_done[b]);
            if (comp_done[b]) cudaEventDestroy(comp_done[b]);
            if (down_done[b]) cudaEventDestroy(down_done[b]);
        }
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
    }
};

struct maf_state_s {
    StateD s;
    DevBuf scratch;  // reductions
    bool m32_valid = false;
    std::unique_ptr<HeffPipe> pipe;
    ~maf_state_s() {
        if (s.stream) cudaStreamSynchronize(s.stream);
        pipe.reset();
        if (s.own_stream && s.stream) cudaStreamDestroy(s.stream);
    }
};

struct maf_term_s {
    std::shared_ptr<Term> t;
};

struct maf_llg_s {
    double alpha = 0;
    DevBuf alpha_field;
    bool has_alpha_field = false;
    int alpha_n = 0;
    std::vector<std::shared_ptr<Term>> terms;
    std::string scheme_name = "RKF45";
    Scheme scheme;
    Controller ctrl;
    double h = 1.01e-15;
    bool dissipation_only = false;
    DevBuf k[8];
    DevBuf mstage64, mstage32, mcand, partials, errbuf, h32out;
    unsigned long long accumulated_steps = 0;
    std::vector<std::string> prof_names;  // interval names of the last maf_llg_attempt_profile
};

namespace {

void ensure_m32(maf_state_s* st) {
    StateD& s = st->s;
    if (s.precision != PREC_FP32_FIELD) return;
    s.m32.ensure(sizeof(float) * 3 * s.md.N());
    if (!st->m32_valid) {
        stage_m32(s.m64.as<double>(), s.m32.as<float>(), 3 * s.md.N(), s.stream);
        st->m32_valid = true;
    }
}

std::vector<Term*> raw_terms(const std::vector<std::shared_ptr<Term>>& v) {
    std::vector<Term*> r;
    for (auto& p : v) r.push_back(p.get());
    return r;
}

// Field of `terms` on the state's current m with the given epilogue.
void eval_on_state(maf_state_s* st, const std::vector<Term*>& terms, EpilogueArgs ep, double* energy = nullptr,
                   const double* m64_for_llg = nullptr, PassMarks* marks = nullptr) {
    StateD& s = st->s;
    if (ep.kind == EPI_LLG && !ep.llg.m64) ep.llg.m64 = m64_for_llg ? m64_for_llg : s.m64.as<double>();
    if (s.precision == PREC_FP32_FIELD) {
        ensure_m32(st);
        eval_terms<float>(terms, s.md, s.m32.as<float>(), s.msinfo(), ep, s.stream, st->scratch, energy, marks);
    } else {
        eval_terms<double>(terms, s.md, s.m64.as<double>(), s.msinfo(), ep, s.stream, st->scratch, energy, marks);
    }
}

// interval names of the attempt profile that carry the number of FP64 k
// buffers a Runge-Kutta kernel reads (its algorithmic bytes depend on it)
const char* const kCombineNames[8] = {"rk_combine_k0", "rk_combine_k1", "rk_combine_k2", "rk_combine_k3",
                                      "rk_combine_k4", "rk_combine_k5", "rk_combine_k6", "rk_combine_k7"};
const char* const kFinalizeNames[9] = {"rk_finalize_k0", "rk_finalize_k1", "rk_finalize_k2",
                                       "rk_finalize_k3", "rk_finalize_k4", "rk_finalize_k5",
                                       "rk_finalize_k6", "rk_finalize_k7", "rk_finalize_k8"};

LLGParams llg_params(const maf_llg_s* l, double scale) {
    LLGParams p;
    const double a = l->alpha;
    p.c_prec = -kGamma / (1. + a * a);
    p.c_damp = -a * kGamma / (1. + a * a);
    p.alpha = l->has_alpha_field ? l->alpha_field.as<double>() : nullptr;
    p.dissipation_only = l->dissipation_only ? 1 : 0;
    p.scale = scale;
    return p;
}

// One RK attempt of `sch` with step dt; leaves m + sumbk (normalised per
// norm_mode) in l->mcand and returns the error norm.
double rk_attempt(maf_llg_s* l, maf_state_s* st, const Scheme& sch, double dt, int norm_mode,
                  PassMarks* marks = nullptr) {
    StateD& s = st->s;
    const int64_t N = s.md.N();
    const int64_t n3 = 3 * N;
    const bool f32 = s.precision == PREC_FP32_FIELD;
    for (int i = 0; i < sch.stages; ++i) l->k[i].ensure(sizeof(double) * n3);
    l->mstage64.ensure(sizeof(double) * n3);
    if (f32) l->mstage32.ensure(sizeof(float) * n3);
    l->mcand.ensure(sizeof(double) * n3);
    l->partials.ensure(sizeof(double) * sm_count() * 8 + 64);
    l->errbuf.ensure(sizeof(double) * 4);
    auto terms = raw_terms(l->terms);
    const double kscale = sch.dt_in_k ? dt : 1.0;
    const double cmul = sch.dt_in_k ? 1.0 : dt;
    for (int stg = 0; stg < sch.stages; ++stg) {
        EpilogueArgs ep;
        ep.kind = EPI_LLG;
        ep.out = l->k[stg].p;
        ep.llg = llg_params(l, kscale);
        if (stg == 0) {
            ep.llg.m64 = s.m64.as<double>();
            if (marks) {
                marks->mark(s.stream, "attempt");
                if (s.precision == PREC_FP32_FIELD) {  // the FP64 form has no FP32 copy
                    ensure_m32(st);
                    marks->mark(s.stream, "stage_m32");
                }
            }
            eval_on_state(st, terms, ep, nullptr, nullptr, marks);
        } else {
            KList kl;
            for (int j = 0; j < stg; ++j) {
                if (sch.a[stg][j] == 0.0) continue;
                kl.k[kl.n] = l->k[j].as<double>();
                kl.c[kl.n] = sch.dt_in_k ? sch.a[stg][j] : dt * sch.a[stg][j];
                ++kl.n;
            }
            rk_combine(s.m64.as<double>(), kl, l->mstage64.as<double>(), f32 ? l->mstage32.as<float>() : nullptr, n3,
                       s.stream);
            if (marks) marks->mark(s.stream, kCombineNames[kl.n]);
            ep.llg.m64 = l->mstage64.as<double>();
            if (f32)
                eval_terms<float>(terms, s.md, l->mstage32.as<float>(), s.msinfo(), ep, s.stream, st->scratch, nullptr,
                                  marks);
            else
                eval_terms<double>(terms, s.md, l->mstage64.as<double>(), s.msinfo(), ep, s.stream, st->scratch,
                                   nullptr, marks);
        }
    }
    KList kb, ke;
    for (int j = 0; j < sch.stages; ++j) {
        if (sch.b[j] != 0.0) {
            kb.k[kb.n] = l->k[j].as<double>();
            kb.c[kb.n] = sch.b[j] * cmul;
            ++kb.n;
        }
        if (sch.e[j] != 0.0) {
            ke.k[ke.n] = l->k[j].as<double>();
            ke.c[ke.n] = sch.e[j] * cmul;
            ++ke.n;
        }
    }
    rk_finalize(s.m64.as<double>(), kb, ke, sch.form, l->ctrl.atol, l->ctrl.rtol, l->mcand.as<double>(), norm_mode, N,
                l->partials.as<double>(), l->errbuf.as<double>(), s.stream);
    if (marks) {
        std::vector<const double*> uniq;
        for (int j = 0; j < kb.n; ++j) uniq.push_back(kb.k[j]);
        for (int j = 0; j < ke.n; ++j)
            if (std::find(uniq.begin(), uniq.end(), ke.k[j]) == uniq.end()) uniq.push_back(ke.k[j]);
        marks->mark(s.stream, kFinalizeNames[std::min<size_t>(uniq.size(), 8)]);
    }
    double err = 0;
    MAF_CUDA(cudaMemcpyAsync(&err, l->errbuf.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MAF_CUDA(cudaStreamSynchronize(s.stream));
    return err;
}

void accept_candidate(maf_llg_s* l, maf_state_s* st) {
    std::swap(st->s.m64, l->mcand);
    st->m32_valid = false;
}

void llg_step(maf_llg_s* l, maf_state_s* st) {
    StateD& s = st->s;
    const int norm_mode = s.has_Ms_field ? 2 : 1;
    while (true) {
        const double err = rk_attempt(l, st, l->scheme, l->h, norm_mode);
        if (!(err == err) || std::isinf(err))
            throw Error(MAF_ERR_NAN, "NaN/Inf in the Runge-Kutta error norm (t=" + std::to_string(s.t) + ")");
        if (l->ctrl.success(err, l->h)) break;
    }
    s.t += l->h;
    l->h = l->ctrl.hnext;
    accept_candidate(l, st);
    s.steps++;
    l->accumulated_steps++;
}

void mean_m_host(maf_state_s* st, const double* m64, double out[3]) {
    StateD& s = st->s;
    const int nres = 4 * mean_m_blocks();
    st->scratch.ensure(sizeof(double) * (nres + 8));
    double* scr = st->scratch.as<double>();
    mean_m(m64, s.md.N(), scr, scr + nres, s.stream);
    MAF_CUDA(cudaMemcpyAsync(out, scr + nres, 3 * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MAF_CUDA(cudaStreamSynchronize(s.stream));
}

double llg_energy(maf_llg_s* l, maf_state_s* st) {
    EpilogueArgs ep;
    ep.kind = EPI_EDENS;
    double e = 0;
    eval_on_state(st, raw_terms(l->terms), ep, &e);
    return e;
}

void upload(DevBuf& b, const double* host, size_t n, cudaStream_t st) {
    b.alloc(sizeof(double) * n);
    MAF_CUDA(cudaMemcpyAsync(b.p, host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    MAF_CUDA(cudaStreamSynchronize(st));
}

void H_to_host(maf_state_s* st, const std::vector<Term*>& terms, double* H_host, float* H32_host, DevBuf& tmp) {
    StateD& s = st->s;
    const int64_t n3 = 3 * s.md.N();
    EpilogueArgs ep;
    ep.kind = EPI_H;
    if (s.precision == PREC_FP32_FIELD) {
        // [float H32 | pad to 256 B | double H64]
        const size_t off = (sizeof(float) * n3 + 255) / 256 * 256;
        tmp.ensure(off + sizeof(double) * n3);
        float* h32 = tmp.as<float>();
        ep.out = h32;
        eval_on_state(st, terms, ep);
        if (H32_host) {
            MAF_CUDA(cudaMemcpyAsync(H32_host, h32, sizeof(float) * n3, cudaMemcpyDeviceToHost, s.stream));
        } else {
            double* h64 = reinterpret_cast<double*>(static_cast<char*>(tmp.p) + off);
            f32_to_f64(h32, h64, n3, s.stream);
            MAF_CUDA(cudaMemcpyAsync(H_host, h64, sizeof(double) * n3, cudaMemcpyDeviceToHost, s.stream));
        }
    } else {
        if (H32_host) throw Error(MAF_ERR_BADARG, "FP32 field output requested from an FP64 state");
        tmp.ensure(sizeof(double) * n3);
        ep.out = tmp.p;
        eval_on_state(st, terms, ep);
        MAF_CUDA(cudaMemcpyAsync(H_host, tmp.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, s.stream));
    }
    MAF_CUDA(cudaStreamSynchronize(s.stream));
}

thread_local DevBuf g_tmp;  // host-copy staging for H outputs

}  // namespace

// ---------------------------------------------------------------------------
// Stochastic LLG (magnumaf/src/integrators/stochastic_integrator.cpp:8-57,
// stochastic_llg.cpp:19-22): fixed-step Heun, semi-implicit Heun and the
// deterministic RK4 reference, with thermal fields from the counter-based
// generator (rng.cuh): the field of noise index n is sigma * xi(seed, member, n).
// Heun step s uses xi(s) as the predictor's ("previous") field and xi(s+1) as
// the corrector's; the semi-implicit scheme draws xi(2s) and xi(2s+1).
// ---------------------------------------------------------------------------
struct maf_stoch_s {
    double alpha = 0, T = 0, dt = 0;
    int mode = 0;  // 0 Heun, 1 SemiHeun, 2 detRK4
    unsigned long long seed = 0;
    unsigned member = 0;
    unsigned long long calls = 0;  // accepted steps
    std::vector<std::shared_ptr<Term>> terms;
    DevBuf k[6];
    DevBuf mstage64, mstage32, mcand, partials, errbuf;
};

namespace {

double thermal_sigma(const maf_stoch_s* h, const StateD& s) {
    // D = alpha kB T / (gamma mu0 Ms dV), h_th = sqrt(2 D / dt) N(0,1)
    const double dV = s.md.dx * s.md.dy * s.md.dz;
    const double D = (h->alpha * kKb * h->T) / (kGamma * kMu0 * s.Ms * dV);
    return std::sqrt((2. * D) / h->dt);
}

struct StochStage {
    int n = 0;
    int j[6] = {};
    double c[6] = {};
    bool noise = false;
    unsigned long long index = 0;
    double scale = 0;
};

// One step.  With q_dev (a device copy of h->calls) the noise stream indices are
// read from q_dev on the device and q_dev is advanced by a device kernel, so the
// step can be captured in a CUDA graph and replayed.
void stoch_step(maf_stoch_s* h, maf_state_s* st, unsigned long long* q_dev = nullptr) {
    StateD& s = st->s;
    if (s.has_Ms_field) throw Error(MAF_ERR_BADARG, "Stochastic_LLG uses the scalar Ms (stochastic_integrator.cpp:9-10)");
    const int64_t N = s.md.N(), n3 = 3 * N;
    const bool f32 = s.precision == PREC_FP32_FIELD;
    const double dt = h->dt;
    const double sigma = thermal_sigma(h, s);
    const unsigned long long q = h->calls;
    std::vector<StochStage> stages;
    KList fin;
    if (h->mode == 0) {  // Heun (stochastic_integrator.cpp:8-17)
        StochStage a; a.noise = true; a.index = q; a.scale = dt;
        StochStage b; b.n = 1; b.j[0] = 0; b.c[0] = 1.0; b.noise = true; b.index = q + 1; b.scale = dt;
        stages = {a, b};
        fin.n = 2; fin.c[0] = 0.5; fin.c[1] = 0.5;  // (k1 + k2) / 2
    } else if (h->mode == 1) {  // semi-implicit Heun (:19-32)
        StochStage a; a.noise = true; a.index = 2 * q; a.scale = dt / 2.;
        stages.push_back(a);
        for (int i = 1; i < 6; ++i) {
            StochStage b; b.n = 1; b.j[0] = i - 1; b.c[0] = 1.0; b.noise = true; b.index = 2 * q + 1;
            b.scale = i < 5 ? dt / 2. : dt;
            stages.push_back(b);
        }
        fin.n = 1; fin.c[0] = 1.0;
    } else {  // deterministic RK4 (:34-40)
        StochStage a; a.scale = dt;
        StochStage b; b.n = 1; b.j[0] = 0; b.c[0] = 1. / 2.; b.scale = dt;
        StochStage c; c.n = 1; c.j[0] = 1; c.c[0] = 1. / 2.; c.scale = dt;
        StochStage d; d.n = 1; d.j[0] = 2; d.c[0] = 1.0; d.scale = dt;
        stages = {a, b, c, d};
        fin.n = 4; fin.c[0] = 1. / 6.; fin.c[1] = 2. / 6.; fin.c[2] = 2. / 6.; fin.c[3] = 1. / 6.;
    }
    for (size_t i = 0; i < stages.size(); ++i) h->k[i].ensure(sizeof(double) * n3);
    h->mstage64.ensure(sizeof(double) * n3);
    if (f32) h->mstage32.ensure(sizeof(float) * n3);
    h->mcand.ensure(sizeof(double) * n3);
    h->partials.ensure(sizeof(double) * sm_count() * 8 + 64);
    h->errbuf.ensure(sizeof(double) * 4);
    std::vector<Term*> terms;
    for (auto& t : h->terms) terms.push_back(t.get());
    for (size_t i = 0; i < stages.size(); ++i) {
        const StochStage& sg = stages[i];
        EpilogueArgs ep;
        ep.kind = EPI_LLG;
        ep.out = h->k[i].p;
        ep.llg.c_prec = -kGamma / (1. + h->alpha * h->alpha);
        ep.llg.c_damp = -h->alpha * kGamma / (1. + h->alpha * h->alpha);
        ep.llg.scale = sg.scale;
        if (sg.noise) {
            ep.llg.sigma = sigma;
            ep.llg.seed = h->seed;
            ep.llg.member = h->member;
            ep.llg.noise_index = sg.index;
            if (q_dev) {  // index = mul * q + offset, q read on the device
                const unsigned mul = h->mode == 1 ? 2u : 1u;
                ep.llg.noise_base = q_dev;
                ep.llg.noise_mul = mul;
                ep.llg.noise_index = sg.index - mul * q;
            }
        }
        if (sg.n == 0) {
            ep.llg.m64 = s.m64.as<double>();
            eval_on_state(st, terms, ep);
        } else {
            KList kl;
            for (int t = 0; t < sg.n; ++t) {
                kl.k[kl.n] = h->k[sg.j[t]].as<double>();
                kl.c[kl.n] = sg.c[t];
                ++kl.n;
            }
            rk_combine(s.m64.as<double>(), kl, h->mstage64.as<double>(), f32 ? h->mstage32.as<float>() : nullptr, n3,
                       s.stream);
            ep.llg.m64 = h->mstage64.as<double>();
            if (f32)
                eval_terms<float>(terms, s.md, h->mstage32.as<float>(), s.msinfo(), ep, s.stream, st->scratch, nullptr);
            else
                eval_terms<double>(terms, s.md, h->mstage64.as<double>(), s.msinfo(), ep, s.stream, st->scratch,
                                   nullptr);
        }
    }
    // m <- normalize(m + sum), normalize = the zero-safe util::normalize (:52)
    const int base = h->mode == 1 ? 5 : 0;
    for (int t = 0; t < fin.n; ++t) fin.k[t] = h->k[base + t].as<double>();
    KList dummy;
    dummy.n = 1;
    dummy.k[0] = fin.k[0];
    dummy.c[0] = 0.0;
    rk_finalize(s.m64.as<double>(), fin, dummy, 0, 1.0, 0.0, h->mcand.as<double>(), 2, N, h->partials.as<double>(),
                h->errbuf.as<double>(), s.stream);
    std::swap(s.m64, h->mcand);
    if (q_dev) inc_counter(q_dev, s.stream);
    st->m32_valid = false;
    s.t += dt;
    s.steps++;
    h->calls++;
}

}  // namespace

// ---------------------------------------------------------------------------
// LBFGS minimiser (magnumaf/src/solvers/lbfgs_minimizer.cpp:33-505): m = 5
// two-loop recursion on the normalised magnetisation with g = m x (m x H),
// More-Thuente line search; scalars and control flow on the host, every
// vector operation on the device (one reduction = one synchronisation, as in
// the reference's scalar<double>() reads).
// ---------------------------------------------------------------------------
struct maf_lbfgs_s {
    std::vector<std::shared_ptr<Term>> terms;
    double tolerance = 1e-6;
    size_t maxIter = 230;
    DevBuf sV[5], yV[5], q, s, y, grad, grad_old, x_old, wa, red;
    DevBuf coef;           // device scalars: alpha[5] of the two-loop recursion, its current dot product, 3 more
    double rho[5] = {};    // 1 / (s . y) of each stored pair
    unsigned long long fevals = 0, iterations = 0;
    double last_gradnorm = 0;
};

namespace {

struct LbfgsCtx {
    maf_lbfgs_s* h;
    maf_state_s* st;
    int64_t n3, N;
    cudaStream_t stream;
    double* red() const { return h->red.as<double>(); }
    double dot(const DevBuf& a, const DevBuf& b) const {
        return dot_host(a.as<double>(), b.as<double>(), n3, red(), stream);
    }
    double maxabs(const double* a) const { return maxabs_host(a, n3, red(), stream); }
};

// EnergyAndGradient of the state's current m and the directional derivative g . s,
// read back with one synchronisation (the energy scaled as eval_terms scales it)
void lbfgs_egrad_dg(const LbfgsCtx& c, DevBuf& g, const DevBuf& s, double& f, double& dg) {
    std::vector<Term*> terms;
    for (auto& t : c.h->terms) terms.push_back(t.get());
    double* two = c.h->coef.as<double>() + 6;
    EpilogueArgs ep;
    ep.kind = EPI_EGRAD;
    ep.out = g.p;
    ep.llg.m64 = c.st->s.m64.as<double>();
    ep.energy_dev = two;
    eval_on_state(c.st, terms, ep, nullptr);
    c.h->fevals++;
    dot_dev(g.as<double>(), s.as<double>(), c.n3, c.red(), two + 1, c.stream);
    double v[2];
    MAF_CUDA(cudaMemcpyAsync(v, two, sizeof(v), cudaMemcpyDeviceToHost, c.stream));
    MAF_CUDA(cudaStreamSynchronize(c.stream));
    const MeshDims& md = c.st->s.md;
    f = v[0] * md.dx * md.dy * md.dz;
    dg = v[1];
}

// EnergyAndGradient (lbfgs_minimizer.cpp:38-42) of the state's current m
double lbfgs_egrad(const LbfgsCtx& c, DevBuf& g) {
    std::vector<Term*> terms;
    for (auto& t : c.h->terms) terms.push_back(t.get());
    EpilogueArgs ep;
    ep.kind = EPI_EGRAD;
    ep.out = g.p;
    ep.llg.m64 = c.st->s.m64.as<double>();
    double e = 0;
    eval_on_state(c.st, terms, ep, &e);
    c.h->fevals++;
    return e;
}

// cstep (lbfgs_minimizer.cpp:362-505)
void cstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp, double fp, double dp,
           bool& brackt, double stpmin, double stpmax, int& info) {
    info = 0;
    bool bound = false;
    if ((brackt && ((stp <= std::min(stx, sty)) || (stp >= std::max(stx, sty)))) || (dx * (stp - stx) >= 0.0) ||
        (stpmax < stpmin))
        return;
    const double sgnd = dp * (dx / std::fabs(dx));
    double stpf = 0, stpc = 0, stpq = 0;
    if (fp > fx) {
        info = 1;
        bound = true;
        const double theta = 3. * (fx - fp) / (stp - stx) + dx + dp;
        const double s = std::max(theta, std::max(dx, dp));
        double gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp < stx) gamma = -gamma;
        const double p = (gamma - dx) + theta;
        const double q = ((gamma - dx) + gamma) + dp;
        const double r = p / q;
        stpc = stx + r * (stp - stx);
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.) * (stp - stx);
        stpf = std::fabs(stpc - stx) < std::fabs(stpq - stx) ? stpc : stpc + (stpq - stpc) / 2;
        brackt = true;
    } else if (sgnd < 0.0) {
        info = 2;
        bound = false;
        const double theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        const double s = std::max(theta, std::max(dx, dp));
        double gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp > stx) gamma = -gamma;
        const double p = (gamma - dp) + theta;
        const double q = ((gamma - dp) + gamma) + dx;
        const double r = p / q;
        stpc = stp + r * (stx - stp);
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
        brackt = true;
    } else if (std::fabs(dp) < std::fabs(dx)) {
        info = 3;
        bound = true;
        const double theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        const double s = std::max(theta, std::max(dx, dp));
        double gamma = s * std::sqrt(std::max(0., (theta / s) * (theta / s) - (dx / s) * (dp / s)));
        if (stp > stx) gamma = -gamma;
        const double p = (gamma - dp) + theta;
        const double q = (gamma + (dx - dp)) + gamma;
        const double r = p / q;
        if ((r < 0.0) && (gamma != 0.0)) stpc = stp + r * (stx - stp);
        else if (stp > stx) stpc = stpmax;
        else stpc = stpmin;
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        if (brackt) stpf = std::fabs(stp - stpc) < std::fabs(stp - stpq) ? stpc : stpq;
        else stpf = std::fabs(stp - stpc) > std::fabs(stp - stpq) ? stpc : stpq;
    } else {
        info = 4;
        bound = false;
        if (brackt) {
            const double theta = 3 * (fp - fy) / (sty - stp) + dy + dp;
            const double s = std::max(theta, std::max(dy, dp));
            double gamma = s * std::sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s));
            if (stp > sty) gamma = -gamma;
            const double p = (gamma - dp) + theta;
            const double q = ((gamma - dp) + gamma) + dy;
            const double r = p / q;
            stpc = stp + r * (sty - stp);
            stpf = stpc;
        } else if (stp > stx) {
            stpf = stpmax;
        } else {
            stpf = stpmin;
        }
    }
    if (fp > fx) {
        sty = stp;
        fy = fp;
        dy = dp;
    } else {
        if (sgnd < 0.0) {
            sty = stx;
            fy = fx;
            dy = dx;
        }
        stx = stp;
        fx = fp;
        dx = dp;
    }
    stpf = std::min(stpmax, stpf);
    stpf = std::max(stpmin, stpf);
    stp = stpf;
    if (brackt && bound) {
        if (sty > stx) stp = std::min(stx + 0.66 * (sty - stx), stp);
        else stp = std::max(stx + 0.66 * (sty - stx), stp);
    }
}

// cvsrch (lbfgs_minimizer.cpp:213-360): wa = x_old, s = search direction (device)
// (dginit_known: g . s when the caller has it already, else NaN)
void cvsrch(const LbfgsCtx& c, const DevBuf& wa, double& f, DevBuf& g, double& stp, const DevBuf& s, double tolf,
            double dginit_known) {
    int infoc = 1;
    const double xtol = 1e-15, ftol = 1.0e-4, gtol = 0.9, eps = tolf;
    const double stpmin = 1e-15, stpmax = 1e15, xtrapf = 4;
    const int maxfev = 20;
    int nfev = 0;
    const double dginit = std::isnan(dginit_known) ? c.dot(g, s) : dginit_known;
    if (dginit >= 0.0) return;  // no descent
    bool brackt = false, stage1 = true;
    const double finit = f, dgtest = ftol * dginit;
    double width = stpmax - stpmin, width1 = 2 * width;
    double stx = 0.0, fx = finit, dgx = dginit, sty = 0.0, fy = finit, dgy = dginit;
    double stmin = 0, stmax = 0;
    StateD& S = c.st->s;
    while (true) {
        if (brackt) {
            stmin = std::min(stx, sty);
            stmax = std::max(stx, sty);
        } else {
            stmin = stx;
            stmax = stp + xtrapf * (stp - stx);
        }
        stp = std::max(stp, stpmin);
        stp = std::min(stp, stpmax);
        if ((brackt && ((stp <= stmin) || (stp >= stmax))) || (nfev >= maxfev - 1) || (infoc == 0) ||
            (brackt && (stmax - stmin <= xtol * stmax)))
            stp = stx;
        normalize_combine(S.m64.as<double>(), wa.as<double>(), stp, s.as<double>(), S.md.N(), c.stream);
        c.st->m32_valid = false;
        double dg;
        lbfgs_egrad_dg(c, g, s, f, dg);
        nfev++;
        const double ftest1 = finit + stp * dgtest;
        const double ftest2 = finit + eps * std::fabs(finit);
        const double ft = 2 * ftol - 1;
        int info = 0;
        if ((brackt && ((stp <= stmin) || (stp >= stmax))) || (infoc == 0)) info = 6;
        if ((stp == stpmax) && (f <= ftest2) && (dg <= dgtest)) info = 5;
        if ((stp == stpmin) && ((f > ftest2) || (dg >= dgtest))) info = 4;
        if (nfev >= maxfev) info = 3;
        if (brackt && (stmax - stmin <= xtol * stmax)) info = 2;
        if ((f <= ftest1) && (std::fabs(dg) <= gtol * (-dginit))) info = 1;
        if (((f <= ftest2) && (ft * dginit >= dg)) && (std::fabs(dg) <= gtol * (-dginit))) info = 1;
        if (info != 0) return;
        if (stage1 && ((f <= ftest2) && (ft * dginit >= dg)) && (dg >= std::min(ftol, gtol) * dginit)) stage1 = false;
        if (stage1 && (f <= fx) && !((f <= ftest2) && (ft * dginit >= dg))) {
            const double fm = f - stp * dgtest;
            double fxm = fx - stx * dgtest, fym = fy - sty * dgtest;
            const double dgm = dg - dgtest;
            double dgxm = dgx - dgtest, dgym = dgy - dgtest;
            cstep(stx, fxm, dgxm, sty, fym, dgym, stp, fm, dgm, brackt, stmin, stmax, infoc);
            fx = fxm + stx * dgtest;
            fy = fym + sty * dgtest;
            dgx = dgxm + dgtest;
            dgy = dgym + dgtest;
        } else {
            cstep(stx, fx, dgx, sty, fy, dgy, stp, f, dg, brackt, stmin, stmax, infoc);
        }
        if (brackt) {
            if (std::fabs(sty - stx) >= 0.66 * width1) stp = stx + 0.5 * (sty - stx);
            width1 = width;
            width = std::fabs(sty - stx);
        }
    }
}

// LBFGS_Minimizer::Minimize (lbfgs_minimizer.cpp:55-198)
double lbfgs_minimize(maf_lbfgs_s* h, maf_state_s* st) {
    StateD& S = st->s;
    const int64_t n3 = 3 * S.md.N();
    for (auto* b : {&h->q, &h->s, &h->y, &h->grad, &h->grad_old, &h->x_old}) b->ensure(sizeof(double) * n3);
    for (int i = 0; i < 5; ++i) {
        h->sV[i].ensure(sizeof(double) * n3);
        h->yV[i].ensure(sizeof(double) * n3);
    }
    h->red.ensure(sizeof(double) * (red_blocks() + 8));
    h->coef.ensure(sizeof(double) * 10);
    double* alpha_d = h->coef.as<double>();  // alpha[0..4]
    double* dot_d = alpha_d + 5;             // the dot product of the current recursion step
    double* trio_d = alpha_d + 6;            // up to three reductions read back with one synchronisation
    auto read_back = [&](int k, double* out) {
        MAF_CUDA(cudaMemcpyAsync(out, trio_d, sizeof(double) * k, cudaMemcpyDeviceToHost, S.stream));
        MAF_CUDA(cudaStreamSynchronize(S.stream));
    };
    LbfgsCtx c{h, st, n3, S.md.N(), S.stream};
    const double eps = 2.22e-16, eps2 = std::sqrt(eps), epsr = std::pow(eps, 0.9);
    const double tolf2 = std::sqrt(h->tolerance), tolf3 = std::pow(h->tolerance, 0.3333333333333333333333333);
    double f = lbfgs_egrad(c, h->grad);
    double gradNorm = c.maxabs(h->grad.as<double>());
    h->iterations = 0;
    h->last_gradnorm = gradNorm;
    if (gradNorm < (epsr * (1 + std::fabs(f)))) return f;
    const size_t m = 5;
    size_t iter = 0, globIter = 0;
    double H0k = 1;
    int order[5] = {0, 1, 2, 3, 4};  // logical slot -> buffer (std::rotate of the reference)
    do {
        const double f_old = f;
        MAF_CUDA(cudaMemcpyAsync(h->x_old.p, S.m64.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
        MAF_CUDA(cudaMemcpyAsync(h->grad_old.p, h->grad.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
        MAF_CUDA(cudaMemcpyAsync(h->q.p, h->grad.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
        const int k = (int)std::min(m, iter);
        // the two-loop recursion stays on the device: alpha_i = rho_i (s_i . q) and
        // beta = rho_i (y_i . q) are formed by the kernels that use them, with the
        // reference's operations in its order (rho_i = 1 / (s_i . y_i) is kept from when
        // the pair was stored: the same value as recomputing it); no host synchronisation
        for (int i = k - 1; i >= 0; --i) {
            const DevBuf& sv = h->sV[order[i]];
            const DevBuf& yv = h->yV[order[i]];
            dot_dev(sv.as<double>(), h->q.as<double>(), n3, c.red(), dot_d, S.stream);
            axpby_rho(h->q.as<double>(), yv.as<double>(), dot_d, h->rho[order[i]], nullptr, alpha_d + i, n3,
                      S.stream);
        }
        axpby(h->q.as<double>(), H0k, h->q.as<double>(), 0.0, nullptr, n3, S.stream);
        for (int i = 0; i < k; ++i) {
            const DevBuf& sv = h->sV[order[i]];
            const DevBuf& yv = h->yV[order[i]];
            dot_dev(yv.as<double>(), h->q.as<double>(), n3, c.red(), dot_d, S.stream);
            axpby_rho(h->q.as<double>(), sv.as<double>(), dot_d, h->rho[order[i]], alpha_d + i, nullptr, n3,
                      S.stream);
        }
        const double phiPrime0 = -c.dot(h->grad, h->q);
        if (phiPrime0 > 0) {
            MAF_CUDA(cudaMemcpyAsync(h->q.p, h->grad.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
            iter = 0;
        }
        // search direction -q (held in s until the step is known)
        axpby(h->s.as<double>(), -1.0, h->q.as<double>(), 0.0, nullptr, n3, S.stream);
        double rate = 1.0;
        // with s = -q exactly (a negation), grad . s = -(grad . q) = phiPrime0 to the bit
        cvsrch(c, h->x_old, f, h->grad, rate, h->s, h->tolerance,
               phiPrime0 > 0 ? std::numeric_limits<double>::quiet_NaN() : phiPrime0);
        const double f1 = 1 + std::fabs(f);
        // max|grad|, and ahead of the convergence test the step s = m - x_old with
        // max|s| and max|m| (unused if the gradient test ends the run): one synchronisation
        axpby(h->s.as<double>(), 1.0, S.m64.as<double>(), -1.0, h->x_old.as<double>(), n3, S.stream);
        double mx[3];
        reduce_dev(h->grad.as<double>(), nullptr, n3, 1, c.red(), trio_d, S.stream);
        reduce_dev(h->s.as<double>(), nullptr, n3, 1, c.red(), trio_d + 1, S.stream);
        reduce_dev(S.m64.as<double>(), nullptr, n3, 1, c.red(), trio_d + 2, S.stream);
        read_back(3, mx);
        gradNorm = mx[0];
        h->last_gradnorm = gradNorm;
        if (gradNorm < (epsr * f1)) {
            h->iterations = globIter;
            return f;
        }
        const double smax = mx[1], mmax = mx[2];
        if (((f_old - f) < (h->tolerance * f1)) && (smax < (tolf2 * (1 + mmax))) && (gradNorm <= (tolf3 * f1))) break;
        axpby(h->y.as<double>(), 1.0, h->grad.as<double>(), -1.0, h->grad_old.as<double>(), n3, S.stream);
        double d3[3];
        dot_dev(h->y.as<double>(), h->s.as<double>(), n3, c.red(), trio_d, S.stream);
        dot_dev(h->y.as<double>(), h->y.as<double>(), n3, c.red(), trio_d + 1, S.stream);
        dot_dev(h->s.as<double>(), h->s.as<double>(), n3, c.red(), trio_d + 2, S.stream);
        read_back(3, d3);
        const double ys = d3[0], yy = d3[1];
        if (ys <= eps2 * std::sqrt(yy) * std::sqrt(d3[2])) {
            // Dennis, Schnabel 9.4.1: skip the update
        } else {
            int slot;
            if (iter < m) {
                slot = order[iter];
            } else {
                const int first = order[0];
                for (int i = 0; i < 4; ++i) order[i] = order[i + 1];
                order[4] = first;
                slot = first;
            }
            MAF_CUDA(cudaMemcpyAsync(h->sV[slot].p, h->s.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
            MAF_CUDA(cudaMemcpyAsync(h->yV[slot].p, h->y.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
            h->rho[slot] = 1.0 / ys;  // = 1 / (s . y): the products commute exactly, same partial-sum order
            H0k = ys / yy;
            iter++;
        }
        globIter++;
    } while (globIter < h->maxIter);
    h->iterations = globIter;
    return f;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* maf_last_error(void) { return g_last_error.c_str(); }

int maf_version(int* major, int* minor) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    return MAF_OK;
}

int maf_device_count(int* n) {
    return guarded([&] {
        int c = 0;
        if (cudaGetDeviceCount(&c) != cudaSuccess) {
            cudaGetLastError();
            c = 0;
        }
        *n = c;
    });
}

// ------------------------------------------------------------------ state
int maf_state_create(maf_state* out, int nx, int ny, int nz, double dx, double dy, double dz, double Ms,
                     const double* Ms_field_host, const double* m_host, int precision) {
    return guarded([&] {
        check(out && m_host, "maf_state_create: NULL argument");
        check(nx > 0 && ny > 0 && nz > 0, "maf_state_create: mesh sizes must be positive");
        check(precision == MAF_FP64 || precision == MAF_FP32_FIELD, "maf_state_create: bad precision");
        require_device();
        noalloc_prepare_current_device();
        auto h = std::make_unique<maf_state_s>();
        StateD& s = h->s;
        s.md = MeshDims{nx, ny, nz, dx, dy, dz};
        s.precision = precision;
        MAF_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        s.own_stream = true;
        const int64_t N = s.md.N();
        upload(s.m64, m_host, 3 * N, s.stream);
        // normalize (state.cpp:92) and count zero-norm cells
        h->scratch.ensure(sizeof(unsigned long long) * 2);
        MAF_CUDA(cudaMemsetAsync(h->scratch.p, 0, sizeof(unsigned long long), s.stream));
        normalize_m(s.m64.as<double>(), N, 2, h->scratch.as<unsigned long long>(), s.stream);
        unsigned long long zeros = 0;
        MAF_CUDA(cudaMemcpyAsync(&zeros, h->scratch.p, sizeof(zeros), cudaMemcpyDeviceToHost, s.stream));
        MAF_CUDA(cudaStreamSynchronize(s.stream));
        if (Ms_field_host) {
            s.Ms = std::numeric_limits<double>::quiet_NaN();
            s.has_Ms_field = true;
            upload(s.Msf64, Ms_field_host, N, s.stream);
        } else {
            s.Ms = Ms;
            if (zeros > 0) {
                s.has_Ms_field = true;
                s.Msf64.alloc(sizeof(double) * N);
            }
        }
        if (s.has_Ms_field) {
            if (precision == PREC_FP32_FIELD) s.Msf32.alloc(sizeof(float) * N);
            if (!Ms_field_host) {
                ms_field_from_m(s.m64.as<double>(), Ms, s.Msf64.as<double>(),
                                precision == PREC_FP32_FIELD ? s.Msf32.as<float>() : nullptr, N, s.stream);
            } else if (precision == PREC_FP32_FIELD) {
                stage_m32(s.Msf64.as<double>(), s.Msf32.as<float>(), N, s.stream);
            }
            MAF_CUDA(cudaStreamSynchronize(s.stream));
        }
        *out = h.release();
    });
}

int maf_state_destroy(maf_state s) {
    return guarded([&] { delete s; });
}

int maf_state_get_m(maf_state st, double* m_host) {
    return guarded([&] {
        check(st && m_host, "NULL argument");
        StateD& s = st->s;
        MAF_CUDA(cudaMemcpyAsync(m_host, s.m64.p, sizeof(double) * 3 * s.md.N(), cudaMemcpyDeviceToHost, s.stream));
        MAF_CUDA(cudaStreamSynchronize(s.stream));
    });
}

int maf_state_set_m(maf_state st, const double* m_host) {
    return guarded([&] {
        check(st && m_host, "NULL argument");
        StateD& s = st->s;
        MAF_CUDA(cudaMemcpyAsync(s.m64.p, m_host, sizeof(double) * 3 * s.md.N(), cudaMemcpyHostToDevice, s.stream));
        normalize_m(s.m64.as<double>(), s.md.N(), 2, nullptr, s.stream);
        st->m32_valid = false;
    });
}

int maf_state_load_m(maf_state st, const double* m_host) {
    return guarded([&] {
        check(st && m_host, "NULL argument");
        StateD& s = st->s;
        MAF_CUDA(cudaMemcpyAsync(s.m64.p, m_host, sizeof(double) * 3 * s.md.N(), cudaMemcpyHostToDevice, s.stream));
        MAF_CUDA(cudaStreamSynchronize(s.stream));
        st->m32_valid = false;
    });
}

int maf_state_get_t(maf_state st, double* t) {
    return guarded([&] { check(st && t, "NULL argument"); *t = st->s.t; });
}
int maf_state_set_t(maf_state st, double t) {
    return guarded([&] { check(st, "NULL argument"); st->s.t = t; });
}
int maf_state_get_steps(maf_state st, unsigned long long* steps) {
    return guarded([&] { check(st && steps, "NULL argument"); *steps = st->s.steps; });
}
int maf_state_mean_m(maf_state st, double out[3]) {
    return guarded([&] {
        check(st && out, "NULL argument");
        mean_m_host(st, st->s.m64.as<double>(), out);
    });
}
int maf_state_get_Ms_field(maf_state st, double* host, int* has_field) {
    return guarded([&] {
        check(st, "NULL argument");
        if (has_field) *has_field = st->s.has_Ms_field ? 1 : 0;
        if (host && st->s.has_Ms_field) {
            MAF_CUDA(cudaMemcpyAsync(host, st->s.Msf64.p, sizeof(double) * st->s.md.N(), cudaMemcpyDeviceToHost,
                                     st->s.stream));
            MAF_CUDA(cudaStreamSynchronize(st->s.stream));
        }
    });
}
int maf_state_get_Ms(maf_state st, double* Ms) {
    return guarded([&] { check(st && Ms, "NULL argument"); *Ms = st->s.Ms; });
}
int maf_state_set_stream(maf_state st, void* stream) {
    return guarded([&] {
        check(st, "NULL argument");
        MAF_CUDA(cudaStreamSynchronize(st->s.stream));
        if (stream) {
            if (st->s.own_stream) cudaStreamDestroy(st->s.stream);
            st->s.own_stream = false;
            st->s.stream = static_cast<cudaStream_t>(stream);
        } else if (!st->s.own_stream) {
            MAF_CUDA(cudaStreamCreateWithFlags(&st->s.stream, cudaStreamNonBlocking));
            st->s.own_stream = true;
        }
    });
}
int maf_state_device_m(maf_state st, void** p) {
    return guarded([&] { check(st && p, "NULL argument"); *p = st->s.m64.p; });
}
int maf_state_precision(maf_state st, int* p) {
    return guarded([&] { check(st && p, "NULL argument"); *p = st->s.precision; });
}

// ------------------------------------------------------------------ terms
static maf_term new_term(std::shared_ptr<Term> t) {
    auto* h = new maf_term_s;
    h->t = std::move(t);
    return h;
}

static int demag_create(maf_term* out, int nx, int ny, int nz, double dx, double dy, double dz,
                        const double* tensor_host) {
    return guarded([&] {
        check(out, "NULL argument");
        check(nx > 0 && ny > 0 && nz > 0 && dx > 0 && dy > 0 && dz > 0, "DemagField: invalid mesh");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_DEMAG;
        t->demag_mesh = MeshDims{nx, ny, nz, dx, dy, dz};
        cudaStream_t st;
        MAF_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        try {
            t->demag = std::make_unique<Demag>(t->demag_mesh, st, tensor_host);
        } catch (...) {
            cudaStreamDestroy(st);
            throw;
        }
        MAF_CUDA(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        *out = new_term(t);
    });
}

int maf_term_demag_create(maf_term* out, int nx, int ny, int nz, double dx, double dy, double dz) {
    return demag_create(out, nx, ny, nz, dx, dy, dz, nullptr);
}

int maf_term_demag_create_from_tensor(maf_term* out, int nx, int ny, int nz, double dx, double dy, double dz,
                                      const double* tensor_host) {
    if (!tensor_host) return fail(MAF_ERR_BADARG, "maf_term_demag_create_from_tensor: NULL tensor");
    return demag_create(out, nx, ny, nz, dx, dy, dz, tensor_host);
}

int maf_term_demag_pbc_create(maf_term* out) {
    return guarded([&] {
        check(out, "NULL argument");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_DEMAG;
        t->p[0] = 1.0;  // periodic form; the plan is made for the first state evaluated
        *out = new_term(t);
    });
}

int maf_term_exchange_create(maf_term* out, double A) {
    return guarded([&] {
        check(out, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_EXCHANGE;
        t->p[0] = A;
        *out = new_term(t);
    });
}

static void set_unit_axis(double* dst, double x, double y, double z, const char* who) {
    const double n = std::sqrt(x * x + y * y + z * z);
    check(n > 0, std::string(who) + ": zero axis");
    dst[0] = x / n;
    dst[1] = y / n;
    dst[2] = z / n;
}

int maf_term_dmi_create(maf_term* out, double D, double ax, double ay, double az) {
    return guarded([&] {
        check(out, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_DMI;
        t->p[0] = D;
        // dmi_field.cpp:43-47: n = D_axis / |D_axis|
        const double norm = std::sqrt(std::pow(ax, 2) + std::pow(ay, 2) + std::pow(az, 2));
        check(norm > 0, "DmiField: zero axis");
        t->p[1] = ax / norm;
        t->p[2] = ay / norm;
        t->p[3] = az / norm;
        *out = new_term(t);
    });
}

int maf_term_dmi_field_create(maf_term* out, int nx, int ny, int nz, const double* D_field, double ax, double ay,
                              double az) {
    return guarded([&] {
        check(out && D_field, "NULL argument");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_DMI;
        const double norm = std::sqrt(std::pow(ax, 2) + std::pow(ay, 2) + std::pow(az, 2));
        check(norm > 0, "DmiField: zero axis");
        t->p[1] = ax / norm;
        t->p[2] = ay / norm;
        t->p[3] = az / norm;
        upload(t->f0, D_field, (size_t)nx * ny * nz, 0);
        t->field_cells = (int64_t)nx * ny * nz;
        t->demag_mesh = MeshDims{nx, ny, nz, 0, 0, 0};
        *out = new_term(t);
    });
}

int maf_term_bulkdmi_exchange_create(maf_term* out, double D, double A) {
    return guarded([&] {
        check(out, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_BULKDMI;
        t->p[0] = D;
        t->p[1] = A;
        *out = new_term(t);
    });
}

int maf_term_uniaxial_create(maf_term* out, double Ku1, double ax, double ay, double az) {
    return guarded([&] {
        check(out, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_UNIAXIAL;
        t->p[0] = Ku1;
        set_unit_axis(t->p + 1, ax, ay, az, "UniaxialAnisotropyField");  // util::normalize_vector
        *out = new_term(t);
    });
}

int maf_term_uniaxial_field_create(maf_term* out, int nx, int ny, int nz, const double* Ku1_field, double Ku1,
                                   const double* axis_field, double ax, double ay, double az) {
    return guarded([&] {
        check(out, "NULL argument");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_UNIAXIAL;
        t->p[0] = Ku1;
        const size_t N = (size_t)nx * ny * nz;
        if (Ku1_field) upload(t->f0, Ku1_field, N, 0);
        if (Ku1_field || axis_field) t->field_cells = (int64_t)N;
        if (axis_field) {
            // util::normalize on the axis field (uniaxial_anisotropy_field.cpp:24)
            upload(t->f1, axis_field, 3 * N, 0);
            normalize_m(t->f1.as<double>(), (int64_t)N, 2, nullptr, 0);
            MAF_CUDA(cudaDeviceSynchronize());
        } else {
            set_unit_axis(t->p + 1, ax, ay, az, "UniaxialAnisotropyField");
        }
        *out = new_term(t);
    });
}

int maf_term_stt_create(maf_term* out, int nx, int ny, int nz, const double* polarization_host, double eta_damping,
                        double eta_field, double j_e, double fl_thickness) {
    return guarded([&] {
        check(out && polarization_host, "NULL argument");
        check(nx > 0 && ny > 0 && nz > 0 && fl_thickness > 0, "SpinTransferTorqueField: bad argument");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_STT;
        t->p[0] = -j_e * kHbar / (2. * kEneg * kMu0 * fl_thickness);
        t->p[1] = eta_damping;
        t->p[2] = eta_field;
        const size_t N = (size_t)nx * ny * nz;
        // util::normalize of the polarisation (spin_transfer_torque_field.cpp:9)
        upload(t->f1, polarization_host, 3 * N, 0);
        t->field_cells = (int64_t)N;
        normalize_m(t->f1.as<double>(), (int64_t)N, 2, nullptr, 0);
        MAF_CUDA(cudaDeviceSynchronize());
        *out = new_term(t);
    });
}

// SparseExchangeField and ExchangeFieldPBC: the matrix is not stored; the kernel
// forms each row's weights from A (or the A field) as the assembly does.
static int sparse_exchange_create(maf_term* out, int nx, int ny, int nz, const double* A_field, double A,
                                  bool periodic, const char* who) {
    return guarded([&] {
        check(out, "NULL argument");
        check(nx > 0 && ny > 0 && nz > 0, std::string(who) + ": bad mesh");
        require_device();
        auto t = std::make_shared<Term>();
        t->kind = TK_SPARSE_EXCH;
        t->p[0] = A;
        t->p[1] = periodic ? 1.0 : 0.0;
        const size_t N = (size_t)nx * ny * nz;
        if (A_field) upload(t->f0, A_field, N, 0);
        t->field_cells = (int64_t)N;  // the matrix is built for this mesh
        *out = new_term(t);
    });
}

int maf_term_sparse_exchange_create(maf_term* out, int nx, int ny, int nz, const double* A_field_host, double A) {
    return sparse_exchange_create(out, nx, ny, nz, A_field_host, A, false, "SparseExchangeField");
}

int maf_term_exchange_pbc_create(maf_term* out, int nx, int ny, int nz, const double* A_field_host, double A) {
    return sparse_exchange_create(out, nx, ny, nz, A_field_host, A, true, "ExchangeFieldPBC");
}

int maf_term_cubic_create(maf_term* out, double Kc1, double Kc2, double Kc3, const double c1[3], const double c2[3]) {
    return guarded([&] {
        check(out && c1 && c2, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_CUBIC;
        t->p[0] = Kc1;
        t->p[1] = Kc2;
        t->p[2] = Kc3;
        double a[3], b[3];
        set_unit_axis(a, c1[0], c1[1], c1[2], "CubicAnisotropyField c1");
        set_unit_axis(b, c2[0], c2[1], c2[2], "CubicAnisotropyField c2");
        const double dot = std::fabs(a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
        check(dot <= 1e-12, "CubicAnisotropyField: provided c1 and c2 are not perpendicular, |c1.c2| = " +
                                std::to_string(dot));
        // c3 = normalize(c1 x c2), cross product of the given (unnormalised) axes
        const double cx = c1[1] * c2[2] - c1[2] * c2[1];
        const double cy = c1[2] * c2[0] - c1[0] * c2[2];
        const double cz = c1[0] * c2[1] - c1[1] * c2[0];
        double c[3];
        set_unit_axis(c, cx, cy, cz, "CubicAnisotropyField c3");
        for (int i = 0; i < 3; ++i) {
            t->p[3 + i] = a[i];
            t->p[6 + i] = b[i];
            t->p[9 + i] = c[i];
        }
        *out = new_term(t);
    });
}

int maf_term_external_create(maf_term* out, int nx, int ny, int nz, const double* h_host) {
    return guarded([&] {
        check(out && h_host, "NULL argument");
        const size_t N = (size_t)nx * ny * nz;
        auto t = std::make_shared<Term>();
        t->kind = TK_ZEEMAN;
        // a field that is the same in every cell is kept as one vector
        bool uniform = true;
        for (int c = 0; c < 3 && uniform; ++c)
            for (size_t i = 1; i < N; ++i)
                if (h_host[c * N + i] != h_host[c * N]) { uniform = false; break; }
        if (uniform) {
            t->p[0] = h_host[0];
            t->p[1] = h_host[N];
            t->p[2] = h_host[2 * N];
        } else {
            require_device();
            upload(t->f0, h_host, 3 * N, 0);
            t->field_cells = (int64_t)N;
        }
        t->demag_mesh = MeshDims{nx, ny, nz, 0, 0, 0};
        *out = new_term(t);
    });
}

int maf_term_external_uniform_create(maf_term* out, double hx, double hy, double hz) {
    return guarded([&] {
        check(out, "NULL argument");
        auto t = std::make_shared<Term>();
        t->kind = TK_ZEEMAN;
        t->p[0] = hx;
        t->p[1] = hy;
        t->p[2] = hz;
        *out = new_term(t);
    });
}

int maf_term_destroy(maf_term t) {
    return guarded([&] { delete t; });
}

static void check_term_state(maf_term t, maf_state s) {
    check(t && s, "NULL argument");
    check(t->t->field_cells == 0 || t->t->field_cells == s->s.md.N(),
          "field-term parameter array does not match the state's mesh");
}

int maf_term_H(maf_term t, maf_state s, double* H) {
    return guarded([&] {
        check_term_state(t, s);
        check(H, "NULL argument");
        H_to_host(s, {t->t.get()}, H, nullptr, g_tmp);
    });
}

int maf_term_H_f32(maf_term t, maf_state s, float* H) {
    return guarded([&] {
        check_term_state(t, s);
        check(H, "NULL argument");
        H_to_host(s, {t->t.get()}, nullptr, H, g_tmp);
    });
}

int maf_term_E(maf_term t, maf_state s, double* E) {
    return guarded([&] {
        check_term_state(t, s);
        check(E, "NULL argument");
        EpilogueArgs ep;
        ep.kind = EPI_EDENS;
        eval_on_state(s, {t->t.get()}, ep, E);
    });
}

int maf_term_demag_tensor(maf_term t, double* host) {
    return guarded([&] {
        check(t && host && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_tensor: not a DemagField");
        t->t->demag->download_tensor(host, 0);
    });
}

int maf_term_demag_real_tensor(maf_term t, double* host, int symmetric) {
    return guarded([&] {
        check(t && host && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_real_tensor: not a DemagField");
        t->t->demag->download_real_tensor(host, symmetric != 0, 0);
    });
}

// ------------------------------------------------------------------ LLG
int maf_llg_create(maf_llg* out, double alpha, const double* alpha_field, int nx, int ny, int nz, const maf_term* terms,
                   int nterms, const char* scheme, double hmin, double hmax, double atol, double rtol,
                   int dissipation_term_only) {
    return guarded([&] {
        check(out, "NULL argument");
        check(nterms >= 0 && (nterms == 0 || terms), "maf_llg_create: bad term list");
        auto l = std::make_unique<maf_llg_s>();
        l->alpha = alpha;
        if (alpha_field) {
            require_device();
            upload(l->alpha_field, alpha_field, (size_t)nx * ny * nz, 0);
            l->has_alpha_field = true;
            l->alpha_n = nx * ny * nz;
        }
        for (int i = 0; i < nterms; ++i) {
            check(terms[i] != nullptr, "maf_llg_create: NULL term");
            l->terms.push_back(terms[i]->t);
        }
        l->scheme_name = scheme ? scheme : "RKF45";
        l->scheme = make_scheme(l->scheme_name);
        l->ctrl.hmin = hmin;
        l->ctrl.hmax = hmax;
        l->ctrl.atol = atol;
        l->ctrl.rtol = rtol;
        l->dissipation_only = dissipation_term_only != 0;
        *out = l.release();
    });
}

int maf_llg_destroy(maf_llg l) {
    return guarded([&] { delete l; });
}

int maf_llg_add_term(maf_llg l, maf_term t) {
    return guarded([&] {
        check(l && t, "NULL argument");
        l->terms.push_back(t->t);
    });
}

int maf_llg_set_alpha(maf_llg l, double alpha) {
    return guarded([&] {
        check(l, "NULL argument");
        l->alpha = alpha;
    });
}

static void check_llg_state(maf_llg l, maf_state s) {
    check(l && s, "NULL argument");
    check(!l->terms.empty(), "LLGIntegrator: no field terms");
    if (l->has_alpha_field) check(l->alpha_n == s->s.md.N(), "alpha field does not match the state's mesh");
}

int maf_llg_step(maf_llg l, maf_state s) {
    return guarded([&] {
        check_llg_state(l, s);
        llg_step(l, s);
    });
}

int maf_llg_steps(maf_llg l, maf_state s, int n) {
    return guarded([&] {
        check_llg_state(l, s);
        for (int i = 0; i < n; ++i) llg_step(l, s);
    });
}

int maf_llg_E(maf_llg l, maf_state s, double* E) {
    return guarded([&] {
        check_llg_state(l, s);
        check(E, "NULL argument");
        *E = llg_energy(l, s);
    });
}

int maf_llg_heff(maf_llg l, maf_state s, double* H) {
    return guarded([&] {
        check_llg_state(l, s);
        check(H, "NULL argument");
        H_to_host(s, raw_terms(l->terms), H, nullptr, g_tmp);
    });
}

int maf_llg_heff_f32(maf_llg l, maf_state s, float* H) {
    return guarded([&] {
        check_llg_state(l, s);
        check(H, "NULL argument");
        H_to_host(s, raw_terms(l->terms), nullptr, H, g_tmp);
    });
}

// H_eff of n magnetisations in a row through pinned host memory: the copy of
// m[i+1] to the device, the evaluation of m[i] and the copy of H[i-1] to the
// host run on three streams with double-buffered device buffers, so the host
// link carries both directions while the field is computed.
// m_host holds FP64 inputs, or FP32 inputs when m_f32 (widened on the device,
// exactly, before the same normalisation).
static void heff_pipeline(maf_llg l, maf_state s, const void* const* m_host, bool m_f32, void* const* H_host, int n) {
    {
        check_llg_state(l, s);
        check(n >= 0 && (n == 0 || (m_host && H_host)), "maf_llg_heff_pipeline: bad argument");
        StateD& st = s->s;
        const int64_t N = st.md.N(), n3 = 3 * N;
        const bool f32 = st.precision == PREC_FP32_FIELD;
        const size_t hsz = (f32 ? sizeof(float) : sizeof(double)) * n3;
        if (!s->pipe) {
            auto p = std::make_unique<HeffPipe>();
            MAF_CUDA(cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
            MAF_CUDA(cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking));
            for (int b = 0; b < 2; ++b) {
                MAF_CUDA(cudaEventCreateWithFlags(&p->up_done[b], cudaEventDisableTiming));
                MAF_CUDA(cudaEventCreateWithFlags(&p->comp_done[b], cudaEventDisableTiming));
                MAF_CUDA(cudaEventCreateWithFlags(&p->down_done[b], cudaEventDisableTiming));
                p->m[b].alloc(sizeof(double) * n3);
                p->h[b].alloc(hsz);
            }
            if (f32) p->m32.alloc(sizeof(float) * n3);
            s->pipe = std::move(p);
        }
        HeffPipe& p = *s->pipe;
        if (m_f32)
            for (int b = 0; b < 2; ++b) p.m_in32[b].ensure(sizeof(float) * n3);
        const auto terms = raw_terms(l->terms);
        MAF_CUDA(cudaStreamSynchronize(st.stream));
        for (int i = 0; i < n; ++i) {
            const int b = i & 1;
            check(m_host[i] && H_host[i], "maf_llg_heff_pipeline: NULL buffer");
            // host -> device, once the evaluation two steps back has released m[b]
            MAF_CUDA(cudaStreamWaitEvent(p.up, p.comp_done[b], 0));
            if (m_f32)
                MAF_CUDA(cudaMemcpyAsync(p.m_in32[b].p, m_host[i], sizeof(float) * n3, cudaMemcpyHostToDevice, p.up));
            else
                MAF_CUDA(cudaMemcpyAsync(p.m[b].p, m_host[i], sizeof(double) * n3, cudaMemcpyHostToDevice, p.up));
            MAF_CUDA(cudaEventRecord(p.up_done[b], p.up));
            // normalise (as maf_state_set_m) and evaluate once H[b] has gone to the host
            MAF_CUDA(cudaStreamWaitEvent(st.stream, p.up_done[b], 0));
            MAF_CUDA(cudaStreamWaitEvent(st.stream, p.down_done[b], 0));
            if (m_f32) widen_m(p.m_in32[b].as<float>(), p.m[b].as<double>(), n3, st.stream);
            normalize_m(p.m[b].as<double>(), N, 2, nullptr, st.stream);
            EpilogueArgs ep;
            ep.kind = EPI_H;
            ep.out = p.h[b].p;
            if (f32) {
                stage_m32(p.m[b].as<double>(), p.m32.as<float>(), n3, st.stream);
                eval_terms<float>(terms, st.md, p.m32.as<float>(), st.msinfo(), ep, st.stream, s->scratch, nullptr);
            } else {
                eval_terms<double>(terms, st.md, p.m[b].as<double>(), st.msinfo(), ep, st.stream, s->scratch,
                                   nullptr);
            }
            MAF_CUDA(cudaEventRecord(p.comp_done[b], st.stream));
            // device -> host
            MAF_CUDA(cudaStreamWaitEvent(p.down, p.comp_done[b], 0));
            MAF_CUDA(cudaMemcpyAsync(H_host[i], p.h[b].p, hsz, cudaMemcpyDeviceToHost, p.down));
            MAF_CUDA(cudaEventRecord(p.down_done[b], p.down));
        }
        if (n > 0) {  // the state keeps the last magnetisation, as after maf_state_set_m
            MAF_CUDA(cudaMemcpyAsync(st.m64.p, p.m[(n - 1) & 1].p, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                                     st.stream));
            s->m32_valid = false;
        }
        MAF_CUDA(cudaStreamSynchronize(p.down));
        MAF_CUDA(cudaStreamSynchronize(p.up));
        MAF_CUDA(cudaStreamSynchronize(st.stream));
    }
}

int maf_llg_heff_pipeline(maf_llg l, maf_state s, const double* const* m_host, void* const* H_host, int n) {
    return guarded([&] { heff_pipeline(l, s, reinterpret_cast<const void* const*>(m_host), false, H_host, n); });
}

int maf_llg_heff_pipeline_m32(maf_llg l, maf_state s, const float* const* m_host, void* const* H_host, int n) {
    return guarded([&] { heff_pipeline(l, s, reinterpret_cast<const void* const*>(m_host), true, H_host, n); });
}

int maf_llg_heff_device(maf_llg l, maf_state s, const void* m_dev, void* H_dev) {
    return guarded([&] {
        check_llg_state(l, s);
        check(m_dev && H_dev, "NULL argument");
        EpilogueArgs ep;
        ep.kind = EPI_H;
        ep.out = H_dev;
        StateD& st = s->s;
        if (st.precision == PREC_FP32_FIELD)
            eval_terms<float>(raw_terms(l->terms), st.md, static_cast<const float*>(m_dev), st.msinfo(), ep, st.stream,
                              s->scratch, nullptr);
        else
            eval_terms<double>(raw_terms(l->terms), st.md, static_cast<const double*>(m_dev), st.msinfo(), ep,
                               st.stream, s->scratch, nullptr);
    });
}

int maf_llg_heff_device_profile(maf_llg l, maf_state s, const void* m_dev, void* H_dev, double* pass_ms,
                                int max_passes, int* npasses) {
    return guarded([&] {
        check_llg_state(l, s);
        check(m_dev && H_dev && pass_ms && npasses, "NULL argument");
        EpilogueArgs ep;
        ep.kind = EPI_H;
        ep.out = H_dev;
        StateD& st = s->s;
        PassMarks marks;
        if (st.precision == PREC_FP32_FIELD)
            eval_terms<float>(raw_terms(l->terms), st.md, static_cast<const float*>(m_dev), st.msinfo(), ep, st.stream,
                              s->scratch, nullptr, &marks);
        else
            eval_terms<double>(raw_terms(l->terms), st.md, static_cast<const double*>(m_dev), st.msinfo(), ep,
                               st.stream, s->scratch, nullptr, &marks);
        MAF_CUDA(cudaStreamSynchronize(st.stream));
        int n = 0;
        for (size_t i = 1; i < marks.ev.size() && n < max_passes; ++i, ++n) {
            float ms = 0;
            MAF_CUDA(cudaEventElapsedTime(&ms, marks.ev[i - 1], marks.ev[i]));
            pass_ms[n] = ms;
        }
        *npasses = n;
    });
}

// Autotuner: times both kernel configurations of every tunable pass on this
// state's mesh and precision (one warm-up, then the mean of `reps` evaluations
// with CUDA events between the passes) and keeps the faster variant per pass.
// Autotuner: times four kernel configurations of the demag passes on this
// state's mesh and precision (one warm-up, then the mean of `reps` evaluations
// with CUDA events between the passes) and keeps the fastest variant per pass:
// y passes (column tile x pipelining x radix sequence, chosen jointly since the
// two passes share the tile and the plan), z convolution, x-inverse epilogue run.
// The choices are cached per (mesh, precision, term kinds) for the process.
namespace {
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tune_cache;

std::string tune_key(const maf_llg_s* l, const StateD& st) {
    std::string k = std::to_string(st.md.nx) + "," + std::to_string(st.md.ny) + "," + std::to_string(st.md.nz) + "," +
                    std::to_string(st.md.dx) + "," + std::to_string(st.md.dy) + "," + std::to_string(st.md.dz) +
                    "," + std::to_string(st.precision) + ",";
    for (auto& t : l->terms) k += std::to_string(t->kind) + ":";
    return k;
}
}  // namespace

int maf_llg_autotune_ex(maf_llg l, maf_state s, int reps, int choices[5], double* pass_ms, int* cached) {
    return guarded([&] {
        check_llg_state(l, s);
        check(choices && reps > 0, "maf_llg_autotune: bad argument");
        Demag* dm = nullptr;
        for (auto& t : l->terms)
            if (t->kind == TK_DEMAG && !t->demag_pbc()) dm = t->demag.get();  // the periodic form has no variants
        TuneChoice best;
        if (cached) *cached = 0;
        if (dm) {
            StateD& st = s->s;
            const std::string key = tune_key(l, st);
            bool hit = false;
            {
                std::lock_guard<std::mutex> lock(g_tune_mu);
                auto it = g_tune_cache.find(key);
                if (it != g_tune_cache.end()) {
                    best = it->second;
                    best.generic = dm->tune.generic;
                    dm->tune = best;
                    hit = true;
                }
            }
            if (cached) *cached = hit ? 1 : 0;
            if (!hit) {
                const bool f32 = st.precision == PREC_FP32_FIELD;
                const int64_t n3 = 3 * st.md.N();
                g_tmp.ensure((f32 ? sizeof(float) : sizeof(double)) * n3);
                if (f32) ensure_m32(s);
                const auto terms = raw_terms(l->terms);
                const int generic = dm->tune.generic;
                auto run = [&](TuneChoice c) {
                    c.generic = generic;
                    dm->tune = c;
                    std::vector<double> acc;
                    for (int r = -1; r < reps; ++r) {  // r = -1: warm-up
                        EpilogueArgs ep;
                        ep.kind = EPI_H;
                        ep.out = g_tmp.p;
                        PassMarks marks;
                        if (f32)
                            eval_terms<float>(terms, st.md, st.m32.as<float>(), st.msinfo(), ep, st.stream, s->scratch,
                                              nullptr, &marks);
                        else
                            eval_terms<double>(terms, st.md, st.m64.as<double>(), st.msinfo(), ep, st.stream,
                                               s->scratch, nullptr, &marks);
                        MAF_CUDA(cudaStreamSynchronize(st.stream));
                        if (r < 0) continue;
                        acc.resize(marks.ev.size() - 1, 0.0);
                        for (size_t i = 1; i < marks.ev.size(); ++i) {
                            float ms = 0;
                            MAF_CUDA(cudaEventElapsedTime(&ms, marks.ev[i - 1], marks.ev[i]));
                            acc[i - 1] += ms / reps;
                        }
                    }
                    return acc;
                };
                //                    wide reg run pipe plan
                const TuneChoice cfg[4] = {{0, 1, 2, 1, 0}, {1, 0, 4, 0, 1}, {0, 1, 2, 0, 1}, {1, 0, 4, 1, 0}};
                std::vector<double> t[4];
                for (int c = 0; c < 4; ++c) t[c] = run(cfg[c]);
                best = cfg[0];
                if (st.md.nz > 1 && t[0].size() == 5) {
                    // y passes: per column tile width (shared by both passes), the fastest
                    // forward (pipelining, plan) and the fastest inverse plan among the
                    // configurations with that width; then the faster width
                    double best_y = 0;
                    for (int wide = 0; wide < 2; ++wide) {
                        int bf = -1, bi = -1;
                        for (int c = 0; c < 4; ++c) {
                            if (cfg[c].cols_wide != wide || t[c].size() != 5) continue;
                            if (bf < 0 || t[c][1] < t[bf][1]) bf = c;
                            if (bi < 0 || t[c][3] < t[bi][3]) bi = c;
                        }
                        if (bf < 0) continue;
                        const double ty = t[bf][1] + t[bi][3];
                        if (wide == 0 || ty < best_y) {
                            best_y = ty;
                            best.cols_wide = wide;
                            best.cols_pipe = cfg[bf].cols_pipe;
                            const bool pf = cfg[bf].cols_plan == 1, pi = cfg[bi].cols_plan == 1;
                            best.cols_plan = pf && pi ? 1 : pf ? 3 : pi ? 2 : 0;
                        }
                    }
                    best.convz_reg = (t[0][2] + t[2][2]) <= (t[1][2] + t[3][2]) ? 1 : 0;
                    best.xinv_run = (t[0][4] + t[2][4]) <= (t[1][4] + t[3][4]) ? 2 : 4;
                } else if (t[0].size() == 3) {
                    best.xinv_run = (t[0][2] + t[2][2]) <= (t[1][2] + t[3][2]) ? 2 : 4;
                }
                best.generic = generic;
                dm->tune = best;
                {
                    std::lock_guard<std::mutex> lock(g_tune_mu);
                    g_tune_cache[key] = best;
                }
                if (pass_ms)
                    for (int c = 0; c < 4; ++c)
                        for (size_t i = 0; i < 5; ++i) pass_ms[5 * c + i] = i < t[c].size() ? t[c][i] : 0.0;
            }
        }
        choices[0] = best.cols_wide;
        choices[1] = best.convz_reg;
        choices[2] = best.xinv_run;
        choices[3] = best.cols_pipe;
        choices[4] = best.cols_plan;
    });
}

int maf_llg_autotune(maf_llg l, maf_state s, int reps, int choices[3], double* pass_ms) {
    int c5[5];
    double ms[20];
    const int rc = maf_llg_autotune_ex(l, s, reps, c5, pass_ms ? ms : nullptr, nullptr);
    if (rc == 0) {
        for (int i = 0; i < 3; ++i) choices[i] = c5[i];
        if (pass_ms)
            for (int i = 0; i < 5; ++i) {  // the defaults and the all-alternative configuration
                pass_ms[i] = ms[i];
                pass_ms[5 + i] = ms[5 + i];
            }
    }
    return rc;
}

int maf_term_demag_get_tune_ex(maf_term t, int choices[5]) {
    return guarded([&] {
        check(t && choices && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_get_tune_ex: not a DemagField");
        const TuneChoice& c = t->t->demag->tune;
        choices[0] = c.cols_wide;
        choices[1] = c.convz_reg;
        choices[2] = c.xinv_run;
        choices[3] = c.cols_pipe;
        choices[4] = c.cols_plan;
    });
}

int maf_term_demag_set_tune_ex(maf_term t, const int choices[5]) {
    return guarded([&] {
        check(t && choices && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_set_tune_ex: not a DemagField");
        check((choices[0] == 0 || choices[0] == 1) && (choices[1] == 0 || choices[1] == 1) &&
                  (choices[2] == 0 || choices[2] == 2 || choices[2] == 4) && (choices[3] == 0 || choices[3] == 1) &&
                  (choices[4] >= 0 && choices[4] <= 3),
              "maf_term_demag_set_tune_ex: choices are {0|1, 0|1, 0|2|4, 0|1, 0..3}");
        TuneChoice& c = t->t->demag->tune;
        c.cols_wide = choices[0];
        c.convz_reg = choices[1];
        c.xinv_run = choices[2];
        c.cols_pipe = choices[3];
        c.cols_plan = choices[4];
    });
}

int maf_term_demag_get_tune(maf_term t, int choices[3]) {
    return guarded([&] {
        check(t && choices && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_get_tune: not a DemagField");
        const TuneChoice& c = t->t->demag->tune;
        choices[0] = c.cols_wide;
        choices[1] = c.convz_reg;
        choices[2] = c.xinv_run;
    });
}

int maf_term_demag_set_tune(maf_term t, const int choices[3]) {
    return guarded([&] {
        check(t && choices && t->t->kind == TK_DEMAG && !t->t->demag_pbc(),
              "maf_term_demag_set_tune: not a DemagField");
        check((choices[0] == 0 || choices[0] == 1) && (choices[1] == 0 || choices[1] == 1) &&
                  (choices[2] == 0 || choices[2] == 2 || choices[2] == 4),
              "maf_term_demag_set_tune: choices are {0|1, 0|1, 0|2|4}");
        TuneChoice& tc = t->t->demag->tune;
        tc.cols_wide = choices[0];
        tc.convz_reg = choices[1];
        tc.xinv_run = choices[2];
    });
}

int maf_term_demag_set_generic(maf_term t, int on) {
    return guarded([&] {
        check(t && t->t->kind == TK_DEMAG && t->t->demag && !t->t->demag_pbc(),
              "maf_term_demag_set_generic: not a DemagField");
        t->t->demag->tune.generic = on ? 1 : 0;
    });
}

// One Runge-Kutta attempt of the integrator's scheme with step dt on the state's
// m (the state is not changed), with CUDA events between its kernels: the
// conversion of m to FP32 (FP32-field form), each stage's combine and field
// passes, and the finalize (sumbk, error norm, candidate).
int maf_llg_attempt_profile(maf_llg l, maf_state s, double dt, double* ms_out, int max_entries, int* n_entries) {
    return guarded([&] {
        check_llg_state(l, s);
        check(ms_out && n_entries && max_entries > 0 && dt > 0, "maf_llg_attempt_profile: bad argument");
        const int norm_mode = s->s.has_Ms_field ? 2 : 1;
        s->m32_valid = false;  // a step starts from a new m: time its FP32 copy too
        PassMarks marks;
        rk_attempt(l, s, l->scheme, dt, norm_mode, &marks);
        MAF_CUDA(cudaStreamSynchronize(s->s.stream));
        l->prof_names.clear();
        int n = 0;
        for (size_t i = 1; i < marks.ev.size() && n < max_entries; ++i, ++n) {
            float ms = 0;
            MAF_CUDA(cudaEventElapsedTime(&ms, marks.ev[i - 1], marks.ev[i]));
            ms_out[n] = ms;
            l->prof_names.emplace_back(marks.names[i]);
        }
        *n_entries = n;
    });
}

int maf_llg_profile_name(maf_llg l, int index, char* buf, int buflen) {
    return guarded([&] {
        check(l && buf && buflen > 0, "NULL argument");
        check(index >= 0 && index < (int)l->prof_names.size(), "profile index out of range");
        std::snprintf(buf, (size_t)buflen, "%s", l->prof_names[(size_t)index].c_str());
    });
}

int maf_llg_pass_name(maf_llg l, maf_state s, int index, char* buf, int buflen) {
    return guarded([&] {
        check_llg_state(l, s);
        check(buf && buflen > 0, "NULL argument");
        bool demag = false;
        for (auto& t : l->terms) demag = demag || t->kind == TK_DEMAG;
        static const char* n3[] = {"x_fwd", "y_fwd", "z_conv", "y_inv", "x_inv_local"};
        static const char* n2[] = {"x_fwd", "y_conv", "x_inv_local"};
        static const char* n0[] = {"local"};
        const char** names = !demag ? n0 : (s->s.md.nz > 1 ? n3 : n2);
        const int count = !demag ? 1 : (s->s.md.nz > 1 ? 5 : 3);
        check(index >= 0 && index < count, "pass index out of range");
        std::snprintf(buf, (size_t)buflen, "%s", names[index]);
    });
}

int maf_llg_dmdt(maf_llg l, maf_state s, double* out) {
    return guarded([&] {
        check_llg_state(l, s);
        check(out, "NULL argument");
        const int64_t n3 = 3 * s->s.md.N();
        l->k[0].ensure(sizeof(double) * n3);
        EpilogueArgs ep;
        ep.kind = EPI_LLG;
        ep.out = l->k[0].p;
        ep.llg = llg_params(l, 1.0);
        eval_on_state(s, raw_terms(l->terms), ep);
        MAF_CUDA(cudaMemcpyAsync(out, l->k[0].p, sizeof(double) * n3, cudaMemcpyDeviceToHost, s->s.stream));
        MAF_CUDA(cudaStreamSynchronize(s->s.stream));
    });
}

int maf_llg_integrate_dense(maf_llg l, maf_state s, double time_in_s, double write_every_dt_in_s, double* rows,
                            int max_rows, int* nrows) {
    return guarded([&] {
        check_llg_state(l, s);
        check(rows && nrows && max_rows > 0, "NULL argument");
        check(write_every_dt_in_s > 0, "integrate_dense: write_every_dt_in_s must be > 0");
        StateD& st = s->s;
        int n = 0;
        auto push = [&](double t, const double mm[3]) {
            if (n < max_rows) {
                rows[4 * n + 0] = t;
                rows[4 * n + 1] = mm[0];
                rows[4 * n + 2] = mm[1];
                rows[4 * n + 3] = mm[2];
                ++n;
            }
        };
        double mm[3];
        mean_m_host(s, st.m64.as<double>(), mm);
        push(st.t, mm);
        const Scheme rkf = make_scheme("RKF45");
        const double time_init = st.t;
        const double time_final = time_init + time_in_s;
        double t_next = time_init + write_every_dt_in_s;
        while (st.t < time_final) {
            llg_step(l, s);
            if (st.t >= t_next) {
                const double backstep = t_next - st.t;  // negative
                // RKF45 back-step from the overshooting state, no normalisation (llg_integrator.cpp:79-94)
                rk_attempt(l, s, rkf, backstep, 0);
                if (t_next >= time_final - 1e-20) {
                    accept_candidate(l, s);
                    st.t += backstep;
                    mean_m_host(s, st.m64.as<double>(), mm);
                    push(st.t, mm);
                    break;
                }
                mean_m_host(s, l->mcand.as<double>(), mm);
                push(st.t + backstep, mm);
                t_next += write_every_dt_in_s;
                while (t_next < st.t) t_next += write_every_dt_in_s;
            }
        }
        *nrows = n;
    });
}

int maf_llg_rk_attempt(maf_llg l, maf_state s, const char* scheme, double dt, double* m_new_host, double* err) {
    return guarded([&] {
        check_llg_state(l, s);
        check(scheme && m_new_host && err, "NULL argument");
        const Scheme sch = make_scheme(scheme);
        *err = rk_attempt(l, s, sch, dt, 0);
        MAF_CUDA(cudaMemcpyAsync(m_new_host, l->mcand.p, sizeof(double) * 3 * s->s.md.N(), cudaMemcpyDeviceToHost,
                                 s->s.stream));
        MAF_CUDA(cudaStreamSynchronize(s->s.stream));
    });
}

int maf_llg_relax(maf_llg l, maf_state s, double precision, int eval_E) {
    return guarded([&] {
        check_llg_state(l, s);
        double E_prev = 1e20;
        double E = llg_energy(l, s);
        while (std::fabs((E_prev - E) / E_prev) > precision) {
            E_prev = E;
            for (int i = 0; i < eval_E; ++i) llg_step(l, s);
            E = llg_energy(l, s);
        }
    });
}

// ------------------------------------------------------------ Stochastic LLG
int maf_stochastic_llg_create(maf_stoch* out, double alpha, double T, double dt, const maf_term* terms, int nterms,
                              const char* smode, unsigned long long seed, unsigned member) {
    return guarded([&] {
        check(out, "NULL argument");
        check(dt > 0, "Stochastic_LLG: dt must be > 0");
        check(T >= 0, "Stochastic_LLG: T must be >= 0");
        auto h = std::make_unique<maf_stoch_s>();
        h->alpha = alpha;
        h->T = T;
        h->dt = dt;
        const std::string m = smode ? smode : "Heun";
        // get_mode (stochastic_integrator.cpp:59-73); unknown strings are rejected instead of falling back to Heun
        if (m == "Heun" || m == "0") h->mode = 0;
        else if (m == "SemiHeun" || m == "1") h->mode = 1;
        else if (m == "detRK4" || m == "2") h->mode = 2;
        else throw Error(MAF_ERR_BADARG, "Stochastic_LLG: integrator mode not recognised: " + m);
        h->seed = seed;
        h->member = member;
        for (int i = 0; i < nterms; ++i) {
            check(terms && terms[i], "Stochastic_LLG: NULL term");
            h->terms.push_back(terms[i]->t);
        }
        check(!h->terms.empty(), "Stochastic_LLG: no field terms");
        *out = h.release();
    });
}

int maf_stochastic_llg_destroy(maf_stoch h) {
    return guarded([&] { delete h; });
}

int maf_stochastic_llg_step(maf_stoch h, maf_state s) {
    return guarded([&] {
        check(h && s, "NULL argument");
        stoch_step(h, s);
    });
}

int maf_stochastic_llg_steps(maf_stoch h, maf_state s, int n) {
    return guarded([&] {
        check(h && s, "NULL argument");
        for (int i = 0; i < n; ++i) stoch_step(h, s);
    });
}

int maf_stochastic_llg_E(maf_stoch h, maf_state s, double* E) {
    return guarded([&] {
        check(h && s && E, "NULL argument");
        std::vector<Term*> terms;
        for (auto& t : h->terms) terms.push_back(t.get());
        EpilogueArgs ep;
        ep.kind = EPI_EDENS;
        eval_on_state(s, terms, ep, E);
    });
}

int maf_stochastic_llg_noise(maf_stoch h, maf_state s, unsigned long long index, double* out) {
    return guarded([&] {
        check(h && s && out, "NULL argument");
        StateD& st = s->s;
        const int64_t n3 = 3 * st.md.N();
        h->mstage64.ensure(sizeof(double) * n3);
        thermal_field(h->mstage64.as<double>(), st.md.N(), thermal_sigma(h, st), h->seed, h->member, index, st.stream);
        MAF_CUDA(cudaMemcpyAsync(out, h->mstage64.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, st.stream));
        MAF_CUDA(cudaStreamSynchronize(st.stream));
    });
}

int maf_stochastic_llg_calls(maf_stoch h, unsigned long long* calls) {
    return guarded([&] { check(h && calls, "NULL argument"); *calls = h->calls; });
}

// ------------------------------------------------------------ LBFGS minimiser
int maf_lbfgs_create(maf_lbfgs* out, const maf_term* terms, int nterms, double tolerance, int maxIter) {
    return guarded([&] {
        check(out, "NULL argument");
        check(maxIter >= 0, "LBFGS_Minimizer: maxIter must be >= 0");
        auto h = std::make_unique<maf_lbfgs_s>();
        for (int i = 0; i < nterms; ++i) {
            check(terms && terms[i], "LBFGS_Minimizer: NULL term");
            h->terms.push_back(terms[i]->t);
        }
        h->tolerance = tolerance;
        h->maxIter = (size_t)maxIter;
        *out = h.release();
    });
}

int maf_lbfgs_destroy(maf_lbfgs h) {
    return guarded([&] { delete h; });
}

int maf_lbfgs_add_term(maf_lbfgs h, maf_term t) {
    return guarded([&] {
        check(h && t, "NULL argument");
        h->terms.push_back(t->t);
    });
}

int maf_lbfgs_minimize(maf_lbfgs h, maf_state s, double* E) {
    return guarded([&] {
        check(h && s && E, "NULL argument");
        // abort_if_size_is_zero (lbfgs_minimizer.cpp:25-30)
        check(!h->terms.empty(), "LBFGS_Minimizer: Number of terms == 0. Please add at least one term.");
        *E = lbfgs_minimize(h, s);
    });
}

int maf_lbfgs_stats(maf_lbfgs h, unsigned long long* iterations, unsigned long long* fevals, double* grad_max) {
    return guarded([&] {
        check(h, "NULL argument");
        if (iterations) *iterations = h->iterations;
        if (fevals) *fevals = h->fevals;
        if (grad_max) *grad_max = h->last_gradnorm;
    });
}

int maf_llg_get_h(maf_llg l, double* h) {
    return guarded([&] { check(l && h, "NULL argument"); *h = l->h; });
}

int maf_llg_get_controller_state(maf_llg l, double out[9]) {
    return guarded([&] {
        check(l && out, "NULL argument");
        const Controller& c = l->ctrl;
        const double v[9] = {l->h, c.errold, c.reject ? 1.0 : 0.0, c.hnext, (double)c.n_accepted, (double)c.n_reject,
                             (double)c.n_hmin, (double)c.n_hmax, (double)l->accumulated_steps};
        std::copy(v, v + 9, out);
    });
}

int maf_llg_set_controller_state(maf_llg l, const double in[9]) {
    return guarded([&] {
        check(l && in, "NULL argument");
        check(in[0] > 0 && std::isfinite(in[0]), "maf_llg_set_controller_state: step size must be positive");
        Controller& c = l->ctrl;
        l->h = in[0];
        c.errold = in[1];
        c.reject = in[2] != 0.0;
        c.hnext = in[3];
        c.n_accepted = (unsigned long long)in[4];
        c.n_reject = (unsigned long long)in[5];
        c.n_hmin = (unsigned long long)in[6];
        c.n_hmax = (unsigned long long)in[7];
        l->accumulated_steps = (unsigned long long)in[8];
    });
}

int maf_state_set_steps(maf_state st, unsigned long long steps) {
    return guarded([&] { check(st, "NULL argument"); st->s.steps = steps; });
}

int maf_llg_counters(maf_llg l, unsigned long long out[4]) {
    return guarded([&] {
        check(l && out, "NULL argument");
        out[0] = l->ctrl.n_accepted;
        out[1] = l->ctrl.n_reject;
        out[2] = l->ctrl.n_hmin;
        out[3] = l->ctrl.n_hmax;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// String method (magnumaf/include/magnumaf/solvers/string_method.hpp:9-39,
//                magnumaf/src/solvers/string_method.cpp:12-314)
//
// The images live on the device as states of the template's mesh and Ms; one
// LLG integrator (borrowed, as the reference's StringMethod holds one
// LLGIntegrator) steps every image in turn, so its controller state carries
// over from image to image exactly as in the reference.  Arc lengths are
// device reductions of sum (m_i - m_{i-1})^2; the re-interpolation and the
// zero-safe normalisation are device kernels.
// ---------------------------------------------------------------------------
struct maf_string_s {
    maf_llg_s* llg = nullptr;
    int n_interp = 0;
    double dt = 0;
    cudaStream_t stream = nullptr;
    std::vector<std::unique_ptr<maf_state_s>> images;
    std::vector<double> x, x_interp, E;
    DevBuf tmp;      // [n_interp][3N] copy of the images for the re-interpolation
    DevBuf scratch;  // reduction partials
    // batched integration (maf_string_set_batched): per image a fixed-step RK4
    // integrator with its own demag buffers and its own stream; every image is
    // advanced by one CUDA graph of the ensemble batch
    int substeps = 0;
    std::vector<std::unique_ptr<maf_stoch_s>> bits;
    std::vector<cudaStream_t> bstreams;
    maf_stoch_batch_s* batch = nullptr;
    void drop_batch() {
        if (batch) maf_stoch_batch_destroy(batch);
        batch = nullptr;
        for (auto& img : images) img->s.stream = stream;
        for (auto st : bstreams) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        bstreams.clear();
        bits.clear();
        substeps = 0;
    }
    ~maf_string_s() {
        if (stream) cudaStreamSynchronize(stream);
        drop_batch();
        images.clear();
        tmp.release();
        scratch.release();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// a state with the template's mesh, precision and Ms (or Ms_field), on stream st
std::unique_ptr<maf_state_s> make_image(const maf_state_s& tmpl, cudaStream_t st) {
    auto h = std::make_unique<maf_state_s>();
    StateD& s = h->s;
    const StateD& t = tmpl.s;
    s.md = t.md;
    s.precision = t.precision;
    s.Ms = t.Ms;
    s.has_Ms_field = t.has_Ms_field;
    s.stream = st;
    s.own_stream = false;
    const int64_t N = s.md.N();
    s.m64.alloc(sizeof(double) * 3 * N);
    if (t.has_Ms_field) {
        s.Msf64.alloc(sizeof(double) * N);
        MAF_CUDA(cudaMemcpyAsync(s.Msf64.p, t.Msf64.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        if (s.precision == PREC_FP32_FIELD) {
            s.Msf32.alloc(sizeof(float) * N);
            MAF_CUDA(cudaMemcpyAsync(s.Msf32.p, t.Msf32.p, sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
        }
    }
    return h;
}

// FrobeniusNorm(a - b) = sqrt(mean((a - b)^2)) over all 3N values (util.cpp:53-55)
double frob_diff(maf_string_s* h, const double* a, const double* b, int64_t n3) {
    h->scratch.ensure(sizeof(double) * (red_blocks() + 2));
    return std::sqrt(sqdiff_host(a, b, n3, h->scratch.as<double>(), h->stream) / (double)n3);
}

// StringMethod::calc_x (string_method.cpp:57-81)
void string_calc_x(maf_string_s* h, const std::vector<const double*>& ms, int64_t n3) {
    h->x.assign(1, 0.0);
    for (size_t i = 1; i < ms.size(); ++i) h->x.push_back(h->x[i - 1] + frob_diff(h, ms[i], ms[i - 1], n3));
    h->x_interp.clear();
    for (int i = 0; i < h->n_interp; ++i)
        h->x_interp.push_back(static_cast<double>(i) / static_cast<double>(h->n_interp - 1) * h->x.back());
}

// the bracket search of string_method.cpp:22-28 / :86-92 (x[j] is only read for
// j < x.size(), which the reference's loop never exceeds either)
int string_bracket(const maf_string_s* h, int i) {
    int j = 0;
    const int jmax = std::min<int>(h->n_interp, (int)h->x.size());
    while (j < jmax && h->x[j] < h->x_interp[i]) ++j;
    if (j > 0) --j;
    return j;
}

void string_normalize(maf_string_s* h) {
    for (auto& img : h->images) {
        normalize_m(img->s.m64.as<double>(), img->s.md.N(), 0, nullptr, h->stream);
        img->m32_valid = false;
    }
}

// StringMethod::integrate (string_method.cpp:108-121); in batched mode every image
// takes `substeps` RK4 steps of dt/substeps, all images in the ensemble graph
void string_integrate(maf_string_s* h) {
    if (h->batch) {
        MAF_CUDA(cudaStreamSynchronize(h->stream));  // the re-interpolation has written the images
        const int rc = maf_stoch_batch_steps(h->batch, h->substeps);
        if (rc != MAF_OK) throw Error(rc, maf_last_error());
        return;
    }
    for (auto& img : h->images) {
        const double t0 = img->s.t;
        while (img->s.t < t0 + h->dt) llg_step(h->llg, img.get());
    }
}

// StringMethod::lin_interpolate (string_method.cpp:83-106)
void string_lin_interpolate(maf_string_s* h) {
    const int n = h->n_interp;
    const int64_t n3 = 3 * h->images[0]->s.md.N();
    h->tmp.ensure(sizeof(double) * n3 * n);
    double* tmp = h->tmp.as<double>();
    std::vector<double> t_tmp(n);
    std::vector<unsigned long long> steps_tmp(n);
    for (int i = 0; i < n; ++i) {
        MAF_CUDA(cudaMemcpyAsync(tmp + i * n3, h->images[i]->s.m64.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                                 h->stream));
        t_tmp[i] = h->images[i]->s.t;
        steps_tmp[i] = h->images[i]->s.steps;
    }
    for (int i = 0; i < n; ++i) {
        const int j = string_bracket(h, i);
        double* out = h->images[i]->s.m64.as<double>();
        if (j < n - 1) {
            lerp(out, tmp + j * n3, tmp + (j + 1) * n3, h->x_interp[i] - h->x[j], h->x[j + 1] - h->x[j], n3,
                 h->stream);
        } else {
            std::printf("Warning: x_interp[j=%d] exceedes x range, y_interp[j] value set to y[j]\n", j);
            MAF_CUDA(cudaMemcpyAsync(out, tmp + j * n3, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
            h->images[i]->s.t = t_tmp[j];
            h->images[i]->s.steps = steps_tmp[j];
        }
    }
    string_normalize(h);
    if (h->batch) MAF_CUDA(cudaStreamSynchronize(h->stream));  // images are read next on their own streams
}

std::vector<const double*> image_ms(const maf_string_s* h) {
    std::vector<const double*> v;
    for (auto& img : h->images) v.push_back(img->s.m64.as<double>());
    return v;
}

// StringMethod::step (string_method.cpp:128-132)
void string_step(maf_string_s* h) {
    string_integrate(h);
    string_calc_x(h, image_ms(h), 3 * h->images[0]->s.md.N());
    string_lin_interpolate(h);
}

// StringMethod::calc_E (string_method.cpp:48-55)
void string_calc_E(maf_string_s* h) {
    h->E.clear();
    for (auto& img : h->images) h->E.push_back(llg_energy(h->llg, img.get()));
}

}  // namespace

namespace {

// gnuplot script of string_method.cpp:145-172 (written, not executed)
void string_write_plotfile(const std::string& filepath) {
    std::ofstream f(filepath + "plot_string_method.gpi");
    f << "set terminal pdf\nset key left top Left\n\n"
      << "set title 'Energy over image ID for each iteration'\nset xlabel 'Image ID'\nset ylabel 'E [J]'\n"
      << "set cblabel 'Iteration'\nset format y '%.1e'\nset output 'E_curves.pdf'\n"
      << "p 'E_curves.dat' u 2:3:1 w l palette t 'E'\n\n"
      << "set title 'Energy barrier over iteration'\nset xlabel 'Iteration'\nset ylabel 'dE [J]'\n"
      << "set output 'dE_over_iteration.pdf'\np 'dE_over_iteration.dat' u 1:2 w l notitle\n\n"
      << "set title 'Energy over image ID'\nset xlabel 'Image ID'\nset ylabel 'E [J]'\nset output 'E.pdf'\n"
      << "p 'E_last_step.dat' u 1:3 w l t 'Last iteration', 'E_max_lowest.dat' u 1:3 w l t 'Lowest barrier'\n";
}

// StringMethod::run (string_method.cpp:174-314): the iteration, the abort
// criteria and the .dat files; the reference's VTK image files and its
// gnuplot call are not produced.  Where the reference indexes E[-1] it means
// the last image; E.back() is written.
double string_run(maf_string_s* h, const std::string& filepath, double rel_abort, double abs_abort, int steps,
                  bool verbose, int* iterations) {
    string_write_plotfile(filepath);
    std::ofstream f_steps(filepath + "dE_over_iteration.dat");
    f_steps << "# i \t dE [J] \t dE rel_diff to step i-1 \t dE abs_diff to step i-1\n";
    f_steps.precision(12);
    std::ofstream f_curves(filepath + "E_curves.dat");
    f_curves << "# step \t image \t dE=E[j]-E[0] \t E[j]-E[-1] \t E[j]\n";
    f_curves.precision(12);
    double max_lowest = 1e100, max_prev = 1e100;
    int i_max_lowest = -1;
    std::vector<double> E_max_lowest;
    int it = 0;
    for (int i = 0; i < steps; ++i) {
        it = i + 1;
        string_step(h);
        string_calc_E(h);
        const double emax = *std::max_element(h->E.begin(), h->E.end());
        const double barrier = emax - h->E[0];
        if (barrier < max_lowest) {
            max_lowest = barrier;
            i_max_lowest = i;
            E_max_lowest = h->E;
        }
        const double abs_diff = std::fabs(barrier - max_prev);
        const double rel_diff = std::fabs((2. * abs_diff) / (barrier + max_prev));
        if (i > 25 && rel_diff < rel_abort) {
            if (verbose)
                std::printf("StringMethod run: relative difference of two consecutive E_barriers is: rel_diff=%e. "
                            "This is smaller than %e\n", rel_diff, rel_abort);
            f_steps << "#StringMethod run: relative difference of two consecutive E_barriers is: rel_diff= "
                    << rel_diff << " This is smaller than " << rel_abort << "\n";
            break;
        }
        if (i > 25 && abs_diff < abs_abort) {
            if (verbose)
                std::printf("StringMethod run: absolute difference of two consecutive E_barriers is: abs_diff=%e "
                            "is smaller than %e\n", abs_diff, abs_abort);
            f_steps << "#StringMethod run: absolute difference of two consecutive E_barriers is: abs_diff= "
                    << abs_diff << " is smaller than " << abs_abort << "\n";
            break;
        }
        {
            std::ofstream fb(filepath + "E_barrier.dat");
            fb.precision(12);
            fb << "# max_lowest \t this->images[0].mesh.nx \t this->images[0].mesh.dx\n"
               << max_lowest << "\t" << h->images[0]->s.md.nx << "\t" << h->images[0]->s.md.dx << "\n";
        }
        for (size_t j = 0; j < h->E.size(); ++j)
            f_curves << i << " " << j << " " << h->E[j] - h->E[0] << " " << h->E[j] - h->E.back() << " " << h->E[j]
                     << "\n";
        f_curves << i << "\n\n\n";
        max_prev = barrier;
        if (verbose)
            std::printf("step=%d, dE[J]=%e, rel_diff[J]= %e, abs_diff[J]=%e\n", i, barrier, rel_diff, abs_diff);
        f_steps << i << "\t" << std::setw(18) << barrier << "\t" << rel_diff << "\t" << abs_diff << "\n";
    }
    if (verbose) std::printf("i=%d, minimal dE=%e\n", i_max_lowest, max_lowest);
    if (!E_max_lowest.empty())
        f_steps << "#i , lowest overall:   max-[0], max-[-1] max [J]: " << i_max_lowest << "\t" << max_lowest << "\t"
                << max_lowest + E_max_lowest[0] - E_max_lowest.back() << "\t" << max_lowest + E_max_lowest[0]
                << "\n";
    std::ofstream fE(filepath + "E_last_step.dat");
    fE << " i \t << E[i] \t << dE = E[i] - E[0] \t << E[i] - E[-1] \n";
    fE.precision(12);
    std::ofstream fL(filepath + "E_max_lowest.dat");
    fL << " i \t << E_max_lowest[i] \t << E_max_lowest[i] - E_max_lowest[0] \t << E_max_lowest[i] - E_max_lowest[-1]\n";
    fL.precision(12);
    for (size_t i = 0; i < h->E.size(); ++i) {
        fE << i << "\t" << h->E[i] << "\t" << h->E[i] - h->E[0] << "\t" << h->E[i] - h->E.back() << "\n";
        if (i < E_max_lowest.size())
            fL << i << "\t" << E_max_lowest[i] << "\t" << E_max_lowest[i] - E_max_lowest[0] << "\t"
               << E_max_lowest[i] - E_max_lowest.back() << "\n";
    }
    if (iterations) *iterations = it;
    return max_lowest;
}

}  // namespace

extern "C" {

int maf_string_create(maf_string* out, maf_state state, const maf_state* inputimages, int n_inputimages, int n_interp,
                      double dt, maf_llg llg) {
    return guarded([&] {
        check(out && state && inputimages && llg, "maf_string_create: NULL argument");
        check(n_inputimages >= 2,
              "StringMethod: invalid inputimages provided, please add at least two states/magnetizations for "
              "interpolation of initial path.");
        check(n_interp >= 2, "StringMethod: n_interp must be at least 2");
        check(!llg->terms.empty(), "LLGIntegrator: no field terms");
        const MeshDims md = state->s.md;
        for (int i = 0; i < n_inputimages; ++i) {
            check(inputimages[i] != nullptr, "maf_string_create: NULL input image");
            check(inputimages[i]->s.md == md, "StringMethod: input image mesh differs from the state's mesh");
        }
        auto h = std::make_unique<maf_string_s>();
        h->llg = llg;
        h->n_interp = n_interp;
        h->dt = dt;
        MAF_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        MAF_CUDA(cudaStreamSynchronize(state->s.stream));
        std::vector<const double*> in_m;
        for (int i = 0; i < n_inputimages; ++i) {
            MAF_CUDA(cudaStreamSynchronize(inputimages[i]->s.stream));
            in_m.push_back(inputimages[i]->s.m64.as<double>());
        }
        const int64_t n3 = 3 * md.N();
        string_calc_x(h.get(), in_m, n3);
        for (int i = 0; i < n_interp; ++i) {
            auto img = make_image(*state, h->stream);
            const int j = string_bracket(h.get(), i);
            if (j < n_interp - 1) {
                lerp(img->s.m64.as<double>(), in_m[j], in_m[j + 1], h->x_interp[i] - h->x[j], h->x[j + 1] - h->x[j],
                     n3, h->stream);
            } else {
                std::printf("Warning: x_interp[j=%d] exceedes x range, y_interp[j] value set to y[j]\n", j);
                MAF_CUDA(cudaMemcpyAsync(img->s.m64.p, in_m[j], sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                                         h->stream));
                img->s.t = inputimages[j]->s.t;
                img->s.steps = inputimages[j]->s.steps;
            }
            h->images.push_back(std::move(img));
        }
        for (auto& img : h->images) check_llg_state(llg, img.get());
        string_normalize(h.get());
        MAF_CUDA(cudaStreamSynchronize(h->stream));
        *out = h.release();
    });
}

int maf_string_destroy(maf_string h) {
    return guarded([&] { delete h; });
}

int maf_string_set_batched(maf_string h, int substeps) {
    return guarded([&] {
        check(h && substeps >= 0, "maf_string_set_batched: bad argument");
        MAF_CUDA(cudaStreamSynchronize(h->stream));
        h->drop_batch();
        if (substeps == 0) return;
        maf_llg_s* l = h->llg;
        check(!l->has_alpha_field, "StringMethod batched: needs a scalar alpha");
        const StateD& s0 = h->images[0]->s;
        check(!s0.has_Ms_field, "StringMethod batched: needs a scalar Ms");
        try {
            // demag terms get a copy per image (their spectral buffers are per plan);
            // the local terms hold no mutable state and are shared
            std::vector<double> tensor;
            for (int i = 0; i < h->n_interp; ++i) {
                cudaStream_t st;
                MAF_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                h->bstreams.push_back(st);
                auto it = std::make_unique<maf_stoch_s>();
                it->alpha = l->alpha;
                it->T = 0.0;
                it->dt = h->dt / substeps;
                it->mode = 2;  // deterministic RK4 (stochastic_integrator.cpp:34-40)
                it->member = (unsigned)i;
                for (auto& t : l->terms) {
                    if (t->kind != TK_DEMAG) {
                        it->terms.push_back(t);
                        continue;
                    }
                    auto c = std::make_shared<Term>();
                    c->kind = TK_DEMAG;
                    c->p[0] = t->p[0];
                    if (!t->demag_pbc()) {
                        if (tensor.empty()) {
                            tensor.resize(t->demag->tensor_elems());
                            t->demag->download_tensor(tensor.data(), 0);
                        }
                        c->demag_mesh = t->demag_mesh;
                        c->demag = std::make_unique<Demag>(t->demag_mesh, st, tensor.data());
                        c->demag->tune = t->demag->tune;
                    }
                    it->terms.push_back(c);
                }
                h->images[i]->s.stream = st;
                h->bits.push_back(std::move(it));
            }
            std::vector<maf_stoch> its;
            std::vector<maf_state> sts;
            for (int i = 0; i < h->n_interp; ++i) {
                its.push_back(h->bits[i].get());
                sts.push_back(h->images[i].get());
            }
            const int rc = maf_stoch_batch_create(&h->batch, its.data(), sts.data(), h->n_interp);
            if (rc != MAF_OK) throw Error(rc, maf_last_error());
            h->substeps = substeps;
        } catch (...) {
            h->drop_batch();
            throw;
        }
    });
}

int maf_string_step(maf_string h) {
    return guarded([&] {
        check(h, "NULL argument");
        string_step(h);
        MAF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int maf_string_calc_E(maf_string h, double* E_out) {
    return guarded([&] {
        check(h, "NULL argument");
        string_calc_E(h);
        if (E_out) std::copy(h->E.begin(), h->E.end(), E_out);
    });
}

int maf_string_run(maf_string h, const char* filepath, double string_abort_rel_diff, double string_abort_abs_diff,
                   int string_steps, int every_string_to_vti, int verbose, double* dE, int* iterations) {
    (void)every_string_to_vti;
    return guarded([&] {
        check(h && filepath && dE, "NULL argument");
        *dE = string_run(h, filepath, string_abort_rel_diff, string_abort_abs_diff, string_steps, verbose != 0,
                         iterations);
    });
}

int maf_string_n_images(maf_string h, int* n) {
    return guarded([&] { check(h && n, "NULL argument"); *n = h->n_interp; });
}

int maf_string_get_x(maf_string h, double* x, double* x_interp) {
    return guarded([&] {
        check(h, "NULL argument");
        if (x) std::copy(h->x.begin(), h->x.end(), x);
        if (x_interp) std::copy(h->x_interp.begin(), h->x_interp.end(), x_interp);
    });
}

int maf_string_image(maf_string h, int i, maf_state* image) {
    return guarded([&] {
        check(h && image, "NULL argument");
        check(i >= 0 && i < h->n_interp, "maf_string_image: image index out of range");
        *image = h->images[i].get();
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched stochastic ensembles: every member (integrator i steps state i) is
// advanced by one CUDA graph.  The graph holds two steps of every member, each
// member on its own state's stream between a fork and a join event, so members
// of uneven meshes run concurrently and two steps of the whole ensemble cost one
// graph launch.  Two steps because a step swaps the state and candidate buffers:
// after two the buffers are back where the graph expects them.  The noise
// stream index comes from a device step counter per member that the graph
// advances, so every replay draws the next numbers; results are bit-identical
// to stepping the members one after another.
// ---------------------------------------------------------------------------
struct maf_stoch_batch_s {
    std::vector<maf_stoch_s*> its;
    std::vector<maf_state_s*> sts;
    bool fused = false;                     // batched passes (one launch per pass for all members)
    std::unique_ptr<mafb::FusedBatch> fb;   // built at capture time when every member qualifies
    bool fused_active = false;              // the current graph runs the batched passes
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    DevBuf q;  // per-member step counters (device)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> m_at_capture;  // state buffers the graph was captured with
    bool warm = false;
    ~maf_stoch_batch_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : join) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (done) cudaEventDestroy(done);
        if (root) cudaStreamDestroy(root);
    }
};

namespace {

void batch_drop_graph(maf_stoch_batch_s* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->fused_active = false;
}

// device counters <- host step counts
void batch_upload_counters(maf_stoch_batch_s* b) {
    std::vector<unsigned long long> q(b->its.size());
    for (size_t i = 0; i < q.size(); ++i) q[i] = b->its[i]->calls;
    MAF_CUDA(cudaMemcpyAsync(b->q.p, q.data(), sizeof(unsigned long long) * q.size(), cudaMemcpyHostToDevice,
                             b->root));
    MAF_CUDA(cudaStreamSynchronize(b->root));
}

// The integrator's scheme with its noise stream indices relative to the step
// counter q (the stages stoch_step builds).
FusedScheme fused_scheme(const maf_stoch_s* h) {
    FusedScheme f;
    const double dt = h->dt;
    if (h->mode == 0) {
        FusedStage a; a.noise = true; a.offset = 0; a.scale = dt;
        FusedStage b; b.n = 1; b.j[0] = 0; b.c[0] = 1.0; b.noise = true; b.offset = 1; b.scale = dt;
        f.stages = {a, b};
        f.nfin = 2; f.fin_base = 0; f.fin_c[0] = 0.5; f.fin_c[1] = 0.5;
        f.noise_mul = 1;
    } else if (h->mode == 1) {
        FusedStage a; a.noise = true; a.offset = 0; a.scale = dt / 2.;
        f.stages.push_back(a);
        for (int i = 1; i < 6; ++i) {
            FusedStage b; b.n = 1; b.j[0] = i - 1; b.c[0] = 1.0; b.noise = true; b.offset = 1;
            b.scale = i < 5 ? dt / 2. : dt;
            f.stages.push_back(b);
        }
        f.nfin = 1; f.fin_base = 5; f.fin_c[0] = 1.0;
        f.noise_mul = 2;
    } else {
        FusedStage a; a.scale = dt;
        FusedStage b; b.n = 1; b.j[0] = 0; b.c[0] = 1. / 2.; b.scale = dt;
        FusedStage c; c.n = 1; c.j[0] = 1; c.c[0] = 1. / 2.; c.scale = dt;
        FusedStage d; d.n = 1; d.j[0] = 2; d.c[0] = 1.0; d.scale = dt;
        f.stages = {a, b, c, d};
        f.nfin = 4; f.fin_base = 0; f.fin_c[0] = 1. / 6.; f.fin_c[1] = 2. / 6.; f.fin_c[2] = 2. / 6.; f.fin_c[3] = 1. / 6.;
    }
    return f;
}

// The batched-pass plan of the batch's members, or null when a member does not
// qualify (3-D mesh, no or periodic DemagField, parameter fields, mixed
// precisions or schemes): those batches keep the per-member graph.
std::unique_ptr<FusedBatch> make_fused(maf_stoch_batch_s* b) {
    const size_t n = b->its.size();
    const FusedScheme sch = fused_scheme(b->its[0]);
    const bool f32 = b->sts[0]->s.precision == PREC_FP32_FIELD;
    std::vector<FusedMember> mem;
    for (size_t i = 0; i < n; ++i) {
        maf_stoch_s* h = b->its[i];
        maf_state_s* st = b->sts[i];
        if (h->mode != b->its[0]->mode || h->dt != b->its[0]->dt) return nullptr;
        if ((st->s.precision == PREC_FP32_FIELD) != f32) return nullptr;
        FusedMember f;
        f.md = st->s.md;
        f.Ms = st->s.Ms;
        for (auto& t : h->terms) {
            if (t->kind == TK_DEMAG) f.demag = t->demag.get();
            f.terms.push_back(t->desc());
        }
        f.m[0] = st->s.m64.as<double>();
        f.m[1] = h->mcand.as<double>();
        f.m32 = f32 ? st->s.m32.as<float>() : nullptr;
        f.mstage64 = h->mstage64.as<double>();
        f.mstage32 = f32 ? h->mstage32.as<float>() : nullptr;
        for (size_t s = 0; s < sch.stages.size(); ++s) f.k[s] = h->k[s].as<double>();
        f.c_prec = -kGamma / (1. + h->alpha * h->alpha);
        f.c_damp = -h->alpha * kGamma / (1. + h->alpha * h->alpha);
        f.sigma = thermal_sigma(h, st->s);
        f.seed = h->seed;
        f.member = h->member;
        f.q = b->q.as<unsigned long long>() + i;
        if (!f.m[1] || !f.mstage64 || (f32 && (!f.m32 || !f.mstage32))) return nullptr;
        mem.push_back(std::move(f));
    }
    if (!fused_supported(mem, sch)) return nullptr;
    return std::make_unique<FusedBatch>(std::move(mem), sch, f32, b->root);
}

void batch_capture(maf_stoch_batch_s* b) {
    batch_drop_graph(b);
    const size_t n = b->its.size();
    auto* q = b->q.as<unsigned long long>();
    b->fb.reset();
    b->fused_active = false;
    if (b->fused) b->fb = make_fused(b);
    // host-side state advances while the work is only recorded: restore it
    std::vector<double> t(n);
    std::vector<unsigned long long> steps(n), calls(n);
    for (size_t i = 0; i < n; ++i) {
        t[i] = b->sts[i]->s.t;
        steps[i] = b->sts[i]->s.steps;
        calls[i] = b->its[i]->calls;
    }
    MAF_CUDA(cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal));
    try {
        if (b->fb) {
            // two steps of every member: the first writes the candidates, the second
            // the states again, so the graph leaves the buffers where it found them
            b->fb->record_step(b->root, 0);
            b->fb->record_step(b->root, 1);
            b->fused_active = true;
        } else {
            MAF_CUDA(cudaEventRecord(b->fork, b->root));
            for (size_t i = 0; i < n; ++i) {
                cudaStream_t s = b->sts[i]->s.stream;
                MAF_CUDA(cudaStreamWaitEvent(s, b->fork, 0));
                stoch_step(b->its[i], b->sts[i], q + i);
                stoch_step(b->its[i], b->sts[i], q + i);
                MAF_CUDA(cudaEventRecord(b->join[i], s));
                MAF_CUDA(cudaStreamWaitEvent(b->root, b->join[i], 0));
            }
        }
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(b->root, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    MAF_CUDA(cudaStreamEndCapture(b->root, &b->graph));
    MAF_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->m_at_capture.clear();
    for (size_t i = 0; i < n; ++i) {
        b->sts[i]->s.t = t[i];
        b->sts[i]->s.steps = steps[i];
        b->its[i]->calls = calls[i];
        b->m_at_capture.push_back(b->sts[i]->s.m64.p);
    }
}

}  // namespace

extern "C" {

int maf_stoch_batch_create(maf_stoch_batch* out, const maf_stoch* integrators, const maf_state* states, int n) {
    return guarded([&] {
        check(out && integrators && states && n > 0, "maf_stoch_batch_create: bad argument");
        auto b = std::make_unique<maf_stoch_batch_s>();
        for (int i = 0; i < n; ++i) {
            check(integrators[i] && states[i], "maf_stoch_batch_create: NULL member");
            check(!integrators[i]->terms.empty(), "Stochastic_LLG: no field terms");
            check(!states[i]->s.has_Ms_field, "Stochastic_LLG uses the scalar Ms (stochastic_integrator.cpp:9-10)");
            for (int j = 0; j < i; ++j) {
                check(states[j] != states[i], "maf_stoch_batch_create: a state appears twice");
                check(integrators[j] != integrators[i], "maf_stoch_batch_create: an integrator appears twice");
                check(states[j]->s.stream != states[i]->s.stream,
                      "maf_stoch_batch_create: members must run on distinct streams");
                // members run concurrently: a demag plan's spectral buffers cannot be shared
                for (auto& ti : integrators[i]->terms)
                    for (auto& tj : integrators[j]->terms)
                        check(ti->kind != TK_DEMAG || ti.get() != tj.get(),
                              "maf_stoch_batch_create: members share a DemagField; give each member its own");
            }
            b->its.push_back(integrators[i]);
            b->sts.push_back(states[i]);
        }
        MAF_CUDA(cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking));
        MAF_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        MAF_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
        b->join.resize(n);
        for (int i = 0; i < n; ++i) MAF_CUDA(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming));
        b->q.alloc(sizeof(unsigned long long) * n);
        *out = b.release();
    });
}

int maf_stoch_batch_destroy(maf_stoch_batch b) {
    return guarded([&] { delete b; });
}

int maf_stoch_batch_set_fused(maf_stoch_batch b, int on) {
    return guarded([&] {
        check(b, "NULL argument");
        if (b->fused != (on != 0)) batch_drop_graph(b);
        b->fused = on != 0;
    });
}

int maf_stoch_batch_is_fused(maf_stoch_batch b, int* active) {
    return guarded([&] {
        check(b && active, "NULL argument");
        *active = b->fused_active ? 1 : 0;
    });
}

int maf_stoch_batch_steps(maf_stoch_batch b, int nsteps) {
    return guarded([&] {
        check(b && nsteps >= 0, "maf_stoch_batch_steps: bad argument");
        const size_t n = b->its.size();
        int left = nsteps;
        for (auto* st : b->sts) MAF_CUDA(cudaStreamSynchronize(st->s.stream));
        // the first step runs eagerly: it sizes every work buffer before a capture
        if (left > 0 && !b->warm) {
            for (size_t i = 0; i < n; ++i) stoch_step(b->its[i], b->sts[i]);
            --left;
            b->warm = true;
        }
        if (left >= 2) {
            bool stale = !b->exec;
            for (size_t i = 0; i < n && !stale; ++i) stale = b->sts[i]->s.m64.p != b->m_at_capture[i];
            for (auto* st : b->sts) MAF_CUDA(cudaStreamSynchronize(st->s.stream));
            batch_upload_counters(b);
            if (stale) batch_capture(b);
            while (left >= 2) {
                MAF_CUDA(cudaGraphLaunch(b->exec, b->root));
                for (size_t i = 0; i < n; ++i) {
                    b->sts[i]->s.t += b->its[i]->dt;  // twice, as two single steps add it
                    b->sts[i]->s.t += b->its[i]->dt;
                    b->sts[i]->s.steps += 2;
                    b->its[i]->calls += 2;
                    b->sts[i]->m32_valid = false;
                }
                left -= 2;
            }
            MAF_CUDA(cudaEventRecord(b->done, b->root));
            for (auto* st : b->sts) MAF_CUDA(cudaStreamWaitEvent(st->s.stream, b->done, 0));
        }
        for (; left > 0; --left)
            for (size_t i = 0; i < n; ++i) stoch_step(b->its[i], b->sts[i]);
        for (auto* st : b->sts) MAF_CUDA(cudaStreamSynchronize(st->s.stream));
        MAF_CUDA(cudaStreamSynchronize(b->root));
    });
}

}  // extern "C"
