// Batched passes of an ensemble of small states (stochastic LLG members,
// string-method images): one kernel launch per pass covers every member.  Each
// CTA of a launch reads its (member, tile) pair from a device work table and
// the member's parameters from a device array, and runs that tile of the
// member's pass (the generic kernels' tile bodies, passes_generic.cuh), so a
// step of M members of uneven sizes costs the launches of one member.
//
// Reference: the ensemble and the string images are stepped one after another
// in magnumaf/src/integrators/stochastic_integrator.cpp:42-57 and
// magnumaf/src/solvers/string_method.cpp:107-121.
#pragma once
#include <vector>

#include "engine.hpp"

namespace mafb {

// One stage of a fixed-step scheme: m_s = m + sum_t c[t] k[j[t]] (stage 0: m),
// k_s = scale * dm/dt(m_s) with the thermal field of stream index
// noise_mul * q + offset when noise is set.
struct FusedStage {
    int n = 0;
    int j[6] = {};
    double c[6] = {};
    bool noise = false;
    unsigned long long offset = 0;
    double scale = 0;
};

// The scheme: its stages, then m <- normalise(m + sum_t fin_c[t] k[fin_base + t])
// (the zero-safe normalisation).
struct FusedScheme {
    std::vector<FusedStage> stages;
    int nfin = 0;
    int fin_base = 0;
    double fin_c[6] = {};
    unsigned noise_mul = 1;
};

// One member: a 2-D mesh with a DemagField and its term list.
struct FusedMember {
    MeshDims md;
    double Ms = 0;
    Demag* demag = nullptr;
    std::vector<TermDesc> terms;  // in list order, the demag entry included
    double* m[2] = {};            // state m and candidate; the roles swap every step
    float* m32 = nullptr;         // FP32 copy of the stage-0 m (FP32-field form)
    double* mstage64 = nullptr;
    float* mstage32 = nullptr;
    double* k[6] = {};
    double c_prec = 0, c_damp = 0, sigma = 0;
    unsigned long long seed = 0;
    unsigned member = 0;
    unsigned long long* q = nullptr;  // device step counter of the member's noise stream
};

class FusedBatch {
  public:
    // All members share the scheme and the precision (f32: FP32 field, FP64 state).
    FusedBatch(std::vector<FusedMember> members, FusedScheme scheme, bool f32, cudaStream_t st);
    ~FusedBatch();
    // Records one step of every member on st; parity p reads m[p] and writes the
    // new state to m[1 - p].  Also advances every member's counter q.
    void record_step(cudaStream_t st, int parity);
    int launches_per_step() const;

  private:
    struct Impl;
    Impl* impl_;
};

// Every member can run in the batched passes (2-D mesh, one non-periodic
// DemagField, at most 6 stages, run-time plans for its lengths).
bool fused_supported(const std::vector<FusedMember>& members, const FusedScheme& scheme);

}  // namespace mafb
