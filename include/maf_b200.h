/*
 * magnum.af B200 field / time-step library: C ABI.
 *
 * Drop-in boundary for magnum.af's effective-field and time-step hot path.
 * Each entry point names the reference interface it replaces (paths relative
 * to the magnum.af project root).  Conventions:
 *   - every function returns an int status (MAF_OK on success); the message of
 *     the last failure on the calling thread is returned by maf_last_error();
 *   - vector fields are double [3][nz][ny][nx] (x fastest, component slowest),
 *     the same bytes as ArrayFire's column-major [nx, ny, nz, 3] arrays that
 *     the reference passes around; scalar fields are [nz][ny][nx];
 *   - the library owns all device memory; one state = one CUDA stream (its own
 *     unless maf_state_set_stream() installs the caller's); handles are not
 *     thread-safe;
 *   - the CUDA path is the only path: there is no CPU fallback, and without a
 *     usable GPU every compute call fails with MAF_ERR_NODEVICE.
 */
#ifndef MAF_B200_H
#define MAF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct maf_state_s* maf_state;
typedef struct maf_term_s* maf_term;
typedef struct maf_llg_s* maf_llg;

enum {
    MAF_OK = 0,
    MAF_ERR_BADARG = 1,      /* invalid argument / shape mismatch */
    MAF_ERR_CUDA = 2,        /* CUDA runtime failure */
    MAF_ERR_OOM = 3,         /* device allocation failed */
    MAF_ERR_NAN = 4,         /* NaN/Inf detected in the RK error norm */
    MAF_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    MAF_ERR_UNSUPPORTED = 6, /* e.g. an FFT length with a prime factor > 13 */
    MAF_ERR_NODEVICE = 7     /* no CUDA device available */
};

enum {
    MAF_FP64 = 0,      /* everything in FP64 (the reference's f64 path) */
    MAF_FP32_FIELD = 1 /* field (demag FFT + stencils) in FP32; RK state, error norm, energies in FP64 */
};

/* Thread-local message of the last failure ("" when none). */
const char* maf_last_error(void);
/* Library version. */
int maf_version(int* major, int* minor);
/* Number of visible CUDA devices (0 without a GPU). */
int maf_device_count(int* n);

/* ---------------------------------------------------------------- State ---
 * Replaces magnumaf::State(Mesh, double Ms, af::array m) and
 * State(Mesh, af::array Ms_field, af::array m)
 * (magnumaf/include/magnumaf/state.hpp:14-15, magnumaf/src/state.cpp:91-111).
 * m is normalised on construction; with a scalar Ms and some |m| == 0 an
 * Ms_field = Ms * (|m| != 0) is created (state.cpp:71-89).
 * Ms_field_host may be NULL (scalar Ms). */
int maf_state_create(maf_state* out, int nx, int ny, int nz, double dx, double dy, double dz, double Ms,
                     const double* Ms_field_host, const double* m_host, int precision);
int maf_state_destroy(maf_state s);
/* copy m to the host: replaces State::m / get_m_addr (state.hpp:32, state.cpp:133) */
int maf_state_get_m(maf_state s, double* m_host);
/* State::set_m: normalises (state.cpp:131) */
int maf_state_set_m(maf_state s, const double* m_host);
/* m copied as it is, without normalisation: restoring a checkpoint or a file (State::_vti_reader,
 * vtk_io.cpp:255-259, assigns the file's values) */
int maf_state_load_m(maf_state s, const double* m_host);
int maf_state_get_t(maf_state s, double* t);
int maf_state_set_t(maf_state s, double t);
int maf_state_get_steps(maf_state s, unsigned long long* steps);
/* State::mean_m (state.cpp:39-45): sum of m over cells / number of cells with |m| != 0 */
int maf_state_mean_m(maf_state s, double out[3]);
/* has_field = 1 and Ms_field copied to host (if non-NULL) when the state carries an Ms_field */
int maf_state_get_Ms_field(maf_state s, double* Ms_field_host, int* has_field);
int maf_state_get_Ms(maf_state s, double* Ms);
/* Use the caller's cudaStream_t for all work on this state (NULL: back to the state's own stream). */
int maf_state_set_stream(maf_state s, void* cuda_stream);
/* Device pointer of m (double [3][N]); it changes after every accepted step. */
int maf_state_device_m(maf_state s, void** m64_dev);
int maf_state_precision(maf_state s, int* precision);

/* ---------------------------------------------------------------- Terms ---
 * Field terms; each replaces a FieldTerm subclass of
 * magnumaf/include/magnumaf/field_terms/field_term.hpp:12-51 with its
 * H_in_Apm(const State&) and Energy_in_J(const State&). */

/* DemagField(Mesh mesh, ...) (magnumaf/src/field_terms/micro/demag_field.cpp:211-213):
 * the Newell tensor is computed on the GPU in FP64 and transformed once.  The term holds one set of
 * spectral work buffers: evaluations of it on different streams must not overlap in time (synchronous
 * calls never do; concurrent ensembles need one DemagField per member). */
int maf_term_demag_create(maf_term* out, int nx, int ny, int nz, double dx, double dy, double dz);
/* DemagField from a reduced spectral tensor saved earlier with maf_term_demag_tensor (the disk cache of
 * get_Nfft(mesh, verbose, caching=true), demag_field.cpp:185-199, and util/cache_manager.cpp:49-116). */
int maf_term_demag_create_from_tensor(maf_term* out, int nx, int ny, int nz, double dx, double dy, double dz,
                                      const double* tensor_host);
/* ExchangeField(double A) (magnumaf/src/field_terms/micro/exchange_field.cpp:115-157) */
int maf_term_exchange_create(maf_term* out, double A);
/* DmiField(double D, std::array<double,3> D_axis) (magnumaf/src/field_terms/micro/dmi_field.cpp:15,41-110) */
int maf_term_dmi_create(maf_term* out, double D, double axis_x, double axis_y, double axis_z);
/* DmiField(af::array D_constants, D_axis) (dmi_field.cpp:17-19); D_field is [nz][ny][nx] */
int maf_term_dmi_field_create(maf_term* out, int nx, int ny, int nz, const double* D_field_host, double axis_x,
                              double axis_y, double axis_z);
/* BulkDMIExchangeField(double D, double A) (magnumaf/src/field_terms/micro/bulk_dmi_exchange_field.cpp:9,95-119) */
int maf_term_bulkdmi_exchange_create(maf_term* out, double D, double A);
/* UniaxialAnisotropyField(double Ku1, std::array<double,3> axis)
 * (magnumaf/src/field_terms/micro/uniaxial_anisotropy_field.cpp:11-12,58-89) */
int maf_term_uniaxial_create(maf_term* out, double Ku1, double axis_x, double axis_y, double axis_z);
/* UniaxialAnisotropyField with an Ku1 field and/or an axis field (uniaxial_anisotropy_field.cpp:14-31);
 * Ku1_field [nz][ny][nx] or NULL (then Ku1 is used), axis_field [3][N] or NULL (then the axis is used) */
int maf_term_uniaxial_field_create(maf_term* out, int nx, int ny, int nz, const double* Ku1_field_host, double Ku1,
                                   const double* axis_field_host, double axis_x, double axis_y, double axis_z);
/* CubicAnisotropyField(Kc1, Kc2, Kc3, c1, c2) (magnumaf/src/field_terms/micro/cubic_anisotropy_field.cpp:9-22,61-113);
 * returns MAF_ERR_BADARG where the reference exits, i.e. when |c1.c2| > 1e-12 */
int maf_term_cubic_create(maf_term* out, double Kc1, double Kc2, double Kc3, const double c1[3], const double c2[3]);
/* SpinTransferTorqueField(polarization, eta_damping, eta_field, j_e, fl_thickness)
 * (magnumaf/src/field_terms/micro/spin_transfer_torque_field.cpp:7-28): H = -j_e hbar / (2 e mu0 Ms d)
 * (eta_d m x p + eta_f p) with the normalised polarisation p [3][N]; zero where Ms = 0 */
int maf_term_stt_create(maf_term* out, int nx, int ny, int nz, const double* polarization_host, double eta_damping,
                        double eta_field, double j_e, double fl_thickness);
/* DemagFieldPBC() (magnumaf/src/field_terms/micro/demag_field_pbc.cpp:36-71): periodic demag through the
 * scalar potential on the mesh's own grid (transforms of nx, ny, nz, no tensor). The plan is made for the
 * mesh of the first state evaluated (and remade when a state of another mesh is evaluated); nx must be even
 * (MAF_ERR_UNSUPPORTED otherwise: the reference's C2R returns 2*(nx/2) columns) */
int maf_term_demag_pbc_create(maf_term* out);
/* SparseExchangeField(A, mesh) and SparseExchangeField(A_field, mesh)
 * (magnumaf/src/field_terms/micro/sparse_exchange_field.cpp:8-18,25-101,183-330, COO assembly, the default):
 * H = (M m) / Ms with the 7-point matrix M of the mesh nx*ny*nz.  A_field_host [nz][ny][nx] or NULL
 * (then the scalar A: neighbours inside the mesh weigh 2A/(mu0 d^2), no diagonal); with a field the
 * weights are 2A_i/(mu0 d^2) * 2A_nb/(A_nb+A_i), the diagonal minus their sum, rows with A_i = 0 empty.
 * The matrix is not stored: the kernel forms each row's weights. Also ExchangeField(A, mesh)
 * (python/magnumaf.pyx:1172-1195) */
int maf_term_sparse_exchange_create(maf_term* out, int nx, int ny, int nz, const double* A_field_host, double A);
/* ExchangeFieldPBC(A, mesh) / (A_field, mesh) (magnumaf/src/field_terms/micro/exchange_field_pbc.cpp:9-19,31-225):
 * the harmonic-mean matrix above with periodic neighbours in x, y and z, also for a scalar A */
int maf_term_exchange_pbc_create(maf_term* out, int nx, int ny, int nz, const double* A_field_host, double A);
/* ExternalField(af::array zee) (magnumaf/src/field_terms/micro/external_field.cpp:9,28-48); h is [3][N] */
int maf_term_external_create(maf_term* out, int nx, int ny, int nz, const double* h_host);
/* ExternalField with one field vector for every cell (set_homogeneous_field, external_field.cpp:19-25) */
int maf_term_external_uniform_create(maf_term* out, double hx, double hy, double hz);
int maf_term_destroy(maf_term t);
/* FieldTerm::H_in_Apm (field_term.hpp:15,55-64); FP32-field states return their FP32 field widened */
int maf_term_H(maf_term t, maf_state s, double* H_host);
/* H_in_Apm of an FP32-field state in its native FP32 */
int maf_term_H_f32(maf_term t, maf_state s, float* H_host);
/* FieldTerm::Energy_in_J (field_term.hpp:19-20,66-86; micro_term.hpp:18-30) */
int maf_term_E(maf_term t, maf_state s, double* E);
/* DemagField only: the symmetry-reduced real spectral tensor, FP64,
 * [ncomp][nz == 1 ? 1 : nz+1][ny+1][nx+1], ncomp = 6 (xx,xy,xz,yy,yz,zz) or 4 (xx,xy,yy,zz) when nz == 1 */
int maf_term_demag_tensor(maf_term t, double* host);
/* DemagField only: the real-space Newell tensor on the padded grid, [6][Pz][Py][Px].
 * symmetric == 0: the reference's setup_N values (DemagField::calc_N, demag_field.cpp:104-121,207-209,
 *                 in the x-fastest layout);
 * symmetric == 1: the parity-exact tensor the spectral pipeline transforms: values at (|j0|,|j1|,|j2|)
 *                 with each component's parity sign, odd components zero on their Nyquist planes. */
int maf_term_demag_real_tensor(maf_term t, double* host, int symmetric);

/* ------------------------------------------------------------ Integrator ---
 * LLGIntegrator(double alpha, vec_uptr_FieldTerm terms, std::string scheme = "RKF45",
 *               Controller(hmin, hmax, atol, rtol), bool dissipation_term_only)
 * (magnumaf/include/magnumaf/integrators/llg_integrator.hpp:28-44,
 *  magnumaf/include/magnumaf/integrators/controller.hpp:16-17).
 * scheme: "RKF45", "DP45" or "BS23".  alpha_field ([nz][ny][nx]) may be NULL.
 * The integrator keeps its own reference to each term. */
int maf_llg_create(maf_llg* out, double alpha, const double* alpha_field_host, int nx, int ny, int nz,
                   const maf_term* terms, int nterms, const char* scheme, double hmin, double hmax, double atol,
                   double rtol, int dissipation_term_only);
int maf_llg_destroy(maf_llg l);
/* Python add_terms() (python/magnumaf.pyx, LLGIntegrator.add_terms) */
int maf_llg_add_term(maf_llg l, maf_term t);
/* LLGIntegrator::alpha setter */
int maf_llg_set_alpha(maf_llg l, double alpha);
/* LLGIntegrator::step -> AdaptiveRungeKutta::step (adaptive_runge_kutta.cpp:39-71) */
int maf_llg_step(maf_llg l, maf_state s);
/* n consecutive steps */
int maf_llg_steps(maf_llg l, maf_state s, int n);
/* LLGIntegrator::E (llg_integrator.cpp:41) */
int maf_llg_E(maf_llg l, maf_state s, double* E);
/* Effective field of all terms (LLGIntegrator::h_addr / fheff, llg_integrator.cpp:11-16,112) */
int maf_llg_heff(maf_llg l, maf_state s, double* H_host);
int maf_llg_heff_f32(maf_llg l, maf_state s, float* H_host);
/* Effective field from a device-resident m (float* for FP32-field states, double* for FP64 states)
 * into a device-resident H of the same type, on the state's stream; no synchronisation. */
int maf_llg_heff_device(maf_llg l, maf_state s, const void* m_dev, void* H_dev);
/* LLGIntegrator::fheff over n host magnetisations in a row (each normalised as by maf_state_set_m):
 * m_host[i] double [3][N] -> H_host[i] (float [3][N] for FP32-field states, double for FP64).  The
 * copy of m[i+1] in, the evaluation of m[i] and the copy of H[i-1] out overlap on three streams (use
 * pinned host memory for full link bandwidth).  The state keeps the last m.  No counterpart in the
 * reference beyond calling H_in_Apm n times. */
int maf_llg_heff_pipeline(maf_llg l, maf_state s, const double* const* m_host, void* const* H_host, int n);
/* maf_llg_heff_pipeline with FP32 host magnetisations (the reference's f32 State arrays; the field of an
 * f32 m is the FP32 form's, demag_field.cpp:217-221): half the host->device bytes; each m is widened to
 * FP64 on the device (exactly) before the same normalisation. */
int maf_llg_heff_pipeline_m32(maf_llg l, maf_state s, const float* const* m_host, void* const* H_host, int n);
/* Autotuner (no counterpart in the reference): the compile-time passes have two kernel variants each --
 * y-pass column tile (choices[0]: 0 default, 1 doubled), z convolution (choices[1]: 1 transforms in
 * registers, 0 shared-memory stages), x-inverse epilogue run length (choices[2]: 2 or 4 cells, 0 = the
 * build's default).  Times both configurations on this state's mesh and precision (one warm-up, then the
 * mean of reps evaluations, CUDA events between passes), keeps the faster variant per pass in the
 * DemagField (shared by every integrator that holds it) and returns the choices; pass_ms (optional, 10
 * values) receives the per-pass times of the two configurations.  Every variant computes the same field
 * up to rounding. */
int maf_llg_autotune(maf_llg l, maf_state s, int reps, int choices[3], double* pass_ms);
/* The autotuner's full search: four configurations of the passes are timed (defaults; all alternatives;
 * and two mixed ones); the y passes' column tile is chosen for both, then the forward pass's pipelining
 * and radix sequence and the inverse pass's radix sequence each from the configurations with that tile,
 * the z convolution and the x-inverse run length per pass.  choices[5] = {cols_wide, convz_reg, xinv_run,
 * cols_pipe, cols_plan}, cols_plan: 0 both y passes 16 16 R, 1 both 16 R 16, 2 the inverse only, 3 the
 * forward only; pass_ms (optional) receives 4 x 5 per-pass times; the
 * result is cached per (mesh, precision, term kinds) for the process, and *cached (optional) reports a
 * cache hit (no timing then). */
int maf_llg_autotune_ex(maf_llg l, maf_state s, int reps, int choices[5], double* pass_ms, int* cached);
int maf_term_demag_get_tune_ex(maf_term t, int choices[5]);
int maf_term_demag_set_tune_ex(maf_term t, const int choices[5]);
int maf_term_demag_get_tune(maf_term t, int choices[3]);
int maf_term_demag_set_tune(maf_term t, const int choices[3]);
/* Runs every pass of this DemagField with the run-time-plan kernels (the ones the batched passes of
 * maf_stoch_batch_set_fused use) instead of the compile-time ones; on = 0 restores the default.  Both
 * compute the same field up to rounding (no counterpart in the reference). */
int maf_term_demag_set_generic(maf_term t, int on);
/* maf_llg_heff_device with a CUDA event after every pass kernel: synchronises and
 * returns each pass's duration in ms (the instrumentation LLGIntegrator::time_heff,
 * llg_integrator.cpp:11-16, and the per-term timers of field_term.hpp:49-86 provide,
 * at pass granularity).  Pass names come from maf_llg_pass_name. */
int maf_llg_heff_device_profile(maf_llg l, maf_state s, const void* m_dev, void* H_dev, double* pass_ms,
                                int max_passes, int* npasses);
int maf_llg_pass_name(maf_llg l, maf_state s, int index, char* buf, int buflen);
/* One Runge-Kutta attempt of the integrator's scheme with step dt from the state's m
 * (AdaptiveRungeKutta's stage loop, adaptive_runge_kutta.cpp:113-173; the state is not
 * changed) with a CUDA event after every kernel: synchronises and returns the duration in
 * ms of each interval -- the FP32 copy of m ("stage_m32"), every stage's combine
 * ("rk_combine_kN": N = FP64 k buffers read) and field passes, and the finalize
 * ("rk_finalize_kN": sumbk, error norm and candidate from N distinct k buffers).  Names
 * come from maf_llg_profile_name (valid until the next profile on this integrator). */
int maf_llg_attempt_profile(maf_llg l, maf_state s, double dt, double* ms_out, int max_entries, int* n_entries);
int maf_llg_profile_name(maf_llg l, int index, char* buf, int buflen);
/* dm/dt = LLGIntegrator::f(state) (llg_integrator.cpp:18-38) */
int maf_llg_dmdt(maf_llg l, maf_state s, double* dmdt_host);
/* LLGIntegrator::integrate_dense (llg_integrator.cpp:68-104): rows of (t, <mx>, <my>, <mz>),
 * the first row being the initial state; at most max_rows rows are written. */
int maf_llg_integrate_dense(maf_llg l, maf_state s, double time_in_s, double write_every_dt_in_s, double* rows,
                            int max_rows, int* nrows);
/* One Runge-Kutta attempt of `scheme` ("RKF45", "DP45", "BS23") with step dt from the
 * state's m, without the step controller: AdaptiveRungeKutta::RKF45/DP45/BS23(state, dt, err)
 * (adaptive_runge_kutta.cpp:75-173, 496-529).  Writes m + sumbk (not normalised) and the
 * scaled error norm; the state is not changed. */
int maf_llg_rk_attempt(maf_llg l, maf_state s, const char* scheme, double dt, double* m_new_host, double* err);
/* LLGIntegrator::relax (llg_integrator.cpp:43-66) */
int maf_llg_relax(maf_llg l, maf_state s, double precision, int eval_E);
/* ------------------------------------------------------- Stochastic LLG ---
 * Stochastic_LLG(alpha, T, dt, State, terms, smode) (magnumaf/include/magnumaf/integrators/stochastic_llg.hpp:9-18,
 * magnumaf/src/integrators/stochastic_integrator.cpp:8-87): fixed-step "Heun", "SemiHeun" or "detRK4" with the
 * thermal field h_th = sqrt(2D/dt) N(0,1), D = alpha kB T / (gamma mu0 Ms dV).  The reference seeds ArrayFire's
 * Philox engine from the wall clock; here the thermal field of noise index n is a pure function of
 * (seed, member, n, cell) (counter-based Philox-4x32-10), so runs are reproducible and every ensemble member has
 * its own stream.  Heun step s uses index s for the predictor (the previous step's field) and s+1 for the
 * corrector (stochastic_integrator.cpp:13-15). */
typedef struct maf_stoch_s* maf_stoch;
int maf_stochastic_llg_create(maf_stoch* out, double alpha, double T, double dt, const maf_term* terms, int nterms,
                              const char* smode, unsigned long long seed, unsigned member);
int maf_stochastic_llg_destroy(maf_stoch h);
/* Stochastic_Integrator::step (stochastic_integrator.cpp:42-57) */
int maf_stochastic_llg_step(maf_stoch h, maf_state s);
int maf_stochastic_llg_steps(maf_stoch h, maf_state s, int n);
/* Stochastic_LLG::E (stochastic_llg.cpp:6) */
int maf_stochastic_llg_E(maf_stoch h, maf_state s, double* E);
/* the thermal field of noise index `index` on this state's mesh, [3][N] (for checking and diagnostics) */
int maf_stochastic_llg_noise(maf_stoch h, maf_state s, unsigned long long index, double* out_host);
/* Stochastic_Integrator::get_calls */
int maf_stochastic_llg_calls(maf_stoch h, unsigned long long* calls);

/* Batched ensemble (no counterpart in the reference, which steps one integrator
 * at a time): member i is integrator i stepping state i (distinct states on
 * distinct streams; any meshes).  maf_stoch_batch_steps advances every member by
 * nsteps steps; after a first eager step, pairs of steps of all members replay
 * one captured CUDA graph in which each member runs on its own stream, so small
 * members run concurrently.  Results are bit-identical to calling
 * maf_stochastic_llg_steps on each member.  Do not change a member's stream
 * while it belongs to a batch. */
typedef struct maf_stoch_batch_s* maf_stoch_batch;
int maf_stoch_batch_create(maf_stoch_batch* out, const maf_stoch* integrators, const maf_state* states, int n);
int maf_stoch_batch_destroy(maf_stoch_batch b);
int maf_stoch_batch_steps(maf_stoch_batch b, int nsteps);
/* Batched passes (no counterpart in the reference): with on = 1 the next capture records every pass of
 * a step as ONE launch for all members -- each CTA takes a (member, tile) pair from a device work table
 * and runs that tile of the member's run-time-plan kernel -- instead of one launch per member and pass.
 * Members must be 2-D meshes with one non-periodic DemagField, scalar parameters, one scheme, dt and
 * precision; a batch that does not qualify keeps the per-member graph.  A member's trajectory equals
 * the one its own integrator computes with maf_term_demag_set_generic(demag, 1), bit for bit.
 * maf_stoch_batch_is_fused reports whether the current graph runs the batched passes. */
int maf_stoch_batch_set_fused(maf_stoch_batch b, int on);
int maf_stoch_batch_is_fused(maf_stoch_batch b, int* active);

/* ------------------------------------------------------------- LBFGS ---
 * LBFGS_Minimizer(terms, tolerance = 1e-6, maxIter = 230)
 * (magnumaf/include/magnumaf/solvers/lbfgs_minimizer.hpp:9-12, magnumaf/src/solvers/lbfgs_minimizer.cpp:19-505):
 * m = 5 LBFGS on the normalised magnetisation, gradient m x (m x H), More-Thuente line search. */
typedef struct maf_lbfgs_s* maf_lbfgs;
int maf_lbfgs_create(maf_lbfgs* out, const maf_term* terms, int nterms, double tolerance, int maxIter);
int maf_lbfgs_destroy(maf_lbfgs h);
int maf_lbfgs_add_term(maf_lbfgs h, maf_term t);
/* LBFGS_Minimizer::Minimize (lbfgs_minimizer.cpp:55-198): minimises in place, returns the final energy */
int maf_lbfgs_minimize(maf_lbfgs h, maf_state s, double* E);
/* iterations of the last minimisation, energy/gradient evaluations so far, max|m x (m x H)| at the end */
int maf_lbfgs_stats(maf_lbfgs h, unsigned long long* iterations, unsigned long long* fevals, double* grad_max);

/* current step size h and the controller counters {accepted, rejected, hmin, hmax}
 * (controller.hpp:26-31) */
int maf_llg_get_h(maf_llg l, double* h);
int maf_llg_counters(maf_llg l, unsigned long long out[4]);
/* Controller state for checkpoints, so that a resumed run takes the same step sizes:
 * {h, errold, reject, hnext, n_accepted, n_reject, n_hmin, n_hmax, accumulated_steps}
 * (controller.hpp:26-31, adaptive_runge_kutta.hpp:39) */
int maf_llg_get_controller_state(maf_llg l, double out[9]);
int maf_llg_set_controller_state(maf_llg l, const double in[9]);
/* State::steps, for restoring a checkpoint */
int maf_state_set_steps(maf_state s, unsigned long long steps);

/* ------------------------------------------------------- String method ---
 * StringMethod(state, inputimages, n_interp, dt, llg)
 * (magnumaf/include/magnumaf/solvers/string_method.hpp:9-39, magnumaf/src/solvers/string_method.cpp:12-46):
 * n_interp images on the device, linearly interpolated along the arc length of
 * the input images (at least two, on the state's mesh) and normalised.  The
 * llg handle is borrowed and must outlive the string; all images are stepped
 * with it, sharing its step-size controller as in the reference. */
typedef struct maf_string_s* maf_string;
int maf_string_create(maf_string* out, maf_state state, const maf_state* inputimages, int n_inputimages, int n_interp,
                      double dt, maf_llg llg);
int maf_string_destroy(maf_string h);
/* Batched integration (no counterpart in the reference, whose integrate() steps the images one after the
 * other with the shared adaptive integrator, string_method.cpp:108-121): with substeps > 0 every image
 * advances its dt by `substeps` fixed RK4 steps of dt/substeps (the deterministic RK4 of
 * stochastic_integrator.cpp:34-40, the llg's alpha and terms, its own demag buffers and CUDA stream), and
 * all images are advanced together by one CUDA graph of the ensemble batch (maf_stoch_batch_*); the arc
 * lengths, re-interpolation and energies stay the reference's.  substeps = 0 returns to the reference's
 * integration.  Needs a scalar alpha and a scalar Ms. */
int maf_string_set_batched(maf_string h, int substeps);
/* StringMethod::step (string_method.cpp:128-132): every image integrated for dt,
 * arc lengths x (FrobeniusNorm of image differences), linear re-interpolation */
int maf_string_step(maf_string h);
/* StringMethod::calc_E (string_method.cpp:48-55): E[i] of every image, E_out[n_interp] */
int maf_string_calc_E(maf_string h, double* E_out);
/* StringMethod::run (string_method.cpp:174-314): returns the lowest barrier max(E) - E[0] in dE and writes
 * the reference's .dat files and gnuplot script under filepath (no VTK files, gnuplot is not run);
 * iterations (optional) receives the number of string steps taken */
int maf_string_run(maf_string h, const char* filepath, double string_abort_rel_diff, double string_abort_abs_diff,
                   int string_steps, int every_string_to_vti, int verbose, double* dE, int* iterations);
int maf_string_n_images(maf_string h, int* n);
/* current arc-length coordinates x[n_interp] and the regular grid x_interp[n_interp] */
int maf_string_get_x(maf_string h, double* x, double* x_interp);
/* image i as a state handle owned by the string (do not destroy it) */
int maf_string_image(maf_string h, int i, maf_state* image);

/* ------------------------------------------------ learned warm start ---
 * No counterpart in the reference.  A small convolutional network proposes a
 * relaxed magnetisation that the LBFGS minimiser then finishes:
 * y = normalize(m + conv_L(relu(...relu(conv_1(x))))), 3x3 convolutions with zero
 * padding, cin input channels (the first three are m, the others parameter
 * maps), `width` channels in the hidden layers, `depth` layers, FP32.  All
 * array arguments are DEVICE pointers, NCHW: x [B][cin][H][W], y and target
 * [B][3][H][W].  Parameters: per layer W[cout][cin][3][3] then b[cout]. */
typedef struct maf_cnn_s* maf_cnn;
/* BF16 GEMM on the tensor cores (tcgen05.mma, FP32 accumulation in tensor memory), the contraction of
 * the warm-start network's convolutions (no counterpart in the reference): C[M][N] (FP32, row stride ldc)
 * = A[M][K] . B[N][K]^T with A, B BF16 device arrays whose K elements are contiguous (row strides lda,
 * ldb and K multiples of 8, rows 16-byte aligned).  Queued on stream (NULL: the legacy default stream);
 * returns after the stream finished it.  MAF_ERR_TIMEOUT if a bounded tensor-core wait gave up. */
int maf_bf16_gemm(const void* A_dev, int lda, const void* B_dev, int ldb, float* C_dev, int ldc, int M, int N, int K,
                  void* stream);
/* Layer kernels of the warm-start U-net (magnumaf/unet.py; no counterpart in the reference).  Device
 * pointers; activations pixel-major ([pixels][channels], pixel (b, y, x) at row (b H + y) W + x); BF16
 * tensors that feed a GEMM have their channels padded with zeros to Cp, a multiple of 8; every call is
 * queued on stream st (NULL: the legacy default stream) and returns without synchronising. */
/* x [B][C][H][W] FP32 -> act [P][Cp] BF16 and m [P][3] FP32 (channels 0..2) */
int maf_nn_input(const float* x, int B, int C, int H, int W, int Cp, void* act_bf16, float* m, void* st);
/* 3x3 im2col (zero padding): col [P][9 Cp] (tap t = 3 (dy + 1) + (dx + 1)), or colT [9 Cp][P] */
int maf_nn_im2col(const void* act, int B, int H, int W, int Cp, void* col, int transposed, void* st);
/* maf_bf16_gemm without the synchronisation, and with the K range split over `splits` partial slabs
 * work [splits][M][N] summed in split order into C [M][N] */
int maf_nn_gemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K, void* st);
int maf_nn_gemm_splitk(const void* A, int lda, const void* B, int ldb, float* C, int M, int N, int K, int splits,
                       float* work, void* st);
/* out [P][C] = relu?(y + bias) (FP32) and, when outb, its BF16 copy [P][Cp] */
int maf_nn_bias_act(const float* y, int ldy, const float* bias, long long P, int C, int relu, float* out,
                    void* outb, int Cp, void* st);
/* 2x2 average pooling [B][H][W][C] -> [B][H/2][W/2][C] (FP32 and BF16 [.][Cp]) and its backward
 * (din (+)= dout / 4 at the four children) */
int maf_nn_pool(const float* in, int B, int H, int W, int C, float* out, void* outb, int Cp, void* st);
int maf_nn_pool_bwd(const float* dout, int B, int H, int W, int C, float* din, int accumulate, void* st);
/* out [B][H][W][Cp] BF16 = nearest-2x-upsampled a [B][H/2][W/2][Ca] | s [B][H][W][Cs]; backward:
 * da = sum of the four children of the first Ca channels of dcat [P][Cp], ds += the next Cs */
int maf_nn_up_cat(const float* a, int Ca, const float* s, int Cs, int B, int H, int W, void* out, int Cp, void* st);
int maf_nn_up_cat_bwd(const float* dcat, int Cp, int Ca, int Cs, int B, int H, int W, float* da, float* ds,
                      void* st);
/* dY = dA * relu'(A) (FP32 [P][C], and BF16 [P][Cp]) */
int maf_nn_relu_bwd(const float* dA, const float* A, long long P, int C, int relu, float* dY, void* dYb, int Cp,
                    void* st);
/* BF16 [R][C] -> [C][R] */
int maf_nn_transpose(const void* in, long long R, int C, void* out, void* st);
/* adjoint of im2col: dX [P][C] (+)= sum over taps of dcol [P][9 Cp] (first C channels) */
int maf_nn_col2im(const float* dcol, int B, int H, int W, int Cp, int C, float* dX, int accumulate, void* st);
/* db [C] = sum over pixels of dY [P][C] (fixed order) */
int maf_nn_colsum(const float* dY, long long P, int C, float* db, void* st);
/* FP32 weights W [Cout][9][Cin] -> BF16 Wb [Cout][9 Cp] and WtB [9 Cp][CoutP] (zero padded); the
 * weight gradient [Cout][9][Cin] from a GEMM result [Cout][9 Cp] */
int maf_nn_wcast(const float* W32, int Cout, int Cin, int Cp, int CoutP, void* Wb, void* WtB, void* st);
int maf_nn_wgrad(const float* g, int Cout, int Cin, int Cp, float* dW, void* st);
/* y = normalize(m + d) [P][3]; with a target t: per-pixel |y - t|^2, its mean in *loss (device) and
 * dL/dd [P][3] in gd */
int maf_nn_head(const float* m, const float* d, int ldd, const float* t, long long P, float* y, float* gd,
                float* cell_loss, float* loss, void* st);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8), step = the 1-based step count for the bias corrections */
int maf_nn_adam(float* w, const float* g, float* m1, float* m2, long long n, float lr, int step, void* st);
int maf_cnn_create(maf_cnn* out, int cin, int width, int depth, unsigned long long seed);
int maf_cnn_destroy(maf_cnn h);
/* dilation of each layer's 3x3 kernel (n = depth values in 1..64; default 1): layer l reads its input at
 * offsets -d_l, 0, +d_l, which widens the receptive field without pooling */
int maf_cnn_set_dilation(maf_cnn h, const int* dilation, int n);
int maf_cnn_n_params(maf_cnn h, long long* n);
int maf_cnn_get_params(maf_cnn h, float* host);
/* also resets the Adam moments */
int maf_cnn_set_params(maf_cnn h, const float* host);
int maf_cnn_forward(maf_cnn h, const float* x_dev, int B, int H, int W, float* y_dev);
/* loss = mean over the B*H*W cells of |y - target|^2, gradient of every parameter (host, optional) */
int maf_cnn_loss_grad(maf_cnn h, const float* x_dev, const float* target_dev, int B, int H, int W, float* loss,
                      float* grad_host);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8) with learning rate lr; returns the loss before the step */
int maf_cnn_train_step(maf_cnn h, const float* x_dev, const float* target_dev, int B, int H, int W, float lr,
                       float* loss);

/* ------------------------------------------------- no-allocation mean ---
 * No counterpart in the reference.  <m> of a device-resident FP64 field
 * m_dev[3][ncells] (e.g. from maf_state_device_m), with the definition of
 * maf_state_mean_m: sum over cells / number of cells with |m| != 0.  It
 * allocates no device memory, for callers that must not: code sampling <m>
 * between steps while other streams run (cudaMalloc can synchronise the
 * device), or an application that has reserved all free device memory.
 * Its scratch is a fixed 128 KiB static device array per device, which limits
 * ncells to 33554432 (2^25); larger ncells return MAF_ERR_BADARG.
 * CUDA loads the code and that array lazily, on first use in a device's
 * context, and the load allocates device memory and may synchronise the
 * device.  maf_state_create performs that load, so once a state exists on the
 * device no call allocates.  A caller that passes a field it did not get from
 * a state should make one warm-up call before it reserves device memory or
 * starts concurrent streams.  Work is queued on cuda_stream (NULL: the legacy
 * default stream) and the call returns after that stream has finished it.  A
 * state's own stream is non-blocking, so a field of a state must be read on the
 * state's stream (the one given to maf_state_set_stream) or after that stream
 * has been synchronised; otherwise <m> may be taken from a half-updated field.
 * Calls that overlap on one device (other streams or host threads, unordered)
 * share the scratch and race: both results are then undefined. */
int maf_mean_m_noalloc(const double* m_dev, long long ncells, double out[3], void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* MAF_B200_H */
