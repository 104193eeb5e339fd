// Host-side engine objects behind the C ABI: device buffers, the demag plan,
// the field evaluator and the adaptive Runge-Kutta integrator.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "fft_engine.cuh"
#include "local_terms.cuh"

namespace mafb {

enum Precision : int { PREC_FP64 = 0, PREC_FP32_FIELD = 1 };

// Owning device allocation.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t n) {
        release();
        if (n) MAF_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    void ensure(size_t n) { if (bytes < n) alloc(n); }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct MeshDims {
    int nx = 0, ny = 0, nz = 0;
    double dx = 0, dy = 0, dz = 0;
    int64_t N() const { return (int64_t)nx * ny * nz; }
    Geom geom() const { return Geom{nx, ny, nz, N(), dx, dy, dz}; }
    bool operator==(const MeshDims& o) const {
        return nx == o.nx && ny == o.ny && nz == o.nz && dx == o.dx && dy == o.dy && dz == o.dz;
    }
};

// Twiddle tables W_L^k, k in [0, L), per length and precision.
class Twiddles {
  public:
    const void* get(int L, bool fp64);
    // the table of get() followed by the per-stage twiddle rows of a radix
    // sequence (fft_ct.cuh: entry (jm, r - 1) of the stage with NS, RAD is
    // W_L^(r jm L / (NS RAD))), for the compile-time transforms of length L
    const void* get_ct(int L, bool fp64, const int* radix, int nstages);
  private:
    std::map<std::pair<int, int>, DevBuf> tables_;
};

FFTPlan make_fft_plan(int L, const void* tw);  // throws MAF_ERR_UNSUPPORTED for primes > 13

// Output handling of the last field pass.
enum Epilogue : int {
    EPI_H = 0,      // write H (precision R) to out[3][N]
    EPI_LLG = 1,    // write k = scale * dm/dt (double) to out[3][N]
    EPI_EDENS = 2,  // accumulate the energy of the term list (double partial sums per CTA)
    EPI_EGRAD = 3,  // energy partials and the LBFGS gradient m x (m x H) (double) to out[3][N]
};

struct LLGParams {
    double c_prec = 0;             // -gamma/(1+alpha^2)
    double c_damp = 0;             // -alpha*gamma/(1+alpha^2)
    const double* alpha = nullptr; // optional alpha field [N]
    int dissipation_only = 0;
    double scale = 1.0;            // dt (RKF45/DP45) or 1 (BS23)
    const double* m64 = nullptr;   // state m in FP64 for the cross products
    // thermal field sigma * xi(seed, member, noise_index, cell) added to H (stochastic LLG)
    double sigma = 0.0;
    unsigned long long seed = 0;
    unsigned member = 0;
    unsigned long long noise_index = 0;
    // when set, the stream index is noise_mul * (*noise_base) + noise_index, read on
    // the device: a captured CUDA graph replays with the step counter it advances
    const unsigned long long* noise_base = nullptr;
    unsigned noise_mul = 0;
    __host__ __device__ unsigned long long stream_index() const {
#ifdef __CUDA_ARCH__
        return noise_base ? noise_mul * (*noise_base) + noise_index : noise_index;
#else
        return noise_index;
#endif
    }
};

struct EpilogueArgs {
    int kind = EPI_H;
    void* out = nullptr;           // H (R) or k (double)
    double* partials = nullptr;    // EPI_EDENS: one double per CTA
    LLGParams llg;
    int edge_exchange = 1;         // EPI_EDENS: exchange energy uses h_withedges
    double* energy_dev = nullptr;  // EPI_EDENS/EGRAD: leave the summed energy density (before the cell
                                   // volume) on the device here instead of reading it back
};

// Optional CUDA-event marks recorded after every pass kernel of a field
// evaluation (used to time the passes individually).
struct PassMarks {
    std::vector<cudaEvent_t> ev;
    std::vector<const char*> names;
    void mark(cudaStream_t st, const char* name) {
        cudaEvent_t e;
        MAF_CUDA(cudaEventCreate(&e));
        MAF_CUDA(cudaEventRecord(e, st));
        ev.push_back(e);
        names.push_back(name);
    }
    ~PassMarks() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

struct MsInfo {
    double Ms = 0;                 // scalar Ms (used when field == nullptr)
    const double* field64 = nullptr;
    const float* field32 = nullptr;
};

// Kernel variants of the compile-time passes, chosen per demag plan (defaults,
// or measured by maf_llg_autotune): y-pass column tile doubled, z convolution
// with register transforms (nz <= 16) or shared-memory stages, x-inverse
// epilogue on runs of 2 or 4 cells (0: the build's default).
struct TuneChoice {
    int cols_wide = 0;
    int convz_reg = 1;
    int xinv_run = 0;
    int cols_pipe = 1;  // forward y pass: persistent kernel staging the next tile's input (cp.async)
    int cols_plan = 0;  // y passes' radix sequences: 0 both 16 16 R, 1 both 16 R 16, 2 inverse only 16 R 16,
                        // 3 forward only 16 R 16
    int generic = 0;    // 1: the run-time-plan kernels for every pass (as the batched passes run)
};

// Demag plan: the symmetry-reduced real spectral Newell tensor and the
// spectral work buffers for one mesh.
class Demag {
  public:
    TuneChoice tune;
    // tensor_host: a reduced spectral tensor from download_tensor (e.g. a disk
    // cache) to upload instead of computing it
    // pbc: the periodic scalar-potential form of DemagFieldPBC
    // (demag_field_pbc.cpp:36-71): transforms of the mesh's own lengths, no
    // tensor; the z (or, for nz == 1, y) pass applies the discrete Poisson
    // operator instead of the tensor product.
    Demag(const MeshDims& md, cudaStream_t st, const double* tensor_host = nullptr, bool pbc = false);
    const MeshDims& mesh() const { return md_; }
    bool pbc() const { return pbc_; }
    int Px() const { return pbc_ ? md_.nx : 2 * md_.nx; }
    int Py() const { return pbc_ ? md_.ny : 2 * md_.ny; }
    int Pz() const { return md_.nz == 1 ? 1 : (pbc_ ? md_.nz : 2 * md_.nz); }
    int nxh() const { return Px() / 2 + 1; }
    int ncomp() const { return md_.nz == 1 ? 4 : 6; }
    // Passes 1..4: spectral convolution of Ms*m, result left in the half-spectrum
    // buffer for the fused x-inverse epilogue.
    template <typename R> void forward_conv(const R* m, const MsInfo& ms, cudaStream_t st, PassMarks* marks = nullptr);
    // Pass 5: x-inverse + local terms + epilogue (called by the field evaluator).
    template <typename R>
    void inverse_x_epilogue(const R* m, const MsInfo& ms, const TermList& tl, const EpilogueArgs& ep,
                            cudaStream_t st, int* nblocks_out, PassMarks* marks = nullptr);
    // reduced real spectral tensor in FP64 [ncomp][kz][ky][kx] (host copy for tests)
    void download_tensor(double* host, cudaStream_t st) const;
    void download_real_tensor(double* host, bool symmetric, cudaStream_t st);  // [6][Pz][Py][Px]
    size_t tensor_elems() const { return (size_t)ncomp() * (md_.nz == 1 ? 1 : md_.nz + 1) * (md_.ny + 1) * nxh(); }
    int pitch() const { return pitch_; }
    template <typename R> int edens_blocks() const;
    // buffers and tables of the generic passes, for the batched passes (batch.cu)
    template <typename R> cplx_t<R>* spectrum() { return S1<R>(); }
    template <typename R> const R* tensor_data() { return tensor<R>(); }
    const void* twiddles(int L, bool fp64) { return tw_.get(L, fp64); }
    Twiddles& twiddle_tables() { return tw_; }

  private:
    template <typename R> const R* tensor() ;
    template <typename R> cplx_t<R>* S1();
    template <typename R> cplx_t<R>* S2();
    void build_tensor(cudaStream_t st);

    MeshDims md_;
    bool pbc_ = false;
    int pitch_;  // complex row pitch of the half spectrum (>= nxh)
    DevBuf Nred64_, Nred32_;
    DevBuf S1_64_, S2_64_, S1_32_, S2_32_;
    Twiddles tw_;
};

// Field-term objects (the C ABI's maf_term).
struct Term {
    int kind = TK_DEMAG;
    double p[12] = {};
    DevBuf f0, f1;                   // optional parameter fields (FP64)
    int64_t field_cells = 0;         // cells of the mesh f0/f1 were given on (0: no field)
    std::unique_ptr<Demag> demag;    // TK_DEMAG (DemagFieldPBC: created for the first state's mesh)
    MeshDims demag_mesh;
    bool demag_pbc() const { return kind == TK_DEMAG && p[0] != 0.0; }
    TermDesc desc() const {
        TermDesc d;
        d.kind = kind;
        for (int i = 0; i < 12; ++i) d.p[i] = p[i];
        d.f0 = f0.p ? f0.as<double>() : nullptr;
        d.f1 = f1.p ? f1.as<double>() : nullptr;
        return d;
    }
};

// Device-resident State.
struct StateD {
    MeshDims md;
    int precision = PREC_FP64;
    double Ms = 0;
    bool has_Ms_field = false;
    DevBuf m64;        // double [3][N]
    DevBuf m32;        // float  [3][N] staged copy (FP32-field form)
    DevBuf Msf64, Msf32;
    double t = 0;
    unsigned long long steps = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    MsInfo msinfo() const {
        MsInfo mi;
        mi.Ms = Ms;
        if (has_Ms_field) { mi.field64 = Msf64.as<double>(); mi.field32 = Msf32.as<float>(); }
        return mi;
    }
};

// Field evaluation of a list of terms on m (precision R), with one epilogue.
template <typename R>
void eval_terms(const std::vector<Term*>& terms, const MeshDims& md, const R* m, const MsInfo& ms,
                const EpilogueArgs& ep, cudaStream_t st, DevBuf& scratch_partials, double* energy_out,
                PassMarks* marks = nullptr);

// FP64 -> FP32 staging of m
void stage_m32(const double* m64, float* m32, int64_t n, cudaStream_t st);
void widen_m(const float* m32, double* m64, int64_t n, cudaStream_t st);  // FP32 -> FP64, exact

// Newell tensor on the padded grid, one component [Pz][Py][Px] (newell.cu);
// symmetric = true gives the parity-exact tensor the spectral pipeline uses.
void newell_component(double* out, int comp, const MeshDims& md, int Px, int Py, int Pz, bool symmetric,
                      cudaStream_t st);

}  // namespace mafb
