// Launch wrappers of the Runge-Kutta / normalisation kernels (llg.cu).
#pragma once
#include "common.cuh"

namespace mafb {

struct KList {
    const double* k[8] = {};
    double c[8] = {};
    int n = 0;
};

void rk_combine(const double* m, const KList& kl, double* out64, float* out32, int64_t n, cudaStream_t st);
// returns the number of partial CTAs; err_dev receives the NaN-propagating max
int rk_finalize(const double* m, const KList& kb, const KList& ke, int form, double atol, double rtol, double* mcand,
                int norm_mode, int64_t N, double* partials, double* err_dev, cudaStream_t st);
void normalize_m(double* m, int64_t N, int mode, unsigned long long* zero_count_dev, cudaStream_t st);
void ms_field_from_m(const double* m, double Ms, double* msf, float* msf32, int64_t N, cudaStream_t st);
// partial-sum blocks of mean_m (its scratch needs 4 per block; out_dev may sit behind them)
int mean_m_blocks();
void mean_m(const double* m, int64_t N, double* scratch, double* out_dev, cudaStream_t st);
void f32_to_f64(const float* a, double* b, int64_t n, cudaStream_t st);
void thermal_field(double* out, int64_t N, double sigma, unsigned long long seed, unsigned member,
                   unsigned long long index, cudaStream_t st);
// LBFGS vector operations; scratch needs red_blocks() + 1 doubles; the reductions synchronise
int red_blocks();
double dot_host(const double* a, const double* b, int64_t n, double* scratch, cudaStream_t st);
double maxabs_host(const double* a, int64_t n, double* scratch, cudaStream_t st);
void axpby(double* out, double a, const double* x, double b, const double* y, int64_t n, cudaStream_t st);
// Device-resident steps of the LBFGS two-loop recursion (no host synchronisation):
// *out = a . b (the same partial sums and order as dot_host), and
// q = 1 q + c y with c = -(rho *d) (alpha_out: t = rho *d, written by one thread)
// or c = *alpha_in - rho *d (the reference's operations; the multiply-add may round
// differently in the last bit from axpby's).
void dot_dev(const double* a, const double* b, int64_t n, double* scratch, double* out, cudaStream_t st);
// reduce_host's mode (0 dot, 1 NaN-propagating max |a|, 2 squared difference) into a device scalar
void reduce_dev(const double* a, const double* b, int64_t n, int mode, double* scratch, double* out, cudaStream_t st);
void axpby_rho(double* q, const double* y, const double* d, double rho, const double* alpha_in, double* alpha_out,
               int64_t n, cudaStream_t st);
void normalize_combine(double* m, const double* wa, double stp, const double* s, int64_t N, cudaStream_t st);
// string method: sum (a-b)^2 over n values (synchronises), out = a + (c1 (b - a)) / c2
double sqdiff_host(const double* a, const double* b, int64_t n, double* scratch, cudaStream_t st);
void lerp(double* out, const double* a, const double* b, double c1, double c2, int64_t n, cudaStream_t st);
// *c += 1 on the device (the step counter of a captured stochastic step)
void inc_counter(unsigned long long* c, cudaStream_t st);

}  // namespace mafb
