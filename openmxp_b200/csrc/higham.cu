// Higham's HPL-AI test matrix A = L U: L unit lower triangular with every
// strictly lower entry alpha, U unit upper triangular with every strictly
// upper entry beta (HMGen, highammgen.hpp:4-30), so
//   a_ij = beta + alpha*beta*i  (i < j),
//          1    + alpha*beta*i  (i = j),
//          alpha + alpha*beta*j (i > j)         (pmatgen, matgen.hpp:157-208)
// with diagonal vector d_i = 1 + alpha*beta*i (pdiaggen, matgen.hpp:399-417).
// beta follows from a wanted infinity-norm condition number kappa and the
// ratio rho = alpha / beta by bisection on Fasi and Higham's closed-form
// estimate of cond(A, inf) (higham_mat_comp_beta, higham_mat_impl.cpp:
// 36-149, from their hpl-ai-matrix project).
//
// Pieces here: the parameter search (host), the FP32 matrix fill, the FP64
// residual GEMV that regenerates a_ij (otf_gemv for HMGen, panel_gemv.hpp:
// 362-388 with hmg_gemv_*, otf_gemv.cpp:135-316) and ||A||_inf
// (higham_infnorm, panel_norm.hpp:136-175).  The reference's hmg_gemv_diag
// has alpha and beta in each other's places for the diagonal blocks
// (otf_gemv.cpp: its strictly lower entries use beta + ab*j and its strictly
// upper ones alpha + ab*i); the GEMV here uses the generator's entries
// everywhere, so the residual is that of the matrix that was factored.
#include <float.h>
#include <math.h>

#include <vector>

#include "mxp_internal.cuh"

namespace mxp {

mxp_status launch_matgen(int n, uint64_t seed, int diag_rule, float *A, int64_t lda, double *d,
                         double *rowsum, double *rhs, cudaStream_t st);

namespace {

// cond(A, inf) estimate for parameters (a, b): the largest of three candidate
// row sums of A times the largest of two candidate row sums of inv(A).  The
// integer terms are 64-bit (the reference's int terms overflow for n above
// about 37800; below that both give the same bits).
double cond_estimate(int n_, double a, double b) {
    if (std::isnan(a)) a = b / 2;
    const int64_t n = n_;
    const int64_t ip = floor(1. / a) < (double)n ? (int64_t)floor(1. / a) : n;
    const int64_t k = floor((1 + b) / b) < (double)(n - 1) ? (int64_t)floor((1 + b) / b) : n - 1;
    const double first = 1 + (n - 1) * b;
    const double middle = 1 + (2 * k - ip + 1) * a + (n - ip) * b +
                          (-k * k + k + 3 * ip * (ip - 1) / 2 - n * ip + n) * a * b;
    const double last = 1 + (2 * k - n + 1) * a + (-k * k + k + n * (n - 1) / 2) * a * b;
    const double norm_a = std::fmax(std::fmax(first, middle), last);
    const double r = (1 + a) * (1 + b);
    const double inv_first = (1 + a) * (1. / (1 + a) + (r == 0. ? 0. : b * (1 - pow(r, n - 1)) / (1 - r)));
    const double inv_last = pow(1 + a, n) * (1. / (1 + a));
    const double c = norm_a * std::fmax(inv_first, inv_last);
    return std::isinf(c) ? DBL_MAX : c;
}

// Bisection on f(x) = cond(rho x, x) - kappa over [lo, hi] with f(lo) <= 0 <=
// f(hi), to a width of about one ulp of hi; NaN when the bracket is wrong.
double bisect(int n, double kappa, double rho, double lo, double hi) {
    auto f = [&](double x) { return cond_estimate(n, rho * x, x) - kappa; };
    if (f(lo) > 0. || f(hi) < 0.) return NAN;
    for (;;) {
        if (hi - lo < (2. * std::fabs(hi) + 0.5) * DBL_EPSILON) break;
        const double mid = (lo + hi) / 2;
        if (mid == lo || mid == hi) break;
        const double fm = f(mid);
        if (fm == 0.) return mid;
        (fm < 0. ? lo : hi) = mid;
    }
    return hi;
}

constexpr int kFillThreads = 256;

// FP32 entries formed in FP32 from the FP32-rounded parameters with one
// fused multiply-add each; d in FP64.
__global__ void higham_fill_kernel(int n, int64_t j0, float fa, float fb, float fab, float *__restrict__ A,
                                   int64_t lda) {
    const int64_t j = j0 + blockIdx.y;
    const float low = __fmaf_rn(fab, (float)j, fa);
    const float dg = __fmaf_rn(fab, (float)j, 1.0f);
    float *col = A + j * lda;
    for (int64_t i = (int64_t)blockIdx.x * kFillThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kFillThreads)
        col[i] = i < j ? __fmaf_rn(fab, (float)i, fb) : (i == j ? dg : low);
}

__global__ void higham_diag_kernel(int n, double ab, double *__restrict__ d) {
    const int64_t i = (int64_t)blockIdx.x * kFillThreads + threadIdx.x;
    if (i < n) d[i] = __fma_rn(ab, (double)i, 1.0);
}

// y = b y + a A x, A regenerated in FP64: one thread per row summing its
// entries in column order with fused multiply-adds (the same sums as the
// oracle's, bit for bit).  x and the column-constant lower entries
// alpha + ab*j go through shared memory in chunks; the row-constant upper
// entry beta + ab*i and the diagonal stay in registers.
constexpr int kGemvRows = 128;
constexpr int kGemvChunk = 1024;

__global__ void __launch_bounds__(kGemvRows)
higham_gemv_kernel(int n, double alpha, double beta, double a, const double *__restrict__ x, double b,
                   double *__restrict__ y) {
    __shared__ double xs[kGemvChunk];
    __shared__ double cs[kGemvChunk];
    const double ab = alpha * beta;
    const int64_t i = (int64_t)blockIdx.x * kGemvRows + threadIdx.x;
    const double up = __fma_rn(ab, (double)i, beta);
    const double dg = __fma_rn(ab, (double)i, 1.0);
    double t = 0.0;
    for (int64_t j0 = 0; j0 < n; j0 += kGemvChunk) {
        const int len = (int)(n - j0 < kGemvChunk ? n - j0 : kGemvChunk);
        __syncthreads();
        for (int q = threadIdx.x; q < len; q += kGemvRows) {
            xs[q] = x[j0 + q];
            cs[q] = __fma_rn(ab, (double)(j0 + q), alpha);
        }
        __syncthreads();
        // columns j < i use cs, j == i the diagonal, j > i the row constant
        const int lo_end = (int)(i <= j0 ? 0 : (i - j0 < len ? i - j0 : len));
        int q = 0;
        for (; q < lo_end; ++q) t = __fma_rn(cs[q], xs[q], t);
        if (q < len && j0 + q == i) {
            t = __fma_rn(dg, xs[q], t);
            ++q;
        }
        for (; q < len; ++q) t = __fma_rn(up, xs[q], t);
    }
    if (i < n) y[i] = b == 0.0 ? a * t : __fma_rn(b, y[i], a * t);
}

}  // namespace

mxp_status launch_higham_gemv(int n, double alpha, double beta, double a, const double *x, double b, double *y,
                              cudaStream_t st) {
    if (n <= 0 || !x || !y) return fail(MXP_INVALID_ARG, "higham_gemv: bad arguments");
    higham_gemv_kernel<<<(unsigned)cdiv(n, kGemvRows), kGemvRows, 0, st>>>(n, alpha, beta, a, x, b, y);
    MXP_LAUNCHED();
    return MXP_OK;
}

// ||A||_inf: all entries are positive; row i sums to
// sum_{j<i} (alpha + ab j) + (1 + ab i) + (n-1-i)(beta + ab i), accumulated
// here with a running prefix sum of the lower entries.
double higham_infnorm(int n, double alpha, double beta) {
    const double ab = alpha * beta;
    double prefix = 0.0, best = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double row = prefix + std::fma(ab, (double)i, 1.0) + (double)(n - 1 - i) * std::fma(ab, (double)i, beta);
        best = row > best ? row : best;
        prefix += std::fma(ab, (double)i, alpha);
    }
    return best;
}

}  // namespace mxp

using namespace mxp;

extern "C" mxp_status mxp_higham_params(int n, double cond, double rho, double *alpha, double *beta) {
    if (n < 2 || !(cond > 1.0) || !(rho > 0.0) || !alpha || !beta)
        return fail(MXP_INVALID_ARG, "higham_params: need n >= 2, cond > 1, rho > 0 and output pointers");
    const double lo = DBL_EPSILON;
    if (!(cond_estimate(n, rho * lo, lo) - cond < 0.))
        return fail(MXP_INVALID_ARG, "higham_params: cond below the smallest reachable value");
    double hi = 1. / rho;
    for (int k = 1; k < 100; ++k) {
        const double f = cond_estimate(n, rho * hi, hi) - cond;
        if (std::isfinite(f) && f > 0.) break;
        hi *= 0.5;
    }
    double b = bisect(n, cond, rho, lo, hi);
    for (int guard = 0; guard < 64 && rho * b > 1.; ++guard) {
        hi *= 0.25;
        b = bisect(n, cond, rho, lo, hi);
    }
    if (!std::isfinite(b) || rho * b > 1.) return fail(MXP_INVALID_ARG, "higham_params: no parameters for this cond");
    *beta = b;
    *alpha = rho * b;
    return MXP_OK;
}

extern "C" mxp_status mxp_matgen_higham(int n, double alpha, double beta, uint64_t seed, float *d_A, int64_t lda,
                                        double *d_d, double *d_rhs, void *stream) {
    if (n <= 0) return fail(MXP_INVALID_ARG, "matgen_higham: n must be positive");
    if (d_A && lda < n) return fail(MXP_INVALID_ARG, "matgen_higham: lda < n");
    if (!(alpha > 0.0) || !(beta > 0.0)) return fail(MXP_INVALID_ARG, "matgen_higham: alpha and beta must be > 0");
    cudaStream_t st = as_stream(stream);
    const float fa = (float)alpha, fb = (float)beta, fab = fa * fb;
    if (d_A) {
        for (int64_t j0 = 0; j0 < n; j0 += 65535) {
            const int64_t cols = n - j0 < 65535 ? n - j0 : 65535;
            dim3 grid((unsigned)imin64(cdiv(n, kFillThreads), 64), (unsigned)cols);
            // columns j0 .. j0+cols, one per blockIdx.y
            higham_fill_kernel<<<grid, kFillThreads, 0, st>>>(n, j0, fa, fb, fab, d_A, lda);
            MXP_LAUNCHED();
        }
    }
    if (d_d) {
        higham_diag_kernel<<<(unsigned)cdiv(n, kFillThreads), kFillThreads, 0, st>>>(n, alpha * beta, d_d);
        MXP_LAUNCHED();
    }
    if (d_rhs) return launch_matgen(n, seed, MXP_DIAG_ROWSUM, nullptr, n, nullptr, nullptr, d_rhs, st);
    return MXP_OK;
}

extern "C" mxp_status mxp_higham_gemv(int n, double alpha, double beta, double a, const double *d_x, double b,
                                      double *d_y, void *stream) {
    return launch_higham_gemv(n, alpha, beta, a, d_x, b, d_y, as_stream(stream));
}

extern "C" mxp_status mxp_higham_infnorm(int n, double alpha, double beta, double *h_out) {
    if (n <= 0 || !h_out) return fail(MXP_INVALID_ARG, "higham_infnorm: bad arguments");
    *h_out = higham_infnorm(n, alpha, beta);
    return MXP_OK;
}
