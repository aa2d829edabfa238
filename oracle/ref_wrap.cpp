// Test infrastructure only.  Compiles the reference's own CPU pieces of the
// solve path in place, from the reference tree (-I <reference>/src), and
// exposes them with C linkage so the oracle can be pinned against them and
// the CPU baseline can run them.  Nothing here is shipped; the output lands
// in oracle/_ref/.
//
// Pieces: the LCG generator (hpl_rand.hpp), the CPU on-the-fly GEMV kernel
// (otf_gemv.cpp through svesim.hpp / fp16sim.hpp on x86), the CPU no-pivot
// LU (sgetrf_nopiv.cpp, naive and the 6-wide OpenMP variant), and the
// parameter search of Higham's HPL-AI matrix (higham_mat_impl.cpp; its
// higham_mat_comp_beta has C linkage already).
#define __HPLAI_DEVICE_MACROS__ 1
#define __host__
#define __device__
#include <cstddef>
#include <cstdint>
int grank = 0;  // declared extern by hpl_rand.hpp:10
#include "hpl_rand.hpp"
#include "otf_gemv.cpp"
#include "sgetrf_nopiv.cpp"
#include "higham_mat_impl.cpp"

extern "C" {
// fill_one_panel_with_rand (hpl_rand.hpp:158-198): FP32 block with the CPU
// calc_diag-order diagonal when the block is square and on the diagonal.
void ref_fill_one_panel_f32(int n, int i0, int j0, int nrow, int ncol, float *a, size_t lda,
                            uint64_t seed, int calc_diag) {
    fill_one_panel_with_rand<float>(n, i0, j0, nrow, ncol, a, lda, seed, calc_diag != 0);
}
// panel_fill_one_with_rand (hpl_rand.hpp:80-129) in FP64: used for the RHS,
// i.e. column j0 = n of the stream (matgen.hpp:419-436).
void ref_panel_fill_f64(int n, int i0, int j0, int nrow, int ncol, double *a, size_t lda,
                        uint64_t seed) {
    panel_fill_one_with_rand<double>(n, i0, j0, nrow, ncol, a, lda, seed, false);
}
double ref_calc_diag(int i, int n, uint64_t seed) { return calc_diag(i, n, seed); }
double ref_mat_elem(int n, int i, int j, int seed) { return mat_elem(n, i, j, seed); }
void ref_rand_pow(uint64_t a, uint64_t c, uint64_t e, uint64_t *oa, uint64_t *oc) {
    RandCoeff r = RandCoeff{a, c}.pow(e);
    *oa = r.a;
    *oc = r.c;
}
void ref_sgetrf_nopiv_naive(int m, int n, float *a, size_t lda) { sgetrf_nopiv_naive(m, n, a, lda); }
void ref_sgetrf_nopiv_tuned(int n, float *a, size_t lda) { sgetrf_nopiv_tuned(n, a, lda); }
unsigned short ref_fp16_bits(float f) {
    fp16 h(f);
    return h.x;
}

// The diagonal-block factor of the CPU baseline: the reference's tuned
// OpenMP no-pivot LU (sgetrf_nopiv_omp<6>, sgetrf_nopiv.cpp:838-940; it
// handles n <= 1280).  The reference does not report bad pivots; this
// wrapper returns 1 + the index of the first zero / non-finite one.
int ref_getrf_diag(int n, float *a, int64_t lda) {
    sgetrf_nopiv_tuned(n, a, (size_t)lda);
    for (int i = 0; i < n; ++i) {
        float v = a[i + lda * i];
        if (v == 0.0f || !(v == v) || v - v != 0.0f) return i + 1;
    }
    return 0;
}

// y = beta y + alpha A x at a 1 x 1 grid, as otf_gemv (panel_gemv.hpp:310-338)
// drives the reference's CPU kernel: row blocks of b in parallel, the b x b
// blocks of a row block in column order; every block off the diagonal is one
// otf_gemv_kernel call (otf_gemv.cpp:5-133) from the LCG state of its first
// element.  A diagonal block goes by 64-row strips as otf_gemv_kernel_diag
// does (panel_gemv.hpp:259-286): the kernel left and right of the strip's
// 64 x 64 diagonal square, and that square row by row with d on the
// diagonal (otf_gemv_small, panel_gemv.hpp:221-237).  Those two are static
// in a header that needs MPI, so their loops are written out here.
void ref_otf_gemv(int n, int b, uint64_t seed, const double *d, double alpha, const double *x, double beta,
                  double *y) {
    const RandCoeff inc1 = RandCoeff::default_vals();
    const RandCoeff jumpn = inc1.pow(n);
    const RandStat s0 = RandStat::initialize(seed);
    auto state = [&](int64_t i, int64_t j) { return inc1.pow((uint64_t)i + (uint64_t)n * (uint64_t)j) * s0; };
    for (int i = 0; i < n; ++i) y[i] = beta == 0.0 ? 0.0 : beta * y[i];
    const int nb = n / b;
#pragma omp parallel for schedule(dynamic, 1)
    for (int pi = 0; pi < nb; ++pi) {
        const int64_t r0 = (int64_t)pi * b;
        for (int pj = 0; pj < nb; ++pj) {
            const int64_t c0 = (int64_t)pj * b;
            if (pi != pj) {
                otf_gemv_kernel(n, b, b, alpha, x + c0, y + r0, state(r0, c0).x);
                continue;
            }
            for (int q = 0; q < b; q += 64) {
                const int bq = b - q < 64 ? b - q : 64;
                if (q) otf_gemv_kernel(n, bq, q, alpha, x + c0, y + r0 + q, state(r0 + q, c0).x);
                RandStat row = state(r0 + q, c0 + q);
                for (int i = 0; i < bq; ++i) {
                    RandStat sj = row;
                    double t = 0.0;
                    for (int j = 0; j < bq; ++j) {
                        double aij = i == j ? d[r0 + q + i] : static_cast<double>(sj);
                        t += aij * x[c0 + q + j];
                        sj = jumpn * sj;
                    }
                    y[r0 + q + i] += alpha * t;
                    row = inc1 * row;
                }
                if (b > q + 64)
                    otf_gemv_kernel(n, bq, b - q - 64, alpha, x + c0 + q + 64, y + r0 + q,
                                    state(r0 + q, c0 + q + 64).x);
            }
        }
    }
}

// y += a A x for Higham's matrix at a 1 x 1 grid, as otf_gemv for HMGen
// (panel_gemv.hpp:362-388) drives the reference's kernels: b x b blocks above
// the diagonal by hmg_gemv_up, below it by hmg_gemv_low, on it by
// hmg_gemv_diag (otf_gemv.cpp:135-316), row blocks in parallel, the blocks of
// a row block in column order.
void ref_higham_gemv(int n, int b, double alpha, double beta, double a, const double *x, double *y) {
    const int nb = n / b;
#pragma omp parallel for schedule(dynamic, 1)
    for (int pi = 0; pi < nb; ++pi)
        for (int pj = 0; pj < nb; ++pj) {
            if (pi < pj)
                hmg_gemv_up(b * pi, alpha, beta, b, b, a, x + b * pj, y + b * pi);
            else if (pi > pj)
                hmg_gemv_low(b * pj, alpha, beta, b, b, a, x + b * pj, y + b * pi);
            else
                hmg_gemv_diag(b * pi, b * pj, alpha, beta, b, b, a, x + b * pj, y + b * pi);
        }
}
}
