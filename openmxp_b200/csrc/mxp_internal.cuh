// Internal declarations shared by the CUDA translation units of libmxp.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/mxp.h"

namespace mxp {

// ---------------------------------------------------------------------------
// Status plumbing
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
mxp_status fail(mxp_status st, const std::string &msg);
mxp_status cuda_fail(cudaError_t e, const char *where);
void count_launch(int n = 1);

#define MXP_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ::mxp::cuda_fail(e_, #call);  \
    } while (0)

#define MXP_LAUNCHED()                                                    \
    do {                                                                  \
        cudaError_t e_ = cudaGetLastError();                              \
        if (e_ != cudaSuccess) return ::mxp::cuda_fail(e_, __func__);     \
        ::mxp::count_launch();                                            \
    } while (0)

// Device status word written by kernels (never by traps): code + two
// integers of detail.  Lives in the workspace.
struct DevStatus {
    int code;   // mxp_status
    int info0;  // e.g. global pivot index
    int info1;  // e.g. timeout site
    int pad;
};

#if defined(__CUDACC__)
__device__ __forceinline__ void report(DevStatus *st, int code, int i0, int i1) {
    if (st && atomicCAS(&st->code, 0, code) == 0) {
        st->info0 = i0;
        st->info1 = i1;
    }
}

// Bounded waits give up after this many nanoseconds of %globaltimer.
constexpr unsigned long long kWaitTimeoutNs = 2000000000ull;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Round-to-nearest FP32 reciprocal without a branch: the hardware FP64
// approximation (rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// r += r (1 - x r) in FP64, then rounded once to FP32.  For a normal FP32 x,
// 1/x is never exactly halfway between two FP32 values and never closer to
// such a point than about 2^-49 (relative), while the refined FP64 value is
// within about 2^-52 of 1/x, so the single rounding gives the correctly
// rounded reciprocal.  It serves where the reciprocal is
// on a latency chain: the IEEE reciprocal of the CUDA runtime takes a
// data-dependent branch that keeps later independent instructions from being
// issued ahead of it.  Checked bit for bit against that reciprocal by
// mxp_check_reciprocal.  Zero, infinite and NaN inputs give NaN (callers
// report such pivots as errors).
__device__ __forceinline__ float rcp_rn_f32(float x) {
    const double d = (double)x;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    return __double2float_rn(r);
}
#endif

// ---------------------------------------------------------------------------
// 64-bit LCG (hpl_rand.hpp:12-78): x <- a*x + c mod 2^64, a = 6364136223846793005.
// ---------------------------------------------------------------------------
struct Aff {
    uint64_t a, c;
};

constexpr uint64_t kLcgA = 6364136223846793005ull;
constexpr uint64_t kLcgC = 1ull;

__host__ __device__ __forceinline__ Aff aff_mul(Aff f, Aff g) {  // f o g
    return Aff{f.a * g.a, f.a * g.c + f.c};
}

__host__ __device__ __forceinline__ Aff aff_pow(Aff f, uint64_t n) {
    Aff r{1ull, 0ull};
    while (n) {
        if (n & 1ull) r = aff_mul(r, f);
        f = aff_mul(f, f);
        n >>= 1;
    }
    return r;
}

__host__ __device__ __forceinline__ uint64_t aff_apply(Aff f, uint64_t x) { return f.a * x + f.c; }

__host__ __device__ __forceinline__ Aff lcg_inc1() { return Aff{kLcgA, kLcgC}; }

// RandStat::initialize(seed) (hpl_rand.hpp:54-57)
__host__ __device__ __forceinline__ uint64_t lcg_stat00(uint64_t seed) {
    return aff_apply(lcg_inc1(), seed);
}

#if defined(__CUDACC__)
// Exact round-to-nearest int64 -> double without the 64-bit converter:
// both 32-bit halves are exact doubles (built by the 2^52 bias trick), and
// hi*2^32 + lo is formed by one fused multiply-add, i.e. a single rounding
// of the exact integer.  Bitwise equal to a correctly rounded conversion.
__device__ __forceinline__ double i64_to_double_rn(uint64_t x) {
    const uint32_t lo = (uint32_t)x;
    const uint32_t hi = (uint32_t)(x >> 32) ^ 0x80000000u;  // signed hi, biased by 2^31
    const double dlo = __hiloint2double(0x43300000, (int)lo) - 4503599627370496.0;   // 2^52
    const double dhi = __hiloint2double(0x43300000, (int)hi) - 4503601774854144.0;   // 2^52 + 2^31
    return __fma_rn(dhi, 4294967296.0, dlo);
}

// RandStat -> double in [-0.5, 0.5] (hpl_rand.hpp:64-66)
__device__ __forceinline__ double lcg_to_double(uint64_t x) {
    return __dmul_rn(i64_to_double_rn(x), 0x1.fffffffffffffP-65);
}
#endif

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Internal operand form of the panel casts and the tensor-core GEMM: one BF16
// value per element, K = b (the single-product TRSM by inverse).
constexpr int kFormBf16 = 3;

// Launchers implemented in the individual translation units ---------------
// Cooperative diagonal-block factorisation (diag_coop.cu): in-place no-pivot LU
// of the n x n block A and, when XU/XL are given, inv(U) -> XU and inv(L) -> XL
// (ld ldx).  tmpU/tmpL: diag_factor_tmp_floats(n) floats each; sync_words: 2
// words of device memory (zeroed on the stream before the launch).
size_t diag_factor_tmp_floats(int n);
// max_grid > 0 caps the number of CTAs (the kernel then shares the GPU with
// work launched on another stream).  inv_stop > 0: the inverses stop before
// the doubling level that joins blocks of that size (finish_inverses_tc
// completes them).
mxp_status launch_diag_factor(int n, float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                              float *tmpU, float *tmpL, unsigned int *sync_words, DevStatus *dst,
                              int pivot_base, cudaStream_t st, int max_grid = 0, int inv_stop = 0);
mxp_status launch_matgen_f64(int n, uint64_t seed, int diag_rule, double *A, int64_t lda,
                             cudaStream_t st);
mxp_status launch_matgen(int n, uint64_t seed, int diag_rule, float *A, int64_t lda, double *d,
                         double *rowsum, double *rhs, cudaStream_t st);

mxp_status launch_getrf_blocked(int n, float *A, int64_t lda, DevStatus *dst, int pivot_base,
                                cudaStream_t st);
mxp_status launch_trsm_runn(int m, int n, const float *U, int64_t ldu, float *B, int64_t ldb,
                            cudaStream_t st);
mxp_status launch_trsm_llnu(int m, int n, const float *L, int64_t ldl, float *B, int64_t ldb,
                            cudaStream_t st);
// tmp: scratch of at least n*n/4 + 64*n floats
mxp_status launch_tri_inv_upper(int n, const float *U, int64_t ldu, float *X, int64_t ldx,
                                float *tmp, cudaStream_t st);
mxp_status launch_tri_inv_lower_unit(int n, const float *L, int64_t ldl, float *X, int64_t ldx,
                                     float *tmp, cudaStream_t st);
mxp_status launch_sgemm_sub(int m, int n, int k, const float *A, int64_t lda, const float *B,
                            int64_t ldb, float *C, int64_t ldc, cudaStream_t st);

// sc_ld: stride (in tiles) between the scale rows of consecutive 128-row
// tiles; <= 0 means ceil(b / 128) (a dense table).
mxp_status launch_cast_left(int form, int m, int b, const float *A, int64_t lda, void *out,
                            int64_t ldk, uint8_t *scales, cudaStream_t st, int sc_ld = 0);
mxp_status launch_cast_right(int form, int m, int b, const float *A, int64_t lda, void *out,
                             int64_t ldk, uint8_t *scales, cudaStream_t st, int sc_ld = 0);
mxp_status launch_half_left_ref(const float *C, int m, int b, int64_t plda, uint16_t *lp,
                                int64_t lplda, cudaStream_t st);
mxp_status launch_half_right_trans_ref(const float *C, int b, int m, int64_t plda, uint16_t *rp,
                                       int64_t rplda, cudaStream_t st);

// How one Schur launch takes its tiles (single-SM kernels only).  grid: CTAs
// to launch (0: one per SM, at most the tile count).  counter: a device int,
// zeroed before the first launch of a pass, from which every CTA of every
// launch that shares it claims tiles (nullptr: static round robin).
// skip_rows x skip_cols: leading corner of C that the pass leaves alone
// (multiples of 128 and 256).
struct SchurSched {
    int grid = 0;
    int *counter = nullptr;
    int skip_rows = 0, skip_cols = 0;
};

// Optional FP8 copy of a store-mode product (FP16/BF16 operands, single-SM
// kernel, n % 256 == 0), with one power-of-two scale per 128 x 128 block of C,
// exactly as the FP8 panel casts of C would write them.  trans == 0 (L panel
// layout): out[i * ldk + j] = E4M3(C(i, j) * 2^e), byte 127 - e at
// sc[(i / 128) * sc_ld + j / 128]; trans == 1 (R panel layout, C holds U
// columns): out[j * ldk + i], scale at sc[(j / 128) * sc_ld + i / 128].
struct F8Out {
    uint8_t *out;
    int64_t ldk;
    uint8_t *sc;
    int sc_ld;
    int trans;
};

mxp_status launch_schur(int form, int m, int n, int k, const void *L, int64_t ldl,
                        const uint8_t *lsc, const void *R, int64_t ldr, const uint8_t *rsc,
                        float *C, int64_t ldc, DevStatus *dst, cudaStream_t st, int store = 0,
                        int lsc_ld = 0, int rsc_ld = 0, int tri_mode = 0, int pair = 0,
                        const SchurSched *sched = nullptr, const F8Out *f8out = nullptr);

mxp_status launch_otf_gemv(int n, uint64_t seed, const double *d, double alpha, const double *x,
                           double beta, double *y, double *partials, int max_splits,
                           cudaStream_t st);
// withhold >= 0: the forward solve never publishes that row block's flag, so
// the blocks that need it give up after the bounded wait (tests of MXP_TIMEOUT).
mxp_status launch_lu_solve(int n, const float *LU, int64_t lda, double *x, int *flags,
                           DevStatus *dst, cudaStream_t st, int withhold = -1);
size_t lu_solve_flag_ints(int n);
// Block triangular solves with the stored FP32 inverses of the b x b diagonal
// blocks (XU: inv(U_kk), XL: inv(L_kk), block k at offset k*xstride, ld b):
// x <- U^{-1} L^{-1} x.  t: 4 b doubles of scratch.  The chain of
// diagonal-block products runs on `side`, the bulk of the trailing updates on
// st, overlapped (side is forked from and joined back to st); ev: 4 events.
// Needs n % b == 0,
// b % 32 == 0, lda % 4 == 0 and 16-byte aligned LU / XU / XL.
bool lu_solve_inv_supported(int n, int b, const float *LU, int64_t lda);
mxp_status launch_lu_solve_inv(int n, int b, const float *LU, int64_t lda, const float *XU,
                               const float *XL, int64_t xstride, double *x, double *t, cudaStream_t st,
                               cudaStream_t side, cudaEvent_t *ev);

mxp_status launch_infnorm(int n, const double *x, double *out, cudaStream_t st);
mxp_status launch_ir_init(int n, const double *rhs, const double *d, double *x, cudaStream_t st);
mxp_status launch_copy(int n, const double *src, double *dst, cudaStream_t st);
mxp_status launch_axpy(int n, double alpha, const double *x, double *y, cudaStream_t st);
mxp_status launch_norma(int n, const double *d, const double *rowsum, double *out,
                        cudaStream_t st);

int num_sms();

}  // namespace mxp
