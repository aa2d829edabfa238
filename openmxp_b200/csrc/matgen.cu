// LCG matrix / RHS generation, bit-exact with the reference generator.
//
// Reference: panel_matgen_dev -> fill_panel_dev / fill_panel_diag_dev
// (matgen.hpp:8-117) and panel_colvgen (matgen.hpp:419-436).
//
// Two kernels:
//  * fill: every element (i, j) of the FP32 matrix (and the FP64 RHS,
//    stream column n).  Lanes own consecutive rows so each column is written
//    with 128-byte coalesced stores; a thread walks across columns with the
//    jump J_n = INC1^n, so the per-thread jump-ahead is paid once per
//    column band, not per element.
//  * diag: d_i = sum_{j != i} |a_ij| in FP64 in exactly the reduction order
//    of fill_panel_diag_dev (512 strided partials per row, tree 512 -> 4,
//    then ((s0+s1)+s2)+s3), so d is bit-identical to the reference's GPU
//    path; then A(i,i) = float(d_i).
#include "mxp_internal.cuh"

namespace mxp {

namespace {

constexpr int kFillThreads = 256;
constexpr int kFillRowsPerThread = 16;                              // rows per thread
constexpr int kFillRowBand = kFillThreads * kFillRowsPerThread;     // 4096 rows
constexpr int kFillColBand = 64;                                    // columns per CTA

// Fill A(r, c) for r in [0, nrows), c in [c0, c0 + ncols) of the generator
// matrix of order n, where output column c lands at out + (c - c0) * ld.
// T = float for the matrix, double for the RHS column.
template <typename T>
__global__ void __launch_bounds__(kFillThreads)
fill_kernel(int n, int64_t nrows, int64_t c0, int64_t ncols, uint64_t s00, Aff jn, T *out,
            int64_t ld) {
    const int t = threadIdx.x;
    const int64_t r_base = (int64_t)blockIdx.x * kFillRowBand;
    const int64_t cb0 = c0 + (int64_t)blockIdx.y * kFillColBand;
    const int64_t cb1 = min(cb0 + kFillColBand, c0 + ncols);
    if (cb0 >= cb1) return;

    // State of element (r_base + t, cb0): INC1^(r_base + t + n*cb0) applied to s00.
    const Aff inc1 = lcg_inc1();
    const uint64_t idx0 = (uint64_t)(r_base + t) + (uint64_t)n * (uint64_t)cb0;
    uint64_t s_row[kFillRowsPerThread];
    {
        uint64_t s = aff_apply(aff_pow(inc1, idx0), s00);
        const Aff step = aff_pow(inc1, kFillThreads);  // next row handled by this thread
#pragma unroll
        for (int q = 0; q < kFillRowsPerThread; ++q) {
            s_row[q] = s;
            s = aff_apply(step, s);
        }
    }
    for (int64_t c = cb0; c < cb1; ++c) {
        T *col = out + (c - c0) * ld;
#pragma unroll
        for (int q = 0; q < kFillRowsPerThread; ++q) {
            const int64_t r = r_base + t + (int64_t)q * kFillThreads;
            if (r < nrows) {
                const double v = lcg_to_double(s_row[q]);
                col[r] = static_cast<T>(v);   // float: round to nearest (RandStat::operator float)
            }
            s_row[q] = aff_apply(jn, s_row[q]);
        }
    }
}

constexpr int kDiagThreads = 512;  // MATGEM_THREADS of matgen.hpp:7, pinned by the reduction order

__global__ void __launch_bounds__(kDiagThreads)
diag_kernel(int n, uint64_t s00, Aff jn, Aff j512, int diag_rule, float *A, double *A64,
            int64_t lda, double *d, double *rowsum) {
    __shared__ double sh[kDiagThreads];
    const int64_t row = blockIdx.x;
    const int t = threadIdx.x;
    double acc = 0.0;
    if (t < n) {
        // element (row, t): INC1^(row + n*t) = J_n^t o INC1^row
        const Aff start = aff_mul(aff_pow(jn, (uint64_t)t), aff_pow(lcg_inc1(), (uint64_t)row));
        uint64_t s = aff_apply(start, s00);
        for (int64_t j = t; j < n; j += kDiagThreads) {
            if (j != row) acc += fabs(lcg_to_double(s));
            s = aff_apply(j512, s);
        }
    }
    sh[t] = acc;
    __syncthreads();
#pragma unroll
    for (int w = 256; w >= 4; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    if (t == 0) {
        const double s = ((sh[0] + sh[1]) + sh[2]) + sh[3];
        const double dv = diag_rule == MXP_DIAG_055_PLUS1 ? __dadd_rn(__dmul_rn(0.55, s), 1.0) : s;
        if (rowsum) rowsum[row] = s;
        if (d) d[row] = dv;
        if (A) A[row * lda + row] = __double2float_rn(dv);
        if (A64) A64[row * lda + row] = dv;
    }
}

}  // namespace

mxp_status launch_matgen(int n, uint64_t seed, int diag_rule, float *A, int64_t lda, double *d,
                         double *rowsum, double *rhs, cudaStream_t st) {
    if (n <= 0) return fail(MXP_INVALID_ARG, "mxp_matgen: n must be positive");
    if (A && lda < n) return fail(MXP_INVALID_ARG, "mxp_matgen: lda < n");
    if (diag_rule != MXP_DIAG_ROWSUM && diag_rule != MXP_DIAG_055_PLUS1)
        return fail(MXP_INVALID_ARG, "mxp_matgen: unknown diag_rule");
    const uint64_t s00 = lcg_stat00(seed);
    const Aff jn = aff_pow(lcg_inc1(), (uint64_t)n);
    const int64_t row_bands = cdiv(n, kFillRowBand);
    if (A) {
        const int64_t col_bands = cdiv(n, kFillColBand);
        for (int64_t cb = 0; cb < col_bands; cb += 65535) {
            const int64_t nb = col_bands - cb < 65535 ? col_bands - cb : 65535;
            dim3 grid((unsigned)row_bands, (unsigned)nb);
            const int64_t c0 = cb * kFillColBand;
            fill_kernel<float><<<grid, kFillThreads, 0, st>>>(n, n, c0, n - c0, s00, jn,
                                                               A + c0 * lda, lda);
            MXP_LAUNCHED();
        }
    }
    if (rhs) {
        dim3 grid((unsigned)row_bands, 1);
        fill_kernel<double><<<grid, kFillThreads, 0, st>>>(n, n, n, 1, s00, jn, rhs, n);
        MXP_LAUNCHED();
    }
    if (A || d || rowsum) {
        const Aff j512 = aff_pow(jn, kDiagThreads);
        diag_kernel<<<n, kDiagThreads, 0, st>>>(n, s00, jn, j512, diag_rule, A, nullptr, lda, d,
                                                 rowsum);
        MXP_LAUNCHED();
    }
    return MXP_OK;
}

mxp_status launch_matgen_f64(int n, uint64_t seed, int diag_rule, double *A, int64_t lda,
                             cudaStream_t st) {
    if (n <= 0 || !A) return fail(MXP_INVALID_ARG, "mxp_matgen_f64: bad arguments");
    if (lda < n) return fail(MXP_INVALID_ARG, "mxp_matgen_f64: lda < n");
    if (diag_rule != MXP_DIAG_ROWSUM && diag_rule != MXP_DIAG_055_PLUS1)
        return fail(MXP_INVALID_ARG, "mxp_matgen_f64: unknown diag_rule");
    const uint64_t s00 = lcg_stat00(seed);
    const Aff jn = aff_pow(lcg_inc1(), (uint64_t)n);
    const int64_t row_bands = cdiv(n, kFillRowBand);
    const int64_t col_bands = cdiv(n, kFillColBand);
    for (int64_t cb = 0; cb < col_bands; cb += 65535) {
        const int64_t nb = col_bands - cb < 65535 ? col_bands - cb : 65535;
        dim3 grid((unsigned)row_bands, (unsigned)nb);
        const int64_t c0 = cb * kFillColBand;
        fill_kernel<double><<<grid, kFillThreads, 0, st>>>(n, n, c0, n - c0, s00, jn, A + c0 * lda,
                                                            lda);
        MXP_LAUNCHED();
    }
    const Aff j512 = aff_pow(jn, kDiagThreads);
    diag_kernel<<<n, kDiagThreads, 0, st>>>(n, s00, jn, j512, diag_rule, nullptr, A, lda, nullptr,
                                             nullptr);
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
