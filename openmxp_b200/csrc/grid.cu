// Device pieces of the 2D block-cyclic driver (openmxp_b200/grid.py): the
// local blocks of the generator matrix, the residual GEMV over them with A
// regenerated in FP64, and an FP32-matrix x FP64-vector block GEMV for the
// distributed triangular solves.  The LU itself reuses the granular entry
// points (GETRF, panel TRSMs, panel casts, tcgen05 Schur update).
//
// Layout (Panels, panel.hpp:189-215; Grid, grid.hpp:25-80): global b x b
// block (I, J) lives on process (I mod P, J mod Q); a process keeps its
// blocks in one column-major local matrix, block (I, J) at local block
// (I div P, J div Q), lda = the local row count.
#include "mxp_internal.cuh"

namespace mxp {

namespace {

struct Cyclic {
    int64_t n;
    int b, nprow, npcol, myrow, mycol;
};

__device__ __forceinline__ int64_t glob_row(const Cyclic &g, int64_t li) {
    return ((li / g.b) * g.nprow + g.myrow) * (int64_t)g.b + li % g.b;
}
__device__ __forceinline__ int64_t glob_col(const Cyclic &g, int64_t lj) {
    return ((lj / g.b) * g.npcol + g.mycol) * (int64_t)g.b + lj % g.b;
}

constexpr int kRows = 256;

// Local matrix of the block-cyclic distribution: thread per local row, CTA =
// 256 local rows x one local column block.  Element (i, j) is stream index
// i + n j (hpl_rand.hpp:249-254): one jump to the block's first column, then
// J_n per column.  A(i, i) = float(d_i) as fill_panel_diag_dev (matgen.hpp:
// 26-65) leaves it.
__global__ void __launch_bounds__(kRows)
fill_local_kernel(Cyclic g, int64_t mloc, uint64_t s00, Aff jn, const double *d, float *A, int64_t lda) {
    const int64_t li = (int64_t)blockIdx.x * kRows + threadIdx.x;
    if (li >= mloc) return;
    const int64_t lj0 = (int64_t)blockIdx.y * g.b;
    const int64_t gi = glob_row(g, li), gj0 = glob_col(g, lj0);
    uint64_t s = aff_apply(aff_pow(lcg_inc1(), (uint64_t)gi + (uint64_t)g.n * (uint64_t)gj0), s00);
    for (int c = 0; c < g.b; ++c) {
        const double v = (gi == gj0 + c) ? d[gi] : lcg_to_double(s);
        A[(lj0 + c) * lda + li] = __double2float_rn(v);
        s = aff_apply(jn, s);
    }
}

// y(gi) += alpha * sum over this process's columns gj of a(gi, gj) x(gj) for
// its rows gi, with a(gi, gj) regenerated in FP64 and a(gi, gi) = d(gi):
// the per-process part of panel_gemv_h (panel_gemv.hpp:119-176) before the
// sum across the process row (:177).  x and y are whole-length vectors.
// Thread per local row, the x values of a column block staged in shared
// memory; every row is summed in a fixed order (deterministic).
__global__ void __launch_bounds__(kRows)
otf_gemv_local_kernel(Cyclic g, int64_t mloc, int64_t nloc, uint64_t s00, Aff jn, const double *d, double alpha,
                      const double *x, double *y) {
    extern __shared__ double xs[];
    const int64_t li = (int64_t)blockIdx.x * kRows + threadIdx.x;
    const bool act = li < mloc;
    const int64_t gi = act ? glob_row(g, li) : 0;
    double acc = 0.0;
    for (int64_t lj0 = 0; lj0 < nloc; lj0 += g.b) {
        const int64_t gj0 = glob_col(g, lj0);
        __syncthreads();
        for (int c = threadIdx.x; c < g.b; c += kRows) xs[c] = x[gj0 + c];
        __syncthreads();
        if (act) {
            uint64_t s = aff_apply(aff_pow(lcg_inc1(), (uint64_t)gi + (uint64_t)g.n * (uint64_t)gj0), s00);
            for (int c = 0; c < g.b; ++c) {
                const double v = (gi == gj0 + c) ? d[gi] : lcg_to_double(s);
                acc = fma(v, xs[c], acc);
                s = aff_apply(jn, s);
            }
        }
    }
    if (act) y[gi] = fma(alpha, acc, y[gi]);
}

// y = beta y + alpha A x, A FP32 (m x n, column-major), x and y FP64: the
// off-diagonal updates and the diagonal-block products of the distributed
// triangular solves (HPLMXP_gemv / gemv_kernel, panel_trsv.hpp:13-225).  CTA:
// 32 rows (a lane per row, 128-byte loads of each column) x 8 warps, warp w
// summing a contiguous eighth of the columns; the eight partials are added in
// warp order (deterministic).
__global__ void __launch_bounds__(256)
block_gemv_kernel(int m, int n, double alpha, const float *A, int64_t lda, const double *x, double beta,
                  double *y) {
    __shared__ double part[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t row = (int64_t)blockIdx.x * 32 + lane;
    const int chunk = (n + 7) / 8;
    const int j0 = w * chunk, j1 = min(n, j0 + chunk);
    double acc = 0.0;
    if (row < m) {
        int j = j0;
        for (; j + 4 <= j1; j += 4) {
            const float a0 = A[(int64_t)j * lda + row], a1 = A[(int64_t)(j + 1) * lda + row];
            const float a2 = A[(int64_t)(j + 2) * lda + row], a3 = A[(int64_t)(j + 3) * lda + row];
            acc = fma((double)a0, x[j], acc);
            acc = fma((double)a1, x[j + 1], acc);
            acc = fma((double)a2, x[j + 2], acc);
            acc = fma((double)a3, x[j + 3], acc);
        }
        for (; j < j1; ++j) acc = fma((double)A[(int64_t)j * lda + row], x[j], acc);
    }
    part[w][lane] = acc;
    __syncthreads();
    if (w == 0 && row < m) {
        double s = part[0][lane];
#pragma unroll
        for (int q = 1; q < 8; ++q) s += part[q][lane];
        y[row] = beta == 0.0 ? alpha * s : fma(alpha, s, beta * y[row]);
    }
}

mxp_status check_grid(int64_t n, int b, int nprow, int npcol, int myrow, int mycol, const char *who) {
    if (n <= 0 || b <= 0 || n % b != 0) return fail(MXP_INVALID_ARG, std::string(who) + ": n must be a positive multiple of b");
    if (nprow <= 0 || npcol <= 0 || myrow < 0 || myrow >= nprow || mycol < 0 || mycol >= npcol)
        return fail(MXP_INVALID_ARG, std::string(who) + ": bad process grid coordinates");
    return MXP_OK;
}

}  // namespace

int64_t local_extent(int64_t n, int b, int nproc, int me) {
    const int64_t nb = n / b;
    const int64_t blocks = nb > me ? (nb - me + nproc - 1) / nproc : 0;
    return blocks * b;
}

}  // namespace mxp

using namespace mxp;

extern "C" mxp_status mxp_local_extent(int n, int b, int nproc, int me, int64_t *h_extent) {
    if (!h_extent || n <= 0 || b <= 0 || n % b != 0 || nproc <= 0 || me < 0 || me >= nproc)
        return fail(MXP_INVALID_ARG, "local_extent: bad arguments");
    *h_extent = local_extent(n, b, nproc, me);
    return MXP_OK;
}

extern "C" mxp_status mxp_matgen_local(int n, int b, uint64_t seed, int nprow, int npcol, int myrow, int mycol,
                                       const double *d_d, float *d_A, int64_t lda, void *stream) {
    mxp_status s = check_grid(n, b, nprow, npcol, myrow, mycol, "matgen_local");
    if (s != MXP_OK) return s;
    if (!d_d || !d_A) return fail(MXP_INVALID_ARG, "matgen_local: NULL argument");
    const int64_t mloc = local_extent(n, b, nprow, myrow), nloc = local_extent(n, b, npcol, mycol);
    if (lda < mloc) return fail(MXP_INVALID_ARG, "matgen_local: lda below the local row count");
    if (mloc == 0 || nloc == 0) return MXP_OK;
    if (nloc / b > 65535) return fail(MXP_INVALID_ARG, "matgen_local: too many local column blocks");
    const Cyclic g{n, b, nprow, npcol, myrow, mycol};
    const Aff jn = aff_pow(lcg_inc1(), (uint64_t)n);
    dim3 grid((unsigned)cdiv(mloc, kRows), (unsigned)(nloc / b));
    fill_local_kernel<<<grid, kRows, 0, (cudaStream_t)stream>>>(g, mloc, lcg_stat00(seed), jn, d_d, d_A, lda);
    MXP_LAUNCHED();
    return MXP_OK;
}

extern "C" mxp_status mxp_otf_gemv_local(int n, int b, uint64_t seed, int nprow, int npcol, int myrow, int mycol,
                                         const double *d_d, double alpha, const double *d_x, double *d_y,
                                         void *stream) {
    mxp_status s = check_grid(n, b, nprow, npcol, myrow, mycol, "otf_gemv_local");
    if (s != MXP_OK) return s;
    if (!d_d || !d_x || !d_y) return fail(MXP_INVALID_ARG, "otf_gemv_local: NULL argument");
    if ((size_t)b * sizeof(double) > 48 * 1024) return fail(MXP_INVALID_ARG, "otf_gemv_local: b above 6144");
    const int64_t mloc = local_extent(n, b, nprow, myrow), nloc = local_extent(n, b, npcol, mycol);
    if (mloc == 0) return MXP_OK;
    const Cyclic g{n, b, nprow, npcol, myrow, mycol};
    const Aff jn = aff_pow(lcg_inc1(), (uint64_t)n);
    otf_gemv_local_kernel<<<(unsigned)cdiv(mloc, kRows), kRows, (size_t)b * sizeof(double), (cudaStream_t)stream>>>(
        g, mloc, nloc, lcg_stat00(seed), jn, d_d, alpha, d_x, d_y);
    MXP_LAUNCHED();
    return MXP_OK;
}

extern "C" mxp_status mxp_block_gemv(int m, int n, double alpha, const float *d_A, int64_t lda, const double *d_x,
                                     double beta, double *d_y, void *stream) {
    if (m < 0 || n < 0) return fail(MXP_INVALID_ARG, "block_gemv: negative size");
    if (m == 0) return MXP_OK;
    if (!d_y || (n > 0 && (!d_A || !d_x))) return fail(MXP_INVALID_ARG, "block_gemv: NULL argument");
    if (n > 0 && lda < m) return fail(MXP_INVALID_ARG, "block_gemv: lda < m");
    block_gemv_kernel<<<(unsigned)cdiv(m, 32), 256, 0, (cudaStream_t)stream>>>(m, n, alpha, d_A, lda, d_x, beta,
                                                                                 d_y);
    MXP_LAUNCHED();
    return MXP_OK;
}
