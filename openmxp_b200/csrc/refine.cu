// FP64 kernels of the iterative refinement.
//
//  * otf_gemv: y = beta*y + alpha*A*x with a_ij regenerated from the LCG in
//    FP64 (otf_gemv_h / otf_gemv_d / otf_gemv_diag_d, panel_gemv.hpp:13-117).
//    The reference launches one <<<b,256>>> kernel per b x b block pair and
//    synchronises after each; here one launch covers the matrix: each thread
//    owns two rows (two independent LCG chains) over a column range and
//    steps the state with J_n = INC1^n per column.  Each state enters as
//    its two exact 32-bit halves (no 64-bit converter, no rounding of the
//    integer), and the 2^-64 scale of RandStat::operator double is folded
//    into x.
//    Column splits write partial sums to the workspace and a second kernel
//    reduces them in a fixed order, so the result is deterministic.
//  * lu_solve: x <- U^{-1} L^{-1} x with the FP32 factors (trsvL_h /
//    trsvU_h, panel_trsv.hpp:308-597).  One persistent launch per triangle:
//    row blocks of 64 are claimed in order through an atomic ticket; a row
//    block streams its part of the factor against the already-solved blocks
//    (waiting, bounded, on per-block completion flags), then solves its 64 x
//    64 diagonal triangle in FP64 and publishes.  Claim order guarantees every
//    awaited block is owned by a CTA that is already running.
//  * lu_solve_inv: the same solve in nb steps of bandwidth-bound products
//    with the stored inverses of the b x b diagonal blocks (used after
//    mxp_panel_lu, which keeps them); no chain of 64-row links.
//  * infnorm / vector ops (panel_norm.hpp:11-58, panel.hpp:525-623).
#include <algorithm>

#include "mxp_internal.cuh"

namespace mxp {

namespace {

// ---------------------------------------------------------------------------
// on-the-fly GEMV
// ---------------------------------------------------------------------------
constexpr int kGemvThreads = 128;
constexpr int kGemvRowsPerThread = 2;
constexpr int kGemvRows = kGemvThreads * kGemvRowsPerThread;  // 256 rows per CTA
constexpr int kGemvXChunk = 1024;
constexpr double kLcgScale = 0x1.fffffffffffffP-65;

// Per element the state s = hi * 2^32 + lo (hi signed, lo unsigned) enters
// as two exact doubles, both made by placing the integer in the mantissa of
// a biased constant: hi * 2^32 = (2^84 + (hi ^ 2^31) * 2^32) - (2^84 + 2^63),
// and 2^52 + lo, whose bias 2^52 is not removed per element: the CTA sums
// 2^52 * xs over its columns once and subtracts it from every row at the
// end (the bias terms are 2^-12 |x| each against |a_ij x| ~ |x|/4, so the
// extra rounding stays far below the FP64 rounding of the sum itself).  The
// diagonal column is accumulated like the others and its LCG value taken
// out afterwards (no compare per element), then d_i x_i is added.
__global__ void __launch_bounds__(kGemvThreads)
otf_gemv_kernel(int n, uint64_t s00, Aff jn, const double *__restrict__ d,
                const double *__restrict__ x, int64_t cols_per_split, double alpha, double beta,
                double *__restrict__ y, double *__restrict__ partials) {
    __shared__ double xs[kGemvXChunk];
    __shared__ double bias_red[kGemvThreads];
    const int64_t r0 = (int64_t)blockIdx.x * kGemvRows + threadIdx.x;
    const int64_t r1 = r0 + kGemvThreads;
    const int64_t j_begin = (int64_t)blockIdx.y * cols_per_split;
    const int64_t j_end = imin64(n, j_begin + cols_per_split);
    constexpr double kHiBias = 0x1p84 + 0x1p63;
    constexpr double kLoBias = 0x1p52;

    const Aff inc1 = lcg_inc1();
    // states of (r0, j_begin) and (r1, j_begin)
    uint64_t s0 = aff_apply(aff_pow(inc1, (uint64_t)r0 + (uint64_t)n * (uint64_t)j_begin), s00);
    uint64_t s1 = aff_apply(aff_pow(inc1, (uint64_t)kGemvThreads), s0);
    double acc0 = 0.0, acc1 = 0.0, bias = 0.0;
    for (int64_t jc = j_begin; jc < j_end; jc += kGemvXChunk) {
        const int len = (int)imin64(kGemvXChunk, j_end - jc);
        __syncthreads();
        for (int q = threadIdx.x; q < len; q += kGemvThreads) {
            const double v = x[jc + q] * kLcgScale;
            xs[q] = v;
            bias = __fma_rn(kLoBias, v, bias);
        }
        __syncthreads();
#pragma unroll 4
        for (int q = 0; q < len; ++q) {
            const double xq = xs[q];
            const double h0 = __hiloint2double(0x45300000, (int)((uint32_t)(s0 >> 32) ^ 0x80000000u)) - kHiBias;
            const double h1 = __hiloint2double(0x45300000, (int)((uint32_t)(s1 >> 32) ^ 0x80000000u)) - kHiBias;
            acc0 = __fma_rn(h0, xq, acc0);
            acc1 = __fma_rn(h1, xq, acc1);
            acc0 = __fma_rn(__hiloint2double(0x43300000, (int)(uint32_t)s0), xq, acc0);
            acc1 = __fma_rn(__hiloint2double(0x43300000, (int)(uint32_t)s1), xq, acc1);
            s0 = aff_apply(jn, s0);
            s1 = aff_apply(jn, s1);
        }
    }
    // the CTA's bias sum, in a fixed order
    bias_red[threadIdx.x] = bias;
    __syncthreads();
    for (int w = kGemvThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) bias_red[threadIdx.x] += bias_red[threadIdx.x + w];
        __syncthreads();
    }
    bias = bias_red[0];
    acc0 -= bias;
    acc1 -= bias;
    // diagonal entries come from d (otf_gemv_diag_d, panel_gemv.hpp:26): the
    // LCG value accumulated at (r, r) is taken out, d_r x_r added
    if (r0 < n && r0 >= j_begin && r0 < j_end) {
        const uint64_t sd = aff_apply(aff_pow(inc1, (uint64_t)r0 + (uint64_t)n * (uint64_t)r0), s00);
        acc0 = __fma_rn(-i64_to_double_rn(sd), x[r0] * kLcgScale, acc0) + d[r0] * x[r0];
    }
    if (r1 < n && r1 >= j_begin && r1 < j_end) {
        const uint64_t sd = aff_apply(aff_pow(inc1, (uint64_t)r1 + (uint64_t)n * (uint64_t)r1), s00);
        acc1 = __fma_rn(-i64_to_double_rn(sd), x[r1] * kLcgScale, acc1) + d[r1] * x[r1];
    }
    if (partials) {
        double *p = partials + (int64_t)blockIdx.y * n;
        if (r0 < n) p[r0] = acc0;
        if (r1 < n) p[r1] = acc1;
    } else {
        if (r0 < n) y[r0] = (beta == 0.0 ? 0.0 : beta * y[r0]) + alpha * acc0;
        if (r1 < n) y[r1] = (beta == 0.0 ? 0.0 : beta * y[r1]) + alpha * acc1;
    }
}

__global__ void gemv_reduce_kernel(int n, int splits, const double *__restrict__ partials,
                                   double alpha, double beta, double *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = 0.0;
    for (int s = 0; s < splits; ++s) t += partials[(int64_t)s * n + i];
    y[i] = (beta == 0.0 ? 0.0 : beta * y[i]) + alpha * t;
}

// ---------------------------------------------------------------------------
// sync-free block triangular solves
// ---------------------------------------------------------------------------
constexpr int kRB = 64;
constexpr int kTrsvThreads = 256;

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block forward (LOWER: unit L) or backward (upper: U) substitution, one
// 64-row block per CTA, CTAs taking row blocks in solve order from a ticket.
// flags[0..nrb): block done; flags[nrb]: ticket.
//
// The blocks form a chain (block b needs x of every earlier block), so the
// time per link is what bounds the solve.  Everything that does not depend
// on the predecessor is done before waiting for it:
//   * Minv = inverse of the diagonal block (FP64, from the FP32 factor) and
//     P = Minv * A_adj, A_adj the off-diagonal block next in the chain;
//   * the products of all other off-diagonal blocks with their (already
//     solved) x, streamed with four column blocks of loads in flight;
//   * w = Minv (r_b - those products).
// When the predecessor publishes its x, the block finishes with one 64 x 64
// FP64 matrix-vector product, x_b = w - P x_adj, and publishes its own x.
// This is the block substitution of the reference's trsvL_h / trsvU_h
// (panel_trsv.hpp:308-597: FP64 solve of each upcast diagonal block, FP32 x
// FP64 products for the rest) with the diagonal solve applied as a product
// with its inverse.
constexpr int kXChunk = 8;  // column blocks whose x is staged in shared memory at a time
constexpr size_t kTrsvSmem = 2 * sizeof(double) * kRB * (kRB + 1) + sizeof(float) * kRB * (kRB + 1) +
                             sizeof(double) * kRB + sizeof(double) * 4 * kRB +
                             sizeof(double) * 2 * kXChunk * kRB + 16;

template <bool LOWER>
__global__ void __launch_bounds__(kTrsvThreads)
trsv_kernel(int n, const float *__restrict__ LU, int64_t lda, double *x, int *flags,
            DevStatus *dst, int withhold) {
    extern __shared__ __align__(16) unsigned char trsv_smem[];
    double(*minv)[kRB + 1] = reinterpret_cast<double(*)[kRB + 1]>(trsv_smem);
    double(*pm)[kRB + 1] = minv + kRB;
    float(*blk)[kRB + 1] = reinterpret_cast<float(*)[kRB + 1]>(pm + kRB);   // blk[col][row]
    double *zs = reinterpret_cast<double *>(blk + kRB);
    double(*part)[kRB] = reinterpret_cast<double(*)[kRB]>(zs + kRB);
    double(*xs)[kXChunk * kRB] = reinterpret_cast<double(*)[kXChunk * kRB]>(part + 4);  // 2 buffers
    int *s_ticket = reinterpret_cast<int *>(xs + 2);

    const int nrb = (n + kRB - 1) / kRB;
    const int tid = threadIdx.x;
    if (tid == 0) *s_ticket = atomicAdd(&flags[nrb], 1);
    __syncthreads();
    const int rb = LOWER ? *s_ticket : nrb - 1 - *s_ticket;
    const int64_t row0 = (int64_t)rb * kRB;
    const int nrows = (int)imin64(kRB, n - row0);
    const int ncb = LOWER ? rb : nrb - 1 - rb;  // off-diagonal column blocks
    const bool has_adj = ncb > 0;
    const int adj = LOWER ? rb - 1 : rb + 1;    // chain predecessor

    // ---- Minv: inverse of the diagonal block (padded with the identity) ----
    for (int idx = tid; idx < kRB * kRB; idx += kTrsvThreads) {
        const int rr = idx % kRB, cc = idx / kRB;
        float v = (rr < nrows && cc < nrows) ? LU[(row0 + cc) * lda + row0 + rr] : 0.0f;
        if (rr == cc && (rr >= nrows || LOWER)) v = 1.0f;
        blk[cc][rr] = v;
    }
    __syncthreads();
    if (tid < kRB) {  // column j of the inverse: T y = e_j
        const int j = tid;
        if (LOWER) {
            for (int i = 0; i < kRB; ++i) {
                double v = (i == j) ? 1.0 : 0.0;
                if (i > j)
                    for (int k = j; k < i; ++k) v = __fma_rn(-(double)blk[k][i], minv[k][j], v);
                minv[i][j] = (i >= j) ? v : 0.0;
            }
        } else {
            for (int i = kRB - 1; i >= 0; --i) {
                double v = (i == j) ? 1.0 : 0.0;
                if (i < j)
                    for (int k = i + 1; k <= j; ++k) v = __fma_rn(-(double)blk[k][i], minv[k][j], v);
                minv[i][j] = (i <= j) ? v / (double)blk[i][i] : 0.0;
            }
        }
    }
    __syncthreads();
    // ---- P = Minv * A_adj ----
    const int pi = tid >> 2, ph = tid & 3;  // row of a 64-vector, quarter of its columns
    if (has_adj) {
        const int64_t c0 = (int64_t)adj * kRB;
        const int ncols = (int)imin64(kRB, n - c0);
        for (int idx = tid; idx < kRB * kRB; idx += kTrsvThreads) {
            const int rr = idx % kRB, cc = idx / kRB;
            blk[cc][rr] = (rr < nrows && cc < ncols) ? LU[(c0 + cc) * lda + row0 + rr] : 0.0f;
        }
        __syncthreads();
#pragma unroll 1
        for (int c = ph * 16; c < ph * 16 + 16; ++c) {
            double v = 0.0;
#pragma unroll 8
            for (int k = 0; k < kRB; ++k) v = __fma_rn(minv[pi][k], (double)blk[c][k], v);
            pm[pi][c] = v;
        }
    }

    // ---- products with every other off-diagonal block ----
    double acc = 0.0;
    int known = LOWER ? -1 : nrb;  // furthest block known complete
    bool timed_out = false;
    const int r = tid % kRB, cph = tid / kRB;  // 4 column phases of 16
    const int64_t grow = row0 + r;
    const bool row_ok = r < nrows;
    const int nstream = has_adj ? ncb - 1 : 0;
    auto load_l = [&](int q, float *d) {
        if (q >= nstream) return;
        const int cb = LOWER ? q : nrb - 1 - q;
        const int64_t c0 = (int64_t)cb * kRB + cph * 16;
        const int clen = (int)imin64(16, n - c0);
        const float *col = LU + c0 * lda + grow;
#pragma unroll
        for (int cc = 0; cc < 16; ++cc) d[cc] = (row_ok && cc < clen) ? col[cc * lda] : 0.0f;
    };
    // Flags are polled by lane 0 of each warp only (every thread spinning on the
    // same lines slows the producer's release) and the outcome is shared by a
    // shuffle; the warp barrier orders the lanes' later loads after the acquire.
    const bool lead = (tid & 31) == 0;
    auto wait_flag = [&](int b) -> bool {
        int ok = 1;
        if (lead) {
            const unsigned long long t0 = globaltimer_ns();
            uint32_t it = 0;
            while (!ld_acquire(&flags[b])) {
                if ((++it & 63u) == 0u && globaltimer_ns() - t0 > kWaitTimeoutNs) {
                    ok = 0;
                    break;
                }
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        return ok != 0;
    };
    auto probe_flag = [&](int b) -> bool {
        int v = lead ? ld_acquire(&flags[b]) : 0;
        v = __shfl_sync(0xffffffffu, v, 0);
        __syncwarp();
        return v != 0;
    };
    // The x of the streamed column blocks is staged in shared memory kXChunk
    // blocks at a time (one coalesced load per thread and one barrier per
    // chunk, double-buffered) instead of one L2 round trip per column block:
    // the stream, not the chain, bounds the late blocks of a large solve.
    auto consume = [&](int buf, int qq, const float *lv) {
        const double *xv = xs[buf] + qq * kRB + cph * 16;
#pragma unroll
        for (int cc = 0; cc < 16; ++cc) acc = __fma_rn((double)lv[cc], xv[cc], acc);
    };
    // factor values do not depend on other blocks: keep four column blocks of
    // loads in flight (a register ring, unrolled so its indices stay static)
    float b0[16], b1[16], b2[16], b3[16];
    load_l(0, b0);
    load_l(1, b1);
    load_l(2, b2);
    load_l(3, b3);
    int buf = 0;
    for (int q0 = 0; q0 < nstream; q0 += kXChunk, buf ^= 1) {
        const int qn = min(kXChunk, nstream - q0);
        const int cb_last = LOWER ? q0 + qn - 1 : nrb - 1 - (q0 + qn - 1);
        // blocks complete in chain order: once the chunk's last block (or the
        // block before the predecessor) is published, so is the whole chunk
        if (!timed_out && (LOWER ? (cb_last > known) : (cb_last < known))) {
            if (probe_flag(adj - (LOWER ? 1 : -1))) {
                known = adj - (LOWER ? 1 : -1);
            } else {
                timed_out = !wait_flag(cb_last);
                known = cb_last;
            }
        }
        for (int e = tid; e < qn * kRB; e += kTrsvThreads) {
            const int qq = e / kRB, cc = e % kRB;
            const int cb = LOWER ? q0 + qq : nrb - 1 - (q0 + qq);
            const int64_t col = (int64_t)cb * kRB + cc;
            xs[buf][e] = (col < n) ? __ldcg(x + col) : 0.0;
        }
        // a wait that gave up anywhere in the CTA ends the stream everywhere
        timed_out = __syncthreads_or(timed_out) != 0;
        if (timed_out) break;
#pragma unroll
        for (int qq = 0; qq < kXChunk; qq += 4) {
            if (qq + 0 < qn) { consume(buf, qq + 0, b0); load_l(q0 + qq + 4, b0); }
            if (qq + 1 < qn) { consume(buf, qq + 1, b1); load_l(q0 + qq + 5, b1); }
            if (qq + 2 < qn) { consume(buf, qq + 2, b2); load_l(q0 + qq + 6, b2); }
            if (qq + 3 < qn) { consume(buf, qq + 3, b3); load_l(q0 + qq + 7, b3); }
        }
    }
    part[cph][r] = acc;
    __syncthreads();
    if (tid < kRB) {
        const double s = part[0][tid] + part[1][tid] + part[2][tid] + part[3][tid];
        zs[tid] = (tid < nrows) ? __ldcg(x + row0 + tid) - s : 0.0;
    }
    __syncthreads();
    // ---- w = Minv z (row pi, four lanes per row) ----
    double w = 0.0;
#pragma unroll
    for (int c = 0; c < 16; ++c) w = __fma_rn(minv[pi][ph * 16 + c], zs[ph * 16 + c], w);
    w += __shfl_xor_sync(0xffffffffu, w, 1);
    w += __shfl_xor_sync(0xffffffffu, w, 2);
    // ---- the chain link: x_b = w - P x_adj ----
    if (has_adj && !timed_out) {
        timed_out = !wait_flag(adj);
        const int64_t c0 = (int64_t)adj * kRB + ph * 16;
        const int clen = (int)imin64(16, n - c0);
        double xa[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) xa[c] = (c < clen) ? __ldcg(x + c0 + c) : 0.0;
        double p = 0.0;
#pragma unroll
        for (int c = 0; c < 16; ++c) p = __fma_rn(pm[pi][ph * 16 + c], xa[c], p);
        p += __shfl_xor_sync(0xffffffffu, p, 1);
        p += __shfl_xor_sync(0xffffffffu, p, 2);
        w -= p;
    }
    if (timed_out) report(dst, MXP_TIMEOUT, 10 + (LOWER ? 0 : 1), rb);
    if (ph == 0 && pi < nrows) __stcg(x + row0 + pi, w);
    __threadfence();
    __syncthreads();
    // published even after a timeout, so successors never stall; `withhold` (a
    // test of the bounded waits) leaves one block's flag unset
    if (tid == 0 && rb != withhold) st_release(&flags[rb], 1);
}

// ---------------------------------------------------------------------------
// block triangular solves with the stored inverses of the diagonal blocks
// ---------------------------------------------------------------------------
// The LU keeps inv(L_kk) and inv(U_kk) of every b x b diagonal block (the
// TRSM-by-inverse computes them anyway).  A triangle is then solved in nb
// steps of bandwidth-bound products instead of a chain of 64-row links:
//   lower, k = 0 .. nb-1:  x_k <- L_kk^{-1} x_k;  x_i -= L(i, k) x_k (rows below)
//   upper, k = nb-1 .. 0:  x_k <- U_kk^{-1} x_k;  x_i -= U(i, k) x_k (rows above)
// Block substitution as trsvL_h / trsvU_h (panel_trsv.hpp:308-597).  The
// diagonal-block solve is a product with the stored inverse X followed by
// one step of refinement against the factor block T, all in FP64:
//   t1 = X v,  s = v - T t1,  t = t1 + X s,
// so the result carries the square of the inverse's relative error (the
// inverse's tensor-core levels are near FP32, not FP32).  The unit diagonal
// of inv(L) and the diagonal 1/u_ii of inv(U) are applied exactly.  Every
// row is summed by one CTA in a fixed order: results are deterministic.
// The diagonal-block products are load-latency bound (a 13 MB triangle at
// b = 2560): small row tiles give many CTAs, each staging only the part of v
// its rows use; the trailing products stream the factor at HBM bandwidth.
constexpr int kIvThreads = 256;

// One CTA: ROWS rows (ROWS/4 quads of four rows, one float4 per column) x
// 256 / (ROWS/4) column groups (ROWS >= 8: a warp reads whole 32-byte
// sectors).  M: column-major FP32, ldm % 4 == 0, 16-byte
// aligned.  v: cols doubles, staged in shared memory.  With sum_i over the
// mode's entries of row i:
//   MODE 0: out[i] = base[i] - sum_j M(i,j) v_j                 (all columns)
//   MODE 1: out[i] = [base[i] +] v_i + sum_{j<i} M(i,j) v_j      (unit lower inverse)
//   MODE 2: out[i] = [base[i] +] v_i / T(i,i) + sum_{j>i} M(i,j) v_j  (upper inverse)
//   MODE 3: out[i] = base[i] - v_i - sum_{j<i} M(i,j) v_j        (v - T v, T unit lower)
//   MODE 4: out[i] = base[i] - sum_{j>=i} M(i,j) v_j             (v - T v, T upper)
// T(i,i) is read from tdiag (ld ldt).  CTA 0 also writes copy_dst[0..cols) = v.
template <int MODE, int ROWS>
__global__ void __launch_bounds__(kIvThreads)
trsv_inv_kernel(int rows, int cols, const float *__restrict__ M, int64_t ldm, const double *v,
                const float *__restrict__ tdiag, int64_t ldt, const double *base, double *out,
                double *copy_dst) {
    constexpr int QUADS = ROWS / 4;
    constexpr int GROUPS = kIvThreads / QUADS;
    extern __shared__ __align__(16) unsigned char iv_smem[];
    double *vs = reinterpret_cast<double *>(iv_smem);
    double(*red)[ROWS + 1] = reinterpret_cast<double(*)[ROWS + 1]>(vs + cols);
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * ROWS;
    constexpr bool kLow = MODE == 1 || MODE == 3;   // strictly lower entries
    constexpr bool kUpS = MODE == 2;                // strictly upper
    constexpr bool kUpD = MODE == 4;                // upper with the diagonal
    // the part of v this CTA reads: its rows and the columns they need
    int s0 = 0, s1 = cols;
    if (MODE != 0 && r0 < rows) {
        if (kLow) s1 = min(cols, r0 + ROWS);
        else s0 = r0;
    }
    for (int j = s0 + tid; j < s1; j += kIvThreads) vs[j] = v[j];
    __syncthreads();
    if (copy_dst && blockIdx.x == 0)
        for (int j = tid; j < cols; j += kIvThreads) copy_dst[j] = vs[j];
    if (r0 >= rows) return;  // a CTA launched only for the copy
    const int q = tid % QUADS, g = tid / QUADS;
    const int ri = r0 + 4 * q;  // first of this thread's four rows
    // column range the CTA's rows need
    int jb = 0, je = cols;
    if (kLow) je = min(cols, r0 + ROWS - 1);
    if (kUpS) jb = r0 + 1;
    if (kUpD) jb = r0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const float *mp = M + ri;
    auto fma4 = [&](float4 m, int j) {
        const double vj = vs[j];
        if (MODE == 0) {
            a0 = __fma_rn((double)m.x, vj, a0);
            a1 = __fma_rn((double)m.y, vj, a1);
            a2 = __fma_rn((double)m.z, vj, a2);
            a3 = __fma_rn((double)m.w, vj, a3);
        } else {
            const bool k0 = kLow ? j < ri : (kUpS ? j > ri : j >= ri);
            const bool k1 = kLow ? j < ri + 1 : (kUpS ? j > ri + 1 : j >= ri + 1);
            const bool k2 = kLow ? j < ri + 2 : (kUpS ? j > ri + 2 : j >= ri + 2);
            const bool k3 = kLow ? j < ri + 3 : (kUpS ? j > ri + 3 : j >= ri + 3);
            a0 = __fma_rn(k0 ? (double)m.x : 0.0, vj, a0);
            a1 = __fma_rn(k1 ? (double)m.y : 0.0, vj, a1);
            a2 = __fma_rn(k2 ? (double)m.z : 0.0, vj, a2);
            a3 = __fma_rn(k3 ? (double)m.w : 0.0, vj, a3);
        }
    };
    int j = jb + g;
    // eight 16-byte loads in flight per thread
    for (; j + 7 * GROUPS < je; j += 8 * GROUPS) {
        float4 m[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            m[u] = __ldcs(reinterpret_cast<const float4 *>(mp + (int64_t)(j + GROUPS * u) * ldm));
#pragma unroll
        for (int u = 0; u < 8; ++u) fma4(m[u], j + GROUPS * u);
    }
    for (; j < je; j += GROUPS) fma4(__ldcs(reinterpret_cast<const float4 *>(mp + (int64_t)j * ldm)), j);
    red[g][4 * q + 0] = a0;
    red[g][4 * q + 1] = a1;
    red[g][4 * q + 2] = a2;
    red[g][4 * q + 3] = a3;
    __syncthreads();
    if (tid < ROWS) {
        double s = 0.0;
#pragma unroll 8
        for (int c = 0; c < GROUPS; ++c) s += red[c][tid];
        const int i = r0 + tid;
        double y;
        if (MODE == 0) y = base[i] - s;
        else if (MODE == 1) y = vs[i] + s;
        else if (MODE == 2) y = vs[i] / (double)tdiag[(int64_t)i * (ldt + 1)] + s;
        else if (MODE == 3) y = base[i] - vs[i] - s;
        else y = base[i] - s;
        if ((MODE == 1 || MODE == 2) && base) y += base[i];
        out[i] = y;
    }
}

constexpr int kIvRowsUpd = 32;   // rows per CTA of the trailing products
constexpr int kIvRowsDiag = 8;   // rows per CTA of the diagonal-block products (b / 8 CTAs)

size_t trsv_inv_smem(int b) { return (size_t)b * sizeof(double) + sizeof(double) * 64 * (kIvRowsUpd + 1); }

// ---------------------------------------------------------------------------
// norms and vector ops
// ---------------------------------------------------------------------------
__global__ void infnorm_kernel(int n, const double *__restrict__ x, unsigned long long *out) {
    double m = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        // non-negative doubles order like their bit patterns; NaN sorts high
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void norma_kernel(int n, const double *__restrict__ d, const double *__restrict__ rs,
                             unsigned long long *out) {
    double m = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, rs ? rs[i] + d[i] : 2.0 * d[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void ir_init_kernel(int n, const double *__restrict__ rhs, const double *__restrict__ d,
                               double *__restrict__ x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = rhs[i] / d[i];
}

__global__ void copy_kernel(int n, const double *__restrict__ s, double *__restrict__ t) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) t[i] = s[i];
}

__global__ void axpy_kernel(int n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += alpha * x[i];
}

}  // namespace

mxp_status launch_otf_gemv(int n, uint64_t seed, const double *d, double alpha, const double *x,
                           double beta, double *y, double *partials, int max_splits,
                           cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    const int row_blocks = (int)cdiv(n, kGemvRows);
    const int target = 4 * num_sms();
    int splits = (target + row_blocks - 1) / row_blocks;
    if (splits > max_splits) splits = max_splits;
    if (!partials) splits = 1;
    int64_t cols = cdiv(n, splits);
    cols = cdiv(cols, 64) * 64;
    splits = (int)cdiv(n, cols);
    if (splits < 1) splits = 1;
    const uint64_t s00 = lcg_stat00(seed);
    const Aff jn = aff_pow(lcg_inc1(), (uint64_t)n);
    dim3 grid((unsigned)row_blocks, (unsigned)splits);
    otf_gemv_kernel<<<grid, kGemvThreads, 0, st>>>(n, s00, jn, d, x, cols, alpha, beta, y,
                                                   splits > 1 ? partials : nullptr);
    MXP_LAUNCHED();
    if (splits > 1) {
        gemv_reduce_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, splits, partials, alpha, beta, y);
        MXP_LAUNCHED();
    }
    return MXP_OK;
}

size_t lu_solve_flag_ints(int n) { return 2 * ((size_t)cdiv(n, kRB) + 1); }

mxp_status launch_lu_solve(int n, const float *LU, int64_t lda, double *x, int *flags,
                           DevStatus *dst, cudaStream_t st, int withhold) {
    if (n <= 0) return MXP_OK;
    if (lda < n) return fail(MXP_INVALID_ARG, "lu_solve: lda < n");
    const int nrb = (int)cdiv(n, kRB);
    MXP_CUDA(cudaMemsetAsync(flags, 0, lu_solve_flag_ints(n) * sizeof(int), st));
    MXP_CUDA(cudaFuncSetAttribute(trsv_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsvSmem));
    MXP_CUDA(cudaFuncSetAttribute(trsv_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsvSmem));
    trsv_kernel<true><<<nrb, kTrsvThreads, kTrsvSmem, st>>>(n, LU, lda, x, flags, dst, withhold);
    MXP_LAUNCHED();
    trsv_kernel<false><<<nrb, kTrsvThreads, kTrsvSmem, st>>>(n, LU, lda, x, flags + nrb + 1, dst, -1);
    MXP_LAUNCHED();
    return MXP_OK;
}

bool lu_solve_inv_supported(int n, int b, const float *LU, int64_t lda) {
    return n > 0 && b > 0 && n % b == 0 && b % kIvRowsUpd == 0 && lda % 4 == 0 &&
           (reinterpret_cast<uintptr_t>(LU) & 15u) == 0 && trsv_inv_smem(b) <= 200 * 1024;
}

mxp_status launch_lu_solve_inv(int n, int b, const float *LU, int64_t lda, const float *XU,
                               const float *XL, int64_t xstride, double *x, double *t, cudaStream_t st,
                               cudaStream_t side, cudaEvent_t *ev) {
    if (n <= 0) return MXP_OK;
    if (!lu_solve_inv_supported(n, b, LU, lda) || xstride % 4 != 0 ||
        ((reinterpret_cast<uintptr_t>(XU) | reinterpret_cast<uintptr_t>(XL)) & 15u))
        return fail(MXP_INVALID_ARG, "lu_solve_inv: shape or alignment not supported");
    const int nb = n / b;
    const size_t smem = trsv_inv_smem(b);
    if (smem > 48 * 1024) {
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<0, kIvRowsUpd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<1, kIvRowsDiag>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<2, kIvRowsDiag>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<3, kIvRowsDiag>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<4, kIvRowsDiag>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MXP_CUDA(cudaFuncSetAttribute(trsv_inv_kernel<0, kIvRowsDiag>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    double *t1 = t, *sv = t + b, *t2 = t + 2 * (int64_t)b;  // 4 b doubles (t2 double-buffered)
    const unsigned dg = (unsigned)(b / kIvRowsDiag);
    auto upd_grid = [](int rows) { return (unsigned)std::max(1, rows / kIvRowsUpd); };
    if (!side || !ev) return fail(MXP_INVALID_ARG, "lu_solve_inv: needs a second stream and four events");
    {
        // Two streams.  The chain that bounds the solve -- the three
        // diagonal-block products of step s and the update of the next
        // block's rows -- runs on `side` (high priority); the update of all
        // rows beyond the next block, which only step s+2 needs, runs on `st`
        // and overlaps the chain of step s+1.  Every row still receives its
        // updates in step order (the next-block update of step s waits for
        // the bulk update of step s-1, which covered that block), so the
        // result is the same, bit for bit, as with every launch on one stream.
        // ev[0]: fork / join, ev[1]: t2 of the step ready, ev[2 + s % 2]: bulk update of step s done.
        for (int tri = 0; tri < 2; ++tri) {
            const bool lower = tri == 0;
            MXP_CUDA(cudaEventRecord(ev[0], st));
            MXP_CUDA(cudaStreamWaitEvent(side, ev[0], 0));
            int bulk_step[2] = {-1, -1};
            for (int s = 0; s < nb; ++s) {
                const int k = lower ? s : nb - 1 - s;
                const int64_t kk = (int64_t)k * b;
                const float *X = (lower ? XL : XU) + k * xstride, *T = LU + kk + kk * lda;
                double *xk = x + kk;
                double *t2s = t2 + (int64_t)(s & 1) * b;
                if (s >= 2 && bulk_step[s & 1] == s - 2) MXP_CUDA(cudaStreamWaitEvent(side, ev[2 + (s & 1)], 0));
                if (lower) {
                    trsv_inv_kernel<1, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, X, b, xk, nullptr, 0, nullptr, t1, nullptr);
                    MXP_LAUNCHED();
                    trsv_inv_kernel<3, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, T, lda, t1, nullptr, 0, xk, sv, nullptr);
                    MXP_LAUNCHED();
                    trsv_inv_kernel<1, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, X, b, sv, nullptr, 0, t1, t2s, nullptr);
                    MXP_LAUNCHED();
                } else {
                    trsv_inv_kernel<2, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, X, b, xk, T, lda, nullptr, t1, nullptr);
                    MXP_LAUNCHED();
                    trsv_inv_kernel<4, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, T, lda, t1, nullptr, 0, xk, sv, nullptr);
                    MXP_LAUNCHED();
                    trsv_inv_kernel<2, kIvRowsDiag><<<dg, kIvThreads, smem, side>>>(b, b, X, b, sv, T, lda, t1, t2s, nullptr);
                    MXP_LAUNCHED();
                }
                MXP_CUDA(cudaEventRecord(ev[1], side));
                // rows of the next block (and x_k = t2) on the chain, after the bulk update of step s-1
                if (s >= 1 && bulk_step[(s - 1) & 1] == s - 1)
                    MXP_CUDA(cudaStreamWaitEvent(side, ev[2 + ((s - 1) & 1)], 0));
                const bool has_next = s + 1 < nb;
                const int64_t nx = lower ? kk + b : kk - b;  // first row of the next block
                // (on the chain: small row tiles, many CTAs)
                trsv_inv_kernel<0, kIvRowsDiag><<<has_next ? dg : 1, kIvThreads, smem, side>>>(
                    has_next ? b : 0, b, LU + (has_next ? nx : 0) + kk * lda, lda, t2s, nullptr, 0,
                    x + (has_next ? nx : 0), x + (has_next ? nx : 0), xk);
                MXP_LAUNCHED();
                // rows beyond the next block
                const int64_t r0 = lower ? kk + 2 * (int64_t)b : 0;
                const int rows = (int)(lower ? n - kk - 2 * (int64_t)b : kk - b);
                if (rows > 0) {
                    MXP_CUDA(cudaStreamWaitEvent(st, ev[1], 0));
                    trsv_inv_kernel<0, kIvRowsUpd><<<upd_grid(rows), kIvThreads, smem, st>>>(
                        rows, b, LU + r0 + kk * lda, lda, t2s, nullptr, 0, x + r0, x + r0, nullptr);
                    MXP_LAUNCHED();
                    MXP_CUDA(cudaEventRecord(ev[2 + (s & 1)], st));
                    bulk_step[s & 1] = s;
                }
            }
            MXP_CUDA(cudaEventRecord(ev[0], side));
            MXP_CUDA(cudaStreamWaitEvent(st, ev[0], 0));
        }
    }
    return MXP_OK;
}

mxp_status launch_infnorm(int n, const double *x, double *out, cudaStream_t st) {
    MXP_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (n <= 0) return MXP_OK;
    const int blocks = (int)imin64(cdiv(n, 256), 2 * num_sms());
    infnorm_kernel<<<blocks, 256, 0, st>>>(n, x, reinterpret_cast<unsigned long long *>(out));
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_norma(int n, const double *d, const double *rowsum, double *out, cudaStream_t st) {
    MXP_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (n <= 0) return MXP_OK;
    const int blocks = (int)imin64(cdiv(n, 256), 2 * num_sms());
    norma_kernel<<<blocks, 256, 0, st>>>(n, d, rowsum, reinterpret_cast<unsigned long long *>(out));
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_ir_init(int n, const double *rhs, const double *d, double *x, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    ir_init_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, rhs, d, x);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_copy(int n, const double *src, double *dst, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    copy_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, src, dst);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_axpy(int n, double alpha, const double *x, double *y, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    axpy_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, alpha, x, y);
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
