// SIMT FP32 building blocks shared by the cooperative diagonal-block
// factorisation (diag_coop.cu) and the batched solver (batched.cu): a
// 128 x 128 GEMM tile, the 64 x 64 no-pivot LU and the two 64-wide strip
// solves.  Every function is called by all kCT threads of the CTA (they
// contain __syncthreads) and reads its inputs through L2 (ld.global.cg), so it
// may follow writes made by other CTAs behind a grid barrier.
#pragma once

#include "mxp_internal.cuh"

namespace mxp {
namespace dt {
namespace {  // internal linkage: each translation unit keeps its own copy

constexpr int kCT = 256;  // threads per CTA
constexpr int kNB = 64;   // inner block of the LU
constexpr int GBM = 128, GBN = 128, GBK = 16;

struct SmemGemm {
    float As[GBK][GBM];
    float Bs[GBK][GBN + 4];
};
struct __align__(16) SmemTri {
    float t[kNB][kNB + 4];   // t[col][row] of a 64 x 64 block (16-byte rows)
    float tt[kNB][kNB + 4];  // tt[row][col]: the same block row-major
    float ub[kNB][kNB + 1];  // staging of 64 U-strip columns, ub[col][row]
    float prow[2][kNB];      // pivot row of the 64 x 64 LU, zero left of the pivot
    float dinv[kNB];
    float pivv[2];
};
union __align__(16) Smem {
    SmemGemm g;
    SmemTri t;
};


// ---- 128 x 128 SIMT GEMM tile ------------------------------------------------
// C[m0:m0+128, n0:n0+128] (clipped to m x n) = alpha * sum_{k in [kb, ke)} A(:,k) B(k,:)
// (+ C when accumulate).  8 x 8 outputs per thread.
// skip > 0 leaves the tile's top-left skip x skip corner untouched (another CTA
// owns it).
__device__ void gemm_tile(Smem &sm, int m, int n, int kb, int ke, float alpha,
                          const float *__restrict__ A, int64_t lda, const float *__restrict__ B,
                          int64_t ldb, bool accumulate, float *C, int64_t ldc, int m0, int n0,
                          int skip = 0) {
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

    float ra[8], rb[8];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + kCT * q;
            const int kk = idx / GBM, r = idx % GBM;
            const int gr = m0 + r, gk = k0 + kk;
            ra[q] = (gr < m && gk < ke) ? __ldcg(A + (int64_t)gk * lda + gr) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + kCT * q;
            const int cc = idx / GBK, kk = idx % GBK;
            const int gc = n0 + cc, gk = k0 + kk;
            rb[q] = (gc < n && gk < ke) ? __ldcg(B + (int64_t)gc * ldb + gk) : 0.0f;
        }
    };
    if (kb < ke) load(kb);
    for (int k0 = kb; k0 < ke; k0 += GBK) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + kCT * q;
            sm.g.As[idx / GBM][idx % GBM] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + kCT * q;
            sm.g.Bs[idx % GBK][idx / GBK] = rb[q];
        }
        __syncthreads();
        if (k0 + GBK < ke) load(k0 + GBK);
#pragma unroll
        for (int kk = 0; kk < GBK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&sm.g.As[kk][tx * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&sm.g.As[kk][64 + tx * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&sm.g.Bs[kk][ty * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&sm.g.Bs[kk][64 + ty * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
    }
    // C is read in full before any store: interleaved loads and stores through a
    // pointer the compiler cannot disambiguate would serialise 64 L2 round trips
    if (accumulate) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int gc = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int gr = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
                acc[i][j] *= alpha;
                if (gr < m && gc < n) acc[i][j] += __ldcg(C + (int64_t)gc * ldc + gr);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[i][j] *= alpha;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int gc = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
        if (gc >= n) continue;
        float *cc = C + (int64_t)gc * ldc;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int gr = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            if (gr < m && !(gr - m0 < skip && gc - n0 < skip)) cc[gr] = acc[i][j];
        }
    }
    __syncthreads();  // shared tiles are reused by the caller's next item
}

// C[0:m, 0:n] += alpha * A(:, 0:k) B(0:k, :) for m, n <= 64 (one 64 x 64 tile,
// 4 x 4 outputs per thread): the look-ahead update of the next diagonal block.
__device__ void gemm_tile64(Smem &sm, int m, int n, int k, float alpha, const float *__restrict__ A, int64_t lda,
                            const float *__restrict__ B, int64_t ldb, float *C, int64_t ldc) {
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < k; k0 += GBK) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = t + kCT * q;           // 0..1023
            const int kk = idx / 64, r = idx % 64;
            const int gk = k0 + kk;
            sm.g.As[kk][r] = (r < m && gk < k) ? __ldcg(A + (int64_t)gk * lda + r) : 0.0f;
            const int c = idx / GBK, kb = idx % GBK;
            const int gkb = k0 + kb;
            sm.g.Bs[kb][c] = (c < n && gkb < k) ? __ldcg(B + (int64_t)c * ldb + gkb) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GBK; ++kk) {
            const float4 a = *reinterpret_cast<const float4 *>(&sm.g.As[kk][tx * 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&sm.g.Bs[kk][ty * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int gc = ty * 4 + j;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gr = tx * 4 + i;
            acc[i][j] *= alpha;
            if (gr < m && gc < n) acc[i][j] += __ldcg(C + (int64_t)gc * ldc + gr);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int gc = ty * 4 + j;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gr = tx * 4 + i;
            if (gr < m && gc < n) C[(int64_t)gc * ldc + gr] = acc[i][j];
        }
    }
    __syncthreads();
}

// ---- 64 x 64 no-pivot LU of D (nb <= 64), one row per thread of warps 0-1 ----
// sgetrf_nopiv_naive order (sgetrf_nopiv.cpp:27-61): scale by the reciprocal
// pivot, then the rank-1 update.  The two working warps meet at a 64-thread
// named barrier once per pivot; the rest of the CTA waits at the final
// __syncthreads.
__device__ __forceinline__ void bar_sync_rows() { asm volatile("bar.sync 1, 64;" ::: "memory"); }

__device__ void getrf64(Smem &sm, int nb, float *D, int64_t lda, DevStatus *dst, int pivot_base) {
    const int i = threadIdx.x;
    if (i < kNB) {
        float a[kNB];
#pragma unroll
        for (int j = 0; j < kNB; ++j) a[j] = (i < nb && j < nb) ? __ldcg(D + (int64_t)j * lda + i) : 0.0f;
#pragma unroll
        for (int k = 0; k < kNB; ++k) {
            if (k < nb) {  // uniform
                float *pr = sm.t.prow[k & 1];
                if (i == k) {  // publish the pivot row, zero at and left of the pivot
#pragma unroll
                    for (int j4 = k / 4; j4 < kNB / 4; ++j4) {
                        float4 v;
                        v.x = (4 * j4 + 0 > k) ? a[4 * j4 + 0] : 0.0f;
                        v.y = (4 * j4 + 1 > k) ? a[4 * j4 + 1] : 0.0f;
                        v.z = (4 * j4 + 2 > k) ? a[4 * j4 + 2] : 0.0f;
                        v.w = (4 * j4 + 3 > k) ? a[4 * j4 + 3] : 0.0f;
                        *reinterpret_cast<float4 *>(pr + 4 * j4) = v;
                    }
                    sm.t.pivv[k & 1] = a[k];
                }
                bar_sync_rows();
                const float piv = sm.t.pivv[k & 1];
                if (i == k && (!(piv != 0.0f) || !isfinite(piv))) report(dst, MXP_ZERO_PIVOT, pivot_base + k + 1, 0);
                const bool act = i > k && i < nb;
                const float l = act ? a[k] * __frcp_rn(piv) : 0.0f;
                if (act) a[k] = l;
                // a(i, j) -= l * u(k, j) for j > k; the zeros of the published row
                // leave columns <= k untouched (and rows <= k have l = 0)
#pragma unroll
                for (int j4 = k / 4; j4 < kNB / 4; ++j4) {
                    const float4 p = *reinterpret_cast<const float4 *>(pr + 4 * j4);
                    if (4 * j4 + 0 > k) a[4 * j4 + 0] = fmaf(-l, p.x, a[4 * j4 + 0]);
                    if (4 * j4 + 1 > k) a[4 * j4 + 1] = fmaf(-l, p.y, a[4 * j4 + 1]);
                    if (4 * j4 + 2 > k) a[4 * j4 + 2] = fmaf(-l, p.z, a[4 * j4 + 2]);
                    if (4 * j4 + 3 > k) a[4 * j4 + 3] = fmaf(-l, p.w, a[4 * j4 + 3]);
                }
            }
        }
        if (i < nb) {
#pragma unroll
            for (int j = 0; j < kNB; ++j)
                if (j < nb) D[(int64_t)j * lda + i] = a[j];
        }
    }
    __syncthreads();
}

// D (nb x nb, factored) into shared memory, t[col][row], plus reciprocal diagonal.
__device__ void load_tri(Smem &sm, int nb, const float *D, int64_t lda) {
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int r = idx % kNB, c = idx / kNB;
        const float v = (r < nb && c < nb) ? __ldcg(D + (int64_t)c * lda + r) : 0.0f;
        sm.t.t[c][r] = v;
        sm.t.tt[r][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < nb) sm.t.dinv[threadIdx.x] = 1.0f / sm.t.t[threadIdx.x][threadIdx.x];
    __syncthreads();
}

// L strip rows [r0, r0 + rows) of B (m x nb), rows <= kCT: X = B U^{-1}, U =
// upper part of the diagonal block in sm.t.  Right-looking (x_k final, then
// x_c -= u_kc x_k for c > k): per element the same operations in the same
// order as the dot-product form, with independent updates instead of one
// dependent chain per row; u_k. is read four at a time from the row-major copy.
__device__ void trsm_rows(Smem &sm, int m, int nb, float *B, int64_t ldb, int r0, int rows = kCT) {
    const int i = r0 + threadIdx.x;
    if (threadIdx.x >= rows || i >= m) return;
    float x[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) x[c] = (c < nb) ? __ldcg(B + (int64_t)c * ldb + i) : 0.0f;
#pragma unroll
    for (int k = 0; k < kNB; ++k) {
        if (k < nb) {
            x[k] *= sm.t.dinv[k];
#pragma unroll
            for (int c4 = (k + 1) / 4; c4 < kNB / 4; ++c4) {
                const float4 u = *reinterpret_cast<const float4 *>(&sm.t.tt[k][4 * c4]);
                if (4 * c4 + 0 > k) x[4 * c4 + 0] = fmaf(-u.x, x[k], x[4 * c4 + 0]);
                if (4 * c4 + 1 > k) x[4 * c4 + 1] = fmaf(-u.y, x[k], x[4 * c4 + 1]);
                if (4 * c4 + 2 > k) x[4 * c4 + 2] = fmaf(-u.z, x[k], x[4 * c4 + 2]);
                if (4 * c4 + 3 > k) x[4 * c4 + 3] = fmaf(-u.w, x[k], x[4 * c4 + 3]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        if (c < nb) B[(int64_t)c * ldb + i] = x[c];
}

// U strip columns [c0, c0 + 64) of B (nb x ncols): X = L^{-1} B, L = unit lower
// part of sm.t.  The 64 x 64 block moves through shared memory with coalesced
// loads and stores; threads 0..63 solve one column each.
__device__ void trsm_cols64(Smem &sm, int ncols, int nb, float *B, int64_t ldb, int c0) {
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int k = idx % kNB, j = idx / kNB;
        sm.t.ub[j][k] = (k < nb && c0 + j < ncols) ? __ldcg(B + (int64_t)(c0 + j) * ldb + k) : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x < kNB) {  // right-looking: x_r -= l_rk x_k for r > k (l_.k contiguous in sm.t)
        const int j = threadIdx.x;
        float x[kNB];
#pragma unroll
        for (int k = 0; k < kNB; ++k) x[k] = sm.t.ub[j][k];
#pragma unroll
        for (int k = 0; k < kNB - 1; ++k) {
            if (k < nb) {
#pragma unroll
                for (int r4 = (k + 1) / 4; r4 < kNB / 4; ++r4) {
                    const float4 l = *reinterpret_cast<const float4 *>(&sm.t.t[k][4 * r4]);
                    if (4 * r4 + 0 > k) x[4 * r4 + 0] = fmaf(-l.x, x[k], x[4 * r4 + 0]);
                    if (4 * r4 + 1 > k) x[4 * r4 + 1] = fmaf(-l.y, x[k], x[4 * r4 + 1]);
                    if (4 * r4 + 2 > k) x[4 * r4 + 2] = fmaf(-l.z, x[k], x[4 * r4 + 2]);
                    if (4 * r4 + 3 > k) x[4 * r4 + 3] = fmaf(-l.w, x[k], x[4 * r4 + 3]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kNB; ++k) sm.t.ub[j][k] = x[k];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int k = idx % kNB, j = idx / kNB;
        if (k < nb && c0 + j < ncols) B[(int64_t)(c0 + j) * ldb + k] = sm.t.ub[j][k];
    }
    __syncthreads();
}

// Inverse of the 64 x 64 diagonal block `blk` of an upper non-unit (upper = true)
// or unit-lower triangle; row i of the inverse solves x T = e_i.
__device__ void inv_diag_block(Smem &sm, int n, const float *T, int64_t ldt, float *X, int64_t ldx,
                               int blk, bool upper) {
    const int r0 = blk * kNB;
    const int nb = min(kNB, n - r0);
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int r = idx % kNB, c = idx / kNB;
        sm.t.t[c][r] = (r < nb && c < nb) ? __ldcg(T + (int64_t)(r0 + c) * ldt + r0 + r) : 0.0f;
    }
    __syncthreads();
    const int i = threadIdx.x;
    if (i < nb) {
        float x[kNB];
        if (upper) {
#pragma unroll
            for (int j = 0; j < kNB; ++j) {
                float v = (j == i) ? 1.0f : 0.0f;
#pragma unroll
                for (int q = 0; q < j; ++q) v -= x[q] * sm.t.t[j][q];
                x[j] = (j >= i && j < nb) ? v / sm.t.t[j][j] : 0.0f;
            }
        } else {
#pragma unroll
            for (int jj = 0; jj < kNB; ++jj) {
                const int j = kNB - 1 - jj;
                float v = (j == i) ? 1.0f : 0.0f;
#pragma unroll
                for (int q = j + 1; q < kNB; ++q) v -= x[q] * sm.t.t[j][q];
                x[j] = (j <= i) ? v : 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < kNB; ++j)
            if (j < nb) X[(int64_t)(r0 + j) * ldx + r0 + i] = x[j];
    }
    __syncthreads();
}

// One batched GEMM of an inverse level.  tri: which operand is triangular, so
// its zero half is skipped along K: 1 A upper, 2 A lower, 3 B upper, 4 B lower.
struct Job {
    int m, n, K, batch, tri;
    float alpha;
    const float *A;
    int64_t lda, sA;
    const float *B;
    int64_t ldb, sB;
    float *C;
    int64_t ldc, sC;
};

__device__ void run_jobs(Smem &sm, const Job *jobs, int njobs, int cta, int ncta) {
    int tiles[4] = {0, 0, 0, 0}, total = 0;
    for (int q = 0; q < njobs; ++q) {
        tiles[q] = ((jobs[q].m + GBM - 1) / GBM) * ((jobs[q].n + GBN - 1) / GBN) * jobs[q].batch;
        total += tiles[q];
    }
    for (int it = cta; it < total; it += ncta) {
        int q = 0, r = it;
        while (r >= tiles[q]) r -= tiles[q++];
        const Job &J = jobs[q];
        const int tm = (J.m + GBM - 1) / GBM, tn = (J.n + GBN - 1) / GBN;
        const int z = r / (tm * tn);
        const int rt = r % (tm * tn);
        const int m0 = (rt % tm) * GBM, n0 = (rt / tm) * GBN;
        int kb = 0, ke = J.K;
        if (J.tri == 1) kb = m0;
        if (J.tri == 2) ke = min(J.K, m0 + GBM);
        if (J.tri == 3) ke = min(J.K, n0 + GBN);
        if (J.tri == 4) kb = n0;
        gemm_tile(sm, J.m, J.n, kb, ke, J.alpha, J.A + J.sA * z, J.lda, J.B + J.sB * z, J.ldb, false,
                  J.C + J.sC * z, J.ldc, m0, n0);
    }
}

// inv(U) -> XU and inv(L) -> XL (unit lower) of the factored n x n block A, by
// recursive doubling: 64 x 64 diagonal blocks first, then for adjacent
// S-blocks the off-diagonal block of the inverse is -inv(A) B inv(C), two GEMM
// phases per level with both triangles in the same phases and the zero half of
// every triangular operand skipped along K.  Work items are spread over
// (cta, ncta); sync(where) separates the phases (a grid barrier across CTAs or
// __syncthreads in a single CTA) and returns false to stop.  tmpU / tmpL hold
// n*n/2 + 64 n floats each.  s_stop > 0: stop before the level that joins
// blocks of size s_stop (the caller finishes those levels elsewhere).
template <typename Sync>
__device__ bool tri_inverses(Smem &sm, int n, const float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                             float *tmpU, float *tmpL, int cta, int G, Sync sync, int s_stop = 0) {
    const int nsteps = (n + kNB - 1) / kNB;
    // invert the diagonal 64 x 64 blocks and zero the opposite block-triangle
    const int nblk = nsteps;
    for (int it = cta; it < 2 * nblk; it += G)
        inv_diag_block(sm, n, A, lda, it < nblk ? XU : XL, ldx, it % nblk, it < nblk);
    for (int64_t idx = (int64_t)cta * kCT + threadIdx.x; idx < (int64_t)n * n; idx += (int64_t)G * kCT) {
        const int r = (int)(idx % n), c = (int)(idx / n);
        if (r / kNB > c / kNB) XU[(int64_t)c * ldx + r] = 0.0f;
        if (r / kNB < c / kNB) XL[(int64_t)c * ldx + r] = 0.0f;
    }
    if (!sync(23)) return false;

    const float *U = A, *L = A;
    const int64_t ldu = lda, ldl = lda;
    for (int S = kNB; S < n && (s_stop <= 0 || S < s_stop); S *= 2) {
        const int np = n / (2 * S);
        const int rem = n - np * 2 * S;
        const int c = rem - S;  // ragged last pair (when > 0)
        const int64_t r0 = (int64_t)np * 2 * S;
        const int64_t stepX = 2 * (int64_t)S * (1 + ldx), stepA = 2 * (int64_t)S * (1 + lda);
        const int64_t SS = (int64_t)S * S;
        Job jb[4];
        int nj = 0;
        // phase a:  T_U = U12 inv(U22);  T_L = L21 inv(L11)
        if (np > 0) {
            jb[nj++] = Job{S, S, S, np, 3, 1.0f, U + (int64_t)S * ldu, ldu, stepA, XU + S + (int64_t)S * ldx,
                           ldx, stepX, tmpU, S, SS};
            jb[nj++] = Job{S, S, S, np, 4, 1.0f, L + S, ldl, stepA, XL, ldx, stepX, tmpL, S, SS};
        }
        if (c > 0) {
            jb[nj++] = Job{S, c, c, 1, 3, 1.0f, U + r0 + (r0 + S) * ldu, ldu, 0,
                           XU + (r0 + S) + (r0 + S) * ldx, ldx, 0, tmpU + np * SS, S, 0};
            jb[nj++] = Job{c, S, S, 1, 4, 1.0f, L + (r0 + S) + r0 * ldl, ldl, 0, XL + r0 + r0 * ldx, ldx, 0,
                           tmpL + np * SS, c, 0};
        }
        run_jobs(sm, jb, nj, cta, G);
        if (!sync(24)) return false;
        // phase b:  X12 = -inv(U11) T_U;  X21 = -inv(L22) T_L
        nj = 0;
        if (np > 0) {
            jb[nj++] = Job{S, S, S, np, 1, -1.0f, XU, ldx, stepX, tmpU, S, SS, XU + (int64_t)S * ldx, ldx, stepX};
            jb[nj++] = Job{S, S, S, np, 2, -1.0f, XL + S + (int64_t)S * ldx, ldx, stepX, tmpL, S, SS, XL + S,
                           ldx, stepX};
        }
        if (c > 0) {
            jb[nj++] = Job{S, c, S, 1, 1, -1.0f, XU + r0 + r0 * ldx, ldx, 0, tmpU + np * SS, S, 0,
                           XU + r0 + (r0 + S) * ldx, ldx, 0};
            jb[nj++] = Job{c, S, c, 1, 2, -1.0f, XL + (r0 + S) + (r0 + S) * ldx, ldx, 0, tmpL + np * SS, c, 0,
                           XL + (r0 + S) + r0 * ldx, ldx, 0};
        }
        run_jobs(sm, jb, nj, cta, G);
        if (!sync(25)) return false;
    }
    return true;
}

}  // namespace
}  // namespace dt
}  // namespace mxp
