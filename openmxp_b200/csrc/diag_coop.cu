// Cooperative factorisation of one diagonal block in a single launch: the
// FP32 no-pivot LU (GPUSOLVER_SGETRF with ipiv = NULL, panel_trf.hpp:547-551,
// 678-681) followed, optionally, by the inverses of its two triangles (the
// operands of the tensor-core TRSM-by-inverse; the reference builds them for
// its -alt path with STRSM on an identity, panel_trf_gdirect.hpp:73-92).
//
// The per-step launch chain of the blocked LU (a 64 x 64 factor, two strip
// solves and a rank-64 update per 64 columns, about 160 launches for a
// 2560 block, plus ~30 for the inverses) is latency-bound: each piece is a
// few microseconds of work.  Here one persistent grid (one CTA per SM, all
// co-resident through a cooperative launch) runs the same steps separated by
// grid barriers:
//
//   LU, for each 64-column step j (D_j = diagonal 64 x 64 block):
//     strips : L strip rows (thread per row, X = B U_jj^{-1}) and U strip
//              columns (thread per column, X = L_jj^{-1} B) against D_j held
//              in shared memory, items of 256 rows / columns over all CTAs;
//     update : trailing rank-64 update in 128 x 128 SIMT tiles.  CTA 0 takes
//              the tile holding D_{j+1} alone and factors D_{j+1} right after
//              it (look-ahead, four threads per row), so the 64-step serial
//              factor overlaps the rest of the update.
//   inverses: 64 x 64 diagonal blocks of inv(U) and inv(L) one per item,
//             then recursive doubling: for adjacent S-blocks the off-diagonal
//             block of the inverse is -inv(A) B inv(C), two GEMM phases per
//             level, with the U and L triangles in the same phases and the
//             zero half of every triangular operand skipped along K.
//
// Grid barriers are a counter in global memory (zeroed on the stream before
// each launch) with release/acquire ordering; every wait is bounded by
// kWaitTimeoutNs, after which the CTA records MXP_TIMEOUT, raises the shared
// abort word so the others leave at their next barrier, and returns.
// All reads of data written by other CTAs go through L2 (ld.global.cg).
#include "mxp_internal.cuh"

namespace mxp {

namespace {

constexpr int kCT = 256;  // threads per CTA
constexpr int kNB = 64;   // inner block of the LU
constexpr int GBM = 128, GBN = 128, GBK = 16;

struct SmemGemm {
    float As[GBK][GBM];
    float Bs[GBK][GBN + 4];
};
struct SmemTri {
    float t[kNB][kNB + 1];  // t[col][row] of a 64 x 64 block
    float dinv[kNB];
    float prow[2][kNB];
};
union __align__(16) Smem {
    SmemGemm g;
    SmemTri t;
};

struct Ctl {
    unsigned int *count;  // grid-barrier arrivals (zero at launch)
    int *abort;           // set by a CTA that gave up waiting
    DevStatus *dst;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier.  Returns false (in every thread of the CTA) when the
// wait timed out or another CTA aborted.
__device__ bool grid_sync(const Ctl &c, unsigned int &epoch, int where) {
    __shared__ int ok_sh;
    __syncthreads();
    epoch += gridDim.x;
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(c.count, 1u);
        const unsigned long long t0 = globaltimer_ns();
        while (ld_acquire_u32(c.count) < epoch) {
            if (ld_relaxed_i32(c.abort)) {
                ok = 0;
                break;
            }
            if (globaltimer_ns() - t0 > kWaitTimeoutNs) {
                ok = 0;
                atomicExch(c.abort, 1);
                report(c.dst, MXP_TIMEOUT, where, blockIdx.x);
                break;
            }
            __nanosleep(64);
        }
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

// ---- 128 x 128 SIMT GEMM tile ------------------------------------------------
// C[m0:m0+128, n0:n0+128] (clipped to m x n) = alpha * sum_{k in [kb, ke)} A(:,k) B(k,:)
// (+ C when accumulate).  8 x 8 outputs per thread.
__device__ void gemm_tile(Smem &sm, int m, int n, int kb, int ke, float alpha,
                          const float *__restrict__ A, int64_t lda, const float *__restrict__ B,
                          int64_t ldb, bool accumulate, float *C, int64_t ldc, int m0, int n0) {
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
            if (gr < m) cc[gr] = acc[i][j];
        }
    }
    __syncthreads();  // shared tiles are reused by the caller's next item
}

// ---- 64 x 64 no-pivot LU of D (nb <= 64): four threads per row, 16 columns each ----
// sgetrf_nopiv_naive order (sgetrf_nopiv.cpp:27-61): scale by the reciprocal
// pivot, then the rank-1 update.  Thread (row i, quarter q) holds a(i, 16q..16q+15)
// in registers; the four threads of a row are adjacent lanes of one warp, so the
// multiplier is shared by a shuffle.  All CTA threads pass the barriers.
__device__ void getrf64(Smem &sm, int nb, float *D, int64_t lda, DevStatus *dst, int pivot_base) {
    const int i = threadIdx.x >> 2, q = threadIdx.x & 3;
    const int lane_base = (threadIdx.x & 31) & ~3;
    float a[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        const int col = q * 16 + c;
        a[c] = (i < nb && col < nb) ? __ldcg(D + (int64_t)col * lda + i) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kNB; ++k) {
        if (k < nb) {  // uniform across the CTA
            const int qk = k >> 4, ck = k & 15;
            if (i == k) {
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (q * 16 + c >= k) sm.t.prow[k & 1][q * 16 + c] = a[c];
            }
            __syncthreads();
            const float piv = sm.t.prow[k & 1][k];
            if (i == k && q == qk && (!(piv != 0.0f) || !isfinite(piv)))
                report(dst, MXP_ZERO_PIVOT, pivot_base + k + 1, 0);
            const float rcp = 1.0f / piv;
            float l = (q == qk) ? a[ck] * rcp : 0.0f;
            l = __shfl_sync(0xffffffffu, l, lane_base + qk);
            if (i > k && i < nb) {
                if (q == qk) a[ck] = l;
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (q * 16 + c > k) a[c] -= l * sm.t.prow[k & 1][q * 16 + c];
            }
        }
    }
    if (i < nb) {
#pragma unroll
        for (int c = 0; c < 16; ++c)
            if (q * 16 + c < nb) D[(int64_t)(q * 16 + c) * lda + i] = a[c];
    }
    __syncthreads();
}

// D (nb x nb, factored) into shared memory, t[col][row], plus reciprocal diagonal.
__device__ void load_tri(Smem &sm, int nb, const float *D, int64_t lda) {
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int r = idx % kNB, c = idx / kNB;
        sm.t.t[c][r] = (r < nb && c < nb) ? __ldcg(D + (int64_t)c * lda + r) : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x < nb) sm.t.dinv[threadIdx.x] = 1.0f / sm.t.t[threadIdx.x][threadIdx.x];
    __syncthreads();
}

// L strip rows [r0, r0 + 256) of B (m x nb): X = B U^{-1}, U = upper part of sm.t.
__device__ void trsm_rows(Smem &sm, int m, int nb, float *B, int64_t ldb, int r0) {
    const int i = r0 + threadIdx.x;
    if (i >= m) return;
    float x[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) x[c] = (c < nb) ? __ldcg(B + (int64_t)c * ldb + i) : 0.0f;
#pragma unroll
    for (int c = 0; c < kNB; ++c) {
        if (c < nb) {
            float v = x[c];
#pragma unroll
            for (int k = 0; k < c; ++k) v -= sm.t.t[c][k] * x[k];
            x[c] = v * sm.t.dinv[c];
        }
    }
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        if (c < nb) B[(int64_t)c * ldb + i] = x[c];
}

// U strip columns [c0, c0 + 256) of B (nb x ncols): X = L^{-1} B, L = unit lower
// part of sm.t; one thread per column, the column's nb values in registers.
__device__ void trsm_cols(Smem &sm, int ncols, int nb, float *B, int64_t ldb, int c0) {
    const int j = c0 + threadIdx.x;
    if (j >= ncols) return;
    float *bj = B + (int64_t)j * ldb;
    float x[kNB];
#pragma unroll
    for (int k = 0; k < kNB; ++k) x[k] = (k < nb) ? __ldcg(bj + k) : 0.0f;
#pragma unroll
    for (int r = 1; r < kNB; ++r) {
        if (r < nb) {
            float v = x[r];
#pragma unroll
            for (int k = 0; k < r; ++k) v -= sm.t.t[k][r] * x[k];
            x[r] = v;
        }
    }
#pragma unroll
    for (int k = 0; k < kNB; ++k)
        if (k < nb) bj[k] = x[k];
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

__global__ void __launch_bounds__(kCT, 1)
diag_factor_kernel(int n, float *A, int64_t lda, float *XU, float *XL, int64_t ldx, float *tmpU,
                   float *tmpL, Ctl ctl, int pivot_base) {
    __shared__ Smem sm;
    const int G = gridDim.x, cta = blockIdx.x;
    unsigned int epoch = 0;
    const int nsteps = (n + kNB - 1) / kNB;

    // ---------------- LU ----------------
    if (cta == 0) getrf64(sm, min(kNB, n), A, lda, ctl.dst, pivot_base);
    if (!grid_sync(ctl, epoch, 20)) return;
    for (int j = 0; j < nsteps; ++j) {
        const int jb = j * kNB;
        const int nbk = min(kNB, n - jb);
        const int rem = n - jb - nbk;
        if (rem <= 0) break;
        float *Djj = A + jb + (int64_t)jb * lda;
        float *Lstrip = Djj + nbk;
        float *Ustrip = Djj + (int64_t)nbk * lda;
        // strips
        const int lit = (rem + kCT - 1) / kCT, uit = (rem + kCT - 1) / kCT;
        if (cta < lit + uit) {
            load_tri(sm, nbk, Djj, lda);
            for (int it = cta; it < lit + uit; it += G) {
                if (it < lit) trsm_rows(sm, rem, nbk, Lstrip, lda, it * kCT);
                else trsm_cols(sm, rem, nbk, Ustrip, lda, (it - lit) * kCT);
            }
        }
        if (!grid_sync(ctl, epoch, 21)) return;
        // trailing rank-nbk update; CTA 0 also factors the next diagonal block
        float *C = Ustrip + nbk;
        const int tm = (rem + GBM - 1) / GBM;
        const int ntiles = tm * tm;
        if (G == 1 || cta == 0) {
            for (int t = 0; t < (G == 1 ? ntiles : 1); ++t)
                gemm_tile(sm, rem, rem, 0, nbk, -1.0f, Lstrip, lda, Ustrip, lda, true, C, lda,
                          (t % tm) * GBM, (t / tm) * GBN);
            getrf64(sm, min(kNB, rem), C, lda, ctl.dst, pivot_base + jb + nbk);
        } else {
            for (int t = cta; t < ntiles; t += G - 1)
                gemm_tile(sm, rem, rem, 0, nbk, -1.0f, Lstrip, lda, Ustrip, lda, true, C, lda,
                          (t % tm) * GBM, (t / tm) * GBN);
        }
        if (!grid_sync(ctl, epoch, 22)) return;
    }
    if (!XU) return;

    // ---------------- triangular inverses ----------------
    // invert the diagonal 64 x 64 blocks and zero the opposite block-triangle
    const int nblk = nsteps;
    for (int it = cta; it < 2 * nblk; it += G)
        inv_diag_block(sm, n, A, lda, it < nblk ? XU : XL, ldx, it % nblk, it < nblk);
    for (int64_t idx = (int64_t)cta * kCT + threadIdx.x; idx < (int64_t)n * n; idx += (int64_t)G * kCT) {
        const int r = (int)(idx % n), c = (int)(idx / n);
        if (r / kNB > c / kNB) XU[(int64_t)c * ldx + r] = 0.0f;
        if (r / kNB < c / kNB) XL[(int64_t)c * ldx + r] = 0.0f;
    }
    if (!grid_sync(ctl, epoch, 23)) return;

    const float *U = A, *L = A;
    const int64_t ldu = lda, ldl = lda;
    for (int S = kNB; S < n; S *= 2) {
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
        if (!grid_sync(ctl, epoch, 24)) return;
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
        if (!grid_sync(ctl, epoch, 25)) return;
    }
}

int coop_grid(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) return 0;
    if (!cached[device]) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_factor_kernel, kCT, 0);
        cached[device] = per_sm > 0 ? sms : -1;
    }
    return cached[device];
}

}  // namespace

size_t diag_factor_tmp_floats(int n) { return (size_t)n * n / 2 + (size_t)64 * n; }

mxp_status launch_diag_factor(int n, float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                              float *tmpU, float *tmpL, unsigned int *sync_words, DevStatus *dst,
                              int pivot_base, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    if (lda < n || (XU && ldx < n)) return fail(MXP_INVALID_ARG, "diag_factor: bad leading dimension");
    if ((XU == nullptr) != (XL == nullptr)) return fail(MXP_INVALID_ARG, "diag_factor: both inverses or none");
    if (XU && (!tmpU || !tmpL)) return fail(MXP_INVALID_ARG, "diag_factor: inverse scratch missing");
    int dev = 0;
    MXP_CUDA(cudaGetDevice(&dev));
    const int sms = coop_grid(dev);
    if (sms <= 0) return fail(MXP_UNSUPPORTED, "diag_factor: kernel cannot be made resident");
    const int tm = (n + GBM - 1) / GBM;
    int grid = min(sms, max(2, tm * tm));
    MXP_CUDA(cudaMemsetAsync(sync_words, 0, 2 * sizeof(unsigned int), st));
    Ctl ctl{sync_words, reinterpret_cast<int *>(sync_words + 1), dst};
    void *args[] = {&n, &A, &lda, &XU, &XL, &ldx, &tmpU, &tmpL, &ctl, &pivot_base};
    MXP_CUDA(cudaLaunchCooperativeKernel((const void *)diag_factor_kernel, dim3(grid), dim3(kCT), args, 0, st));
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
