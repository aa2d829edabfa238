// FP32 dense kernels of the panel factorisation: the diagonal-block no-pivot
// LU and the two panel TRSMs, blocked by 64 with a shared-memory /
// register kernel for each 64-wide triangle and a SIMT FP32 GEMM for the
// rank-64 updates.
//
// Reference: GPUSOLVER_SGETRF -> rocsolver_sgetrf_npvt / cusolverDnSgetrf
// with ipiv = NULL (panel_trf.hpp:547-551, 678-681); GPUBLAS_STRSM
// (R,U,N,NonUnit) for the L panel (panel_trf.hpp:188-207) and (L,L,N,Unit)
// for the U panel (panel_trf.hpp:225-246).  The unblocked kernel follows
// sgetrf_nopiv_naive (sgetrf_nopiv.cpp:27-61): scale the column by the
// reciprocal pivot, then a rank-1 update.
#include "mxp_internal.cuh"

namespace mxp {

namespace {

constexpr int kNB = 64;  // inner block of the blocked LU / TRSM

// ---- 64 x 64 no-pivot LU, one row per thread in registers -----------------
// Step k: the owner of row k publishes it to shared memory; every row below
// scales its column-k entry by the reciprocal pivot and applies the rank-1
// update (sgetrf_nopiv_naive order, sgetrf_nopiv.cpp:27-61).  One barrier
// per step.
__global__ void __launch_bounds__(kNB)
getrf_small_kernel(int nb, float *A, int64_t lda, DevStatus *dst, int pivot_base) {
    __shared__ float prow[2][kNB];
    const int i = threadIdx.x;
    float a[kNB];
#pragma unroll
    for (int j = 0; j < kNB; ++j) a[j] = (i < nb && j < nb) ? A[(int64_t)j * lda + i] : 0.0f;
#pragma unroll
    for (int k = 0; k < kNB; ++k) {
        if (k < nb) {
            if (i == k) {
#pragma unroll
                for (int j = 0; j < kNB; ++j)
                    if (j >= k) prow[k & 1][j] = a[j];
            }
            __syncthreads();
            const float piv = prow[k & 1][k];
            if (i == k && (!(piv != 0.0f) || !isfinite(piv))) report(dst, MXP_ZERO_PIVOT, pivot_base + k + 1, 0);
            if (i > k && i < nb) {
                const float l = a[k] * (1.0f / piv);
                a[k] = l;
#pragma unroll
                for (int j = 0; j < kNB; ++j)
                    if (j > k) a[j] -= l * prow[k & 1][j];
            }
        }
    }
    if (i < nb) {
#pragma unroll
        for (int j = 0; j < kNB; ++j)
            if (j < nb) A[(int64_t)j * lda + i] = a[j];
    }
}

// ---- X = B * U^{-1}, U (nb x nb) upper non-unit; one thread per row -------
__global__ void __launch_bounds__(128)
trsm_runn_small_kernel(int m, int nb, const float *U, int64_t ldu, float *B, int64_t ldb) {
    __shared__ float u[kNB][kNB + 1];  // u[col][row]
    __shared__ float uinv[kNB];
    for (int idx = threadIdx.x; idx < nb * nb; idx += 128) {
        const int r = idx % nb, c = idx / nb;
        u[c][r] = U[(int64_t)c * ldu + r];
    }
    __syncthreads();
    if (threadIdx.x < nb) uinv[threadIdx.x] = 1.0f / u[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * 128 + threadIdx.x;
    if (i >= m) return;
    float x[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) x[c] = (c < nb) ? B[(int64_t)c * ldb + i] : 0.0f;
#pragma unroll
    for (int c = 0; c < kNB; ++c) {
        if (c < nb) {
            float v = x[c];
#pragma unroll
            for (int k = 0; k < c; ++k) v -= u[c][k] * x[k];
            x[c] = v * uinv[c];
        }
    }
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        if (c < nb) B[(int64_t)c * ldb + i] = x[c];
}

// ---- X = L^{-1} B, L (nb x nb) unit lower; one warp per column ------------
__global__ void __launch_bounds__(256)
trsm_llnu_small_kernel(int ncols, int nb, const float *L, int64_t ldl, float *B, int64_t ldb) {
    __shared__ float l[kNB][kNB + 1];  // l[col][row]
    for (int idx = threadIdx.x; idx < nb * nb; idx += 256) {
        const int r = idx % nb, c = idx / nb;
        l[c][r] = L[(int64_t)c * ldl + r];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t col0 = (int64_t)blockIdx.x * 64;
    for (int cc = warp; cc < 64; cc += 8) {
        const int64_t j = col0 + cc;
        if (j >= ncols) break;
        float *bj = B + j * ldb;
        float x0 = (lane < nb) ? bj[lane] : 0.0f;
        float x1 = (lane + 32 < nb) ? bj[lane + 32] : 0.0f;
        for (int k = 0; k < nb; ++k) {
            const float xk = __shfl_sync(0xffffffffu, k < 32 ? x0 : x1, k & 31);
            if (lane > k) x0 -= l[k][lane] * xk;
            if (lane + 32 > k && lane + 32 < nb) x1 -= l[k][lane + 32] * xk;
        }
        if (lane < nb) bj[lane] = x0;
        if (lane + 32 < nb) bj[lane + 32] = x1;
    }
}

// ---- C -= A * B, FP32 SIMT GEMM, 128 x 128 tiles, 8 x 8 per thread --------
constexpr int BM = 128, BN = 128, BK = 16;

// C_z = alpha * A_z * B_z + beta * C_z for batch z = blockIdx.z (pointer strides
// sA, sB, sC); beta == 0 does not read C.
__global__ void __launch_bounds__(256)
sgemm_kernel(int m, int n, int k, float alpha, const float *__restrict__ A, int64_t lda,
             int64_t sA, const float *__restrict__ B, int64_t ldb, int64_t sB, float beta,
             float *__restrict__ C, int64_t ldc, int64_t sC) {
    __shared__ __align__(16) float As[BK][BM];
    __shared__ __align__(16) float Bs[BK][BN + 4];
    A += sA * blockIdx.z;
    B += sB * blockIdx.z;
    C += sC * blockIdx.z;
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    const int64_t m0 = (int64_t)blockIdx.x * BM, n0 = (int64_t)blockIdx.y * BN;

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

    float ra[8], rb[8];
    auto load_tile = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + 256 * q;
            const int kk = idx / BM, r = idx % BM;
            const int64_t gr = m0 + r;
            const int gk = k0 + kk;
            ra[q] = (gr < m && gk < k) ? A[(int64_t)gk * lda + gr] : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + 256 * q;
            const int c = idx / BK, kk = idx % BK;
            const int64_t gc = n0 + c;
            const int gk = k0 + kk;
            rb[q] = (gc < n && gk < k) ? B[gc * ldb + gk] : 0.0f;
        }
    };
    auto store_tile = [&]() {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + 256 * q;
            As[idx / BM][idx % BM] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = t + 256 * q;
            Bs[idx % BK][idx / BK] = rb[q];
        }
    };

    load_tile(0);
    for (int k0 = 0; k0 < k; k0 += BK) {
        __syncthreads();
        store_tile();
        __syncthreads();
        if (k0 + BK < k) load_tile(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[kk][tx * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[kk][64 + tx * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[kk][ty * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[kk][64 + ty * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
    }
    // C is read in full before any store (loads interleaved with stores through
    // one pointer would be serialised by the compiler)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t gc = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t gr = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            acc[i][j] *= alpha;
            if (beta != 0.0f && gr < m && gc < n) acc[i][j] += beta * C[gc * ldc + gr];
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t gc = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
        if (gc >= n) continue;
        float *cc = C + gc * ldc;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t gr = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            if (gr < m) cc[gr] = acc[i][j];
        }
    }
}


}  // namespace

static mxp_status sgemm_batched(int m, int n, int k, float alpha, const float *A, int64_t lda,
                                int64_t sA, const float *B, int64_t ldb, int64_t sB, float beta,
                                float *C, int64_t ldc, int64_t sC, int batch, cudaStream_t st) {
    if (m <= 0 || n <= 0 || k <= 0 || batch <= 0) return MXP_OK;
    dim3 grid((unsigned)cdiv(m, BM), (unsigned)cdiv(n, BN), (unsigned)batch);
    sgemm_kernel<<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
    MXP_LAUNCHED();
    return MXP_OK;
}

// Triangular inverses by recursive doubling (the reference builds its
// inverse for the -alt path with STRSM on an identity,
// panel_trf_gdirect.hpp:73-92; this computes the same X with far fewer,
// wider launches):
//   level 0: every 64 x 64 diagonal block is inverted by one CTA;
//   level S: for adjacent S-blocks [A B; 0 C] (upper) the off-diagonal block
//   of the inverse is -inv(A) * B * inv(C), two batched SGEMMs per level
//   through the scratch tmp (>= n*n/4 floats).
// Upper non-unit: row i of a diagonal block's inverse satisfies x U = e_i.
__global__ void __launch_bounds__(kNB)
inv_diag_upper_kernel(int n, const float *__restrict__ U, int64_t ldu, float *__restrict__ X, int64_t ldx) {
    __shared__ float u[kNB][kNB + 1];  // u[col][row]
    const int r0 = blockIdx.x * kNB;
    const int nb = min(kNB, n - r0);
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kNB) {
        const int r = idx % kNB, c = idx / kNB;
        u[c][r] = (r < nb && c < nb) ? U[(int64_t)(r0 + c) * ldu + r0 + r] : 0.0f;
    }
    __syncthreads();
    const int i = threadIdx.x;
    if (i >= nb) return;
    float x[kNB];
#pragma unroll
    for (int j = 0; j < kNB; ++j) {
        float v = (j == i) ? 1.0f : 0.0f;
#pragma unroll
        for (int q = 0; q < j; ++q) v -= x[q] * u[j][q];
        x[j] = (j >= i && j < nb) ? v / u[j][j] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < kNB; ++j)
        if (j < nb) X[(int64_t)(r0 + j) * ldx + r0 + i] = x[j];
}

// Unit lower: row i of the inverse satisfies x L = e_i, solved from the right.
__global__ void __launch_bounds__(kNB)
inv_diag_lower_unit_kernel(int n, const float *__restrict__ L, int64_t ldl, float *__restrict__ X,
                           int64_t ldx) {
    __shared__ float l[kNB][kNB + 1];  // l[col][row]
    const int r0 = blockIdx.x * kNB;
    const int nb = min(kNB, n - r0);
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kNB) {
        const int r = idx % kNB, c = idx / kNB;
        l[c][r] = (r < nb && c < nb) ? L[(int64_t)(r0 + c) * ldl + r0 + r] : 0.0f;
    }
    __syncthreads();
    const int i = threadIdx.x;
    if (i >= nb) return;
    float x[kNB];
#pragma unroll
    for (int jj = 0; jj < kNB; ++jj) {
        const int j = kNB - 1 - jj;
        float v = (j == i) ? 1.0f : 0.0f;
#pragma unroll
        for (int q = j + 1; q < kNB; ++q) v -= x[q] * l[j][q];
        x[j] = (j <= i) ? v : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < kNB; ++j)
        if (j < nb) X[(int64_t)(r0 + j) * ldx + r0 + i] = x[j];
}

__global__ void set_zero_kernel(int n, float *X, int64_t ldx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) X[(int64_t)blockIdx.y * ldx + i] = 0.0f;
}

mxp_status launch_tri_inv_upper(int n, const float *U, int64_t ldu, float *X, int64_t ldx,
                                float *tmp, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    set_zero_kernel<<<dim3((unsigned)cdiv(n, 256), (unsigned)n), 256, 0, st>>>(n, X, ldx);
    MXP_LAUNCHED();
    inv_diag_upper_kernel<<<(unsigned)cdiv(n, kNB), kNB, 0, st>>>(n, U, ldu, X, ldx);
    MXP_LAUNCHED();
    for (int S = kNB; S < n; S *= 2) {
        const int np = n / (2 * S);
        const int rem = n - np * 2 * S;
        const int64_t step = 2 * (int64_t)S * (1 + ldx), stepU = 2 * (int64_t)S * (1 + ldu);
        const int64_t SS = (int64_t)S * S;
        // T_p = U12_p * inv(U22_p);  X12_p = -inv(U11_p) * T_p
        mxp_status s = sgemm_batched(S, S, S, 1.0f, U + (int64_t)S * ldu, ldu, stepU,
                                     X + S + (int64_t)S * ldx, ldx, step, 0.0f, tmp, S, SS, np, st);
        if (s == MXP_OK)
            s = sgemm_batched(S, S, S, -1.0f, X, ldx, step, tmp, S, SS, 0.0f, X + (int64_t)S * ldx, ldx,
                              step, np, st);
        if (s == MXP_OK && rem > S) {  // ragged last pair: C block of rem - S
            const int c = rem - S;
            const int64_t r0 = (int64_t)np * 2 * S;
            s = sgemm_batched(S, c, c, 1.0f, U + r0 + (r0 + S) * ldu, ldu, 0, X + (r0 + S) + (r0 + S) * ldx,
                              ldx, 0, 0.0f, tmp, S, 0, 1, st);
            if (s == MXP_OK)
                s = sgemm_batched(S, c, S, -1.0f, X + r0 + r0 * ldx, ldx, 0, tmp, S, 0, 0.0f,
                                  X + r0 + (r0 + S) * ldx, ldx, 0, 1, st);
        }
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

mxp_status launch_tri_inv_lower_unit(int n, const float *L, int64_t ldl, float *X, int64_t ldx,
                                     float *tmp, cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    set_zero_kernel<<<dim3((unsigned)cdiv(n, 256), (unsigned)n), 256, 0, st>>>(n, X, ldx);
    MXP_LAUNCHED();
    inv_diag_lower_unit_kernel<<<(unsigned)cdiv(n, kNB), kNB, 0, st>>>(n, L, ldl, X, ldx);
    MXP_LAUNCHED();
    for (int S = kNB; S < n; S *= 2) {
        const int np = n / (2 * S);
        const int rem = n - np * 2 * S;
        const int64_t step = 2 * (int64_t)S * (1 + ldx), stepL = 2 * (int64_t)S * (1 + ldl);
        const int64_t SS = (int64_t)S * S;
        // [A 0; B C]:  T_p = B_p * inv(A_p);  X21_p = -inv(C_p) * T_p
        mxp_status s = sgemm_batched(S, S, S, 1.0f, L + S, ldl, stepL, X, ldx, step, 0.0f, tmp, S, SS, np, st);
        if (s == MXP_OK)
            s = sgemm_batched(S, S, S, -1.0f, X + S + (int64_t)S * ldx, ldx, step, tmp, S, SS, 0.0f, X + S,
                              ldx, step, np, st);
        if (s == MXP_OK && rem > S) {
            const int c = rem - S;
            const int64_t r0 = (int64_t)np * 2 * S;
            s = sgemm_batched(c, S, S, 1.0f, L + (r0 + S) + r0 * ldl, ldl, 0, X + r0 + r0 * ldx, ldx, 0,
                              0.0f, tmp, c, 0, 1, st);
            if (s == MXP_OK)
                s = sgemm_batched(c, S, c, -1.0f, X + (r0 + S) + (r0 + S) * ldx, ldx, 0, tmp, c, 0, 0.0f,
                                  X + (r0 + S) + r0 * ldx, ldx, 0, 1, st);
        }
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

mxp_status launch_sgemm_sub(int m, int n, int k, const float *A, int64_t lda, const float *B,
                            int64_t ldb, float *C, int64_t ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0 || k <= 0) return MXP_OK;
    dim3 grid((unsigned)cdiv(m, BM), (unsigned)cdiv(n, BN));
    if (grid.y > 65535) return fail(MXP_UNSUPPORTED, "sgemm_sub: n too large");
    sgemm_kernel<<<grid, 256, 0, st>>>(m, n, k, -1.0f, A, lda, 0, B, ldb, 0, 1.0f, C, ldc, 0);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_getrf_blocked(int n, float *A, int64_t lda, DevStatus *dst, int pivot_base,
                                cudaStream_t st) {
    if (n <= 0) return MXP_OK;
    if (lda < n) return fail(MXP_INVALID_ARG, "getrf: lda < n");
    for (int jb = 0; jb < n; jb += kNB) {
        const int nbk = n - jb < kNB ? n - jb : kNB;
        float *Ajj = A + jb + (int64_t)jb * lda;
        getrf_small_kernel<<<1, kNB, 0, st>>>(nbk, Ajj, lda, dst, pivot_base + jb);
        MXP_LAUNCHED();
        const int rem = n - jb - nbk;
        if (rem <= 0) continue;
        trsm_runn_small_kernel<<<(unsigned)cdiv(rem, 128), 128, 0, st>>>(rem, nbk, Ajj, lda,
                                                                         Ajj + nbk, lda);
        MXP_LAUNCHED();
        trsm_llnu_small_kernel<<<(unsigned)cdiv(rem, 64), 256, 0, st>>>(
            rem, nbk, Ajj, lda, Ajj + (int64_t)nbk * lda, lda);
        MXP_LAUNCHED();
        mxp_status s = launch_sgemm_sub(rem, rem, nbk, Ajj + nbk, lda, Ajj + (int64_t)nbk * lda,
                                        lda, Ajj + nbk + (int64_t)nbk * lda, lda, st);
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

mxp_status launch_trsm_runn(int m, int n, const float *U, int64_t ldu, float *B, int64_t ldb,
                            cudaStream_t st) {
    if (m <= 0 || n <= 0) return MXP_OK;
    if (ldu < n || ldb < m) return fail(MXP_INVALID_ARG, "trsm_right_upper: bad leading dimension");
    for (int jb = 0; jb < n; jb += kNB) {
        const int nbk = n - jb < kNB ? n - jb : kNB;
        const float *Ujj = U + jb + (int64_t)jb * ldu;
        float *Bj = B + (int64_t)jb * ldb;
        trsm_runn_small_kernel<<<(unsigned)cdiv(m, 128), 128, 0, st>>>(m, nbk, Ujj, ldu, Bj, ldb);
        MXP_LAUNCHED();
        const int rem = n - jb - nbk;
        if (rem <= 0) continue;
        mxp_status s = launch_sgemm_sub(m, rem, nbk, Bj, ldb, Ujj + (int64_t)nbk * ldu, ldu,
                                        Bj + (int64_t)nbk * ldb, ldb, st);
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

mxp_status launch_trsm_llnu(int m, int n, const float *L, int64_t ldl, float *B, int64_t ldb,
                            cudaStream_t st) {
    if (m <= 0 || n <= 0) return MXP_OK;
    if (ldl < m || ldb < m) return fail(MXP_INVALID_ARG, "trsm_left_lower_unit: bad leading dimension");
    for (int jb = 0; jb < m; jb += kNB) {
        const int nbk = m - jb < kNB ? m - jb : kNB;
        const float *Ljj = L + jb + (int64_t)jb * ldl;
        trsm_llnu_small_kernel<<<(unsigned)cdiv(n, 64), 256, 0, st>>>(n, nbk, Ljj, ldl, B + jb, ldb);
        MXP_LAUNCHED();
        const int rem = m - jb - nbk;
        if (rem <= 0) continue;
        mxp_status s = launch_sgemm_sub(rem, n, nbk, Ljj + nbk, ldl, B + jb, ldb, B + jb + nbk,
                                        ldb, st);
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

}  // namespace mxp
