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
//              columns (thread per column, X = L_jj^{-1} B, staged through
//              shared memory), 64 per item, right-looking against D_j held in
//              shared memory, items spread over all CTAs;
//     update : trailing rank-64 update in 128 x 128 SIMT tiles.  CTA 0
//              updates only D_{j+1} (64 x 64) and factors it right away
//              (look-ahead), so the 64-step serial factor overlaps the rest of
//              the update; the CTA owning tile 0 skips that corner.
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
#include "dense_tile.cuh"
#include "mxp_internal.cuh"

namespace mxp {

namespace {

using namespace dt;

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
    extern __shared__ __align__(16) unsigned char coop_smem[];
    Smem &sm = *reinterpret_cast<Smem *>(coop_smem);
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
        const int lit = (rem + kNB - 1) / kNB, uit = (rem + kNB - 1) / kNB;  // 64-row / 64-column items
        if (cta < lit + uit) {
            load_tri(sm, nbk, Djj, lda);
            for (int it = cta; it < lit + uit; it += G) {
                if (it < lit) trsm_rows(sm, rem, nbk, Lstrip, lda, it * kNB, kNB);
                else trsm_cols64(sm, rem, nbk, Ustrip, lda, (it - lit) * kNB);
            }
        }
        if (!grid_sync(ctl, epoch, 21)) return;
        // trailing rank-nbk update.  CTA 0 updates only the next diagonal block
        // (64 x 64) and factors it at once (look-ahead); the CTA owning tile 0
        // leaves that corner alone.
        float *C = Ustrip + nbk;
        const int tm = (rem + GBM - 1) / GBM;
        const int ntiles = tm * tm;
        const int dn = min(kNB, rem);
        if (cta == 0) {
            gemm_tile64(sm, dn, dn, nbk, -1.0f, Lstrip, lda, Ustrip, lda, C, lda);
            getrf64(sm, dn, C, lda, ctl.dst, pivot_base + jb + nbk);
        }
        if (G == 1 || cta > 0) {
            const int first = G == 1 ? 0 : cta - 1, stride = G == 1 ? 1 : G - 1;
            for (int t = first; t < ntiles; t += stride)
                gemm_tile(sm, rem, rem, 0, nbk, -1.0f, Lstrip, lda, Ustrip, lda, true, C, lda,
                          (t % tm) * GBM, (t / tm) * GBN, t == 0 ? kNB : 0);
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
        cudaFuncSetAttribute(diag_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_factor_kernel, kCT, sizeof(Smem));
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
    MXP_CUDA(cudaLaunchCooperativeKernel((const void *)diag_factor_kernel, dim3(grid), dim3(kCT), args,
                                         sizeof(Smem), st));
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
