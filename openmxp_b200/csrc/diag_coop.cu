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

// Dynamic shared memory.  kStaged: the 128 x 128 update tiles are
// gemm_tile_v's (the Smem union and its two 64-deep slices share ~132 KB);
// otherwise gemm_tile's, in the ~50 KB of the Smem union.  Blocks below
// kStagedMinN have few update tiles per step, none on the step's critical
// path, and run ~2 % faster with the smaller allocation.
constexpr size_t kSmemPlain = sizeof(Smem);
constexpr size_t kSmemStaged = sizeof(Smem) > sizeof(SmemGV) ? sizeof(Smem) : sizeof(SmemGV);
constexpr int kStagedMinN = 2048;

template <bool kStaged>
__global__ void __launch_bounds__(kCT, 1)
diag_factor_kernel(int n, float *A, int64_t lda, float *XU, float *XL, int64_t ldx, float *tmpU,
                   float *tmpL, Ctl ctl, int pivot_base, int inv_stop) {
    extern __shared__ __align__(16) unsigned char coop_smem[];
    Smem &sm = *reinterpret_cast<Smem *>(coop_smem);
    SmemGV &sv = *reinterpret_cast<SmemGV *>(coop_smem);  // the same memory, for gemm_tile_v (kStaged)
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
            // the first item's operands are requested before the diagonal
            // block, so the two L2 round trips overlap
            // (a row of the L strip in x, or the U strip block in x[0..15])
            float x[kNB];
            const int it0 = cta;
            if (it0 < lit) trsm_rows_load(x, rem, nbk, Lstrip, lda, it0 * kNB, kNB);
            else load_block64(x, Ustrip + (int64_t)(it0 - lit) * kNB * lda, lda, nbk, rem - (it0 - lit) * kNB);
            load_tri(sm, nbk, Djj, lda);
            if (it0 < lit) trsm_rows_solve(sm, x, rem, nbk, Lstrip, lda, it0 * kNB, kNB);
            else trsm_cols64_loaded(sm, x, rem, nbk, Ustrip, lda, (it0 - lit) * kNB);
            for (int it = cta + G; it < lit + uit; it += G) {
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
        if (cta == 0) {  // the updated block stays in shared memory for the factor
            gemm_tile64(sm, dn, dn, nbk, -1.0f, Lstrip, lda, Ustrip, lda, C, lda, /*to_smem=*/true);
            getrf64(sm, dn, C, lda, ctl.dst, pivot_base + jb + nbk, /*in_smem=*/true);
        }
        if (G == 1 || cta > 0) {
            const int first = G == 1 ? 0 : cta - 1, stride = G == 1 ? 1 : G - 1;
            const bool vec = kStaged && gemm_tile_v_ok(Lstrip, lda, Ustrip, lda, C, lda, 0);
            for (int t = first; t < ntiles; t += stride) {
                if (vec)
                    gemm_tile_v(sv, rem, rem, 0, nbk, -1.0f, Lstrip, lda, Ustrip, lda, true, C, lda,
                                (t % tm) * GBM, (t / tm) * GBN, t == 0 ? kNB : 0);
                else
                    gemm_tile(sm, rem, rem, 0, nbk, -1.0f, Lstrip, lda, Ustrip, lda, true, C, lda,
                              (t % tm) * GBM, (t / tm) * GBN, t == 0 ? kNB : 0);
            }
        }
        if (!grid_sync(ctl, epoch, 22)) return;
    }
    if (!XU) return;

    // ---------------- triangular inverses ----------------
    auto gsync = [&](int where) { return grid_sync(ctl, epoch, where); };
    tri_inverses(sm, n, A, lda, XU, XL, ldx, tmpU, tmpL, cta, G, gsync, inv_stop, kStaged ? &sv : nullptr);
}

template <bool kStaged>
int coop_grid(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) return 0;
    if (!cached[device]) {
        const size_t smem = kStaged ? kSmemStaged : kSmemPlain;
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaFuncSetAttribute(diag_factor_kernel<kStaged>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_factor_kernel<kStaged>, kCT, smem);
        cached[device] = per_sm > 0 ? sms : -1;
    }
    return cached[device];
}

// rcp_rn_f32 against the runtime's IEEE reciprocal: sign (bit 0 of i),
// exponent 1..254 and 65536 mantissas per exponent (the extremes near 0 and
// near 0x7fffff, the rest spread by a multiplicative hash).
__global__ void check_reciprocal_kernel(unsigned long long *counts) {
    unsigned long long bad = 0, n = 0;
    const unsigned total = 2u * 254u * 65536u;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned sign = (i & 1u) << 31;
        const unsigned e = 1u + (i >> 1) % 254u;
        const unsigned q = (i >> 1) / 254u;
        const unsigned mant = q < 64 ? (q == 0 ? 0u : 0x7fffffu - (q - 1)) : (q * 2654435761u) & 0x7fffffu;
        const float x = __uint_as_float(sign | (e << 23) | mant);
        ++n;
        if (__float_as_uint(__frcp_rn(x)) != __float_as_uint(rcp_rn_f32(x))) ++bad;
    }
    atomicAdd(counts, bad);
    atomicAdd(counts + 1, n);
}

}  // namespace

extern "C" mxp_status mxp_check_reciprocal(uint64_t *h_mismatches, uint64_t *h_checked) {
    if (!h_mismatches || !h_checked) return fail(MXP_INVALID_ARG, "check_reciprocal: NULL argument");
    unsigned long long *d = nullptr;
    MXP_CUDA(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemset(d, 0, sizeof(h));
    if (e == cudaSuccess) {
        check_reciprocal_kernel<<<1184, 256>>>(d);
        e = cudaGetLastError();
        if (e == cudaSuccess) count_launch();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "check_reciprocal");
    *h_mismatches = h[0];
    *h_checked = h[1];
    return MXP_OK;
}

size_t diag_factor_tmp_floats(int n) { return (size_t)n * n / 2 + (size_t)64 * n; }

mxp_status launch_diag_factor(int n, float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                              float *tmpU, float *tmpL, unsigned int *sync_words, DevStatus *dst,
                              int pivot_base, cudaStream_t st, int max_grid, int inv_stop) {
    if (n <= 0) return MXP_OK;
    if (lda < n || (XU && ldx < n)) return fail(MXP_INVALID_ARG, "diag_factor: bad leading dimension");
    if ((XU == nullptr) != (XL == nullptr)) return fail(MXP_INVALID_ARG, "diag_factor: both inverses or none");
    if (XU && (!tmpU || !tmpL)) return fail(MXP_INVALID_ARG, "diag_factor: inverse scratch missing");
    int dev = 0;
    MXP_CUDA(cudaGetDevice(&dev));
    const bool staged = n >= kStagedMinN;
    const int sms = staged ? coop_grid<true>(dev) : coop_grid<false>(dev);
    if (sms <= 0) return fail(MXP_UNSUPPORTED, "diag_factor: kernel cannot be made resident");
    const int tm = (n + GBM - 1) / GBM;
    int grid = min(sms, max(2, tm * tm));
    if (max_grid > 0) grid = min(grid, max(2, max_grid));
    MXP_CUDA(cudaMemsetAsync(sync_words, 0, 2 * sizeof(unsigned int), st));
    Ctl ctl{sync_words, reinterpret_cast<int *>(sync_words + 1), dst};
    void *args[] = {&n, &A, &lda, &XU, &XL, &ldx, &tmpU, &tmpL, &ctl, &pivot_base, &inv_stop};
    if (staged)
        MXP_CUDA(cudaLaunchCooperativeKernel((const void *)diag_factor_kernel<true>, dim3(grid), dim3(kCT), args,
                                             kSmemStaged, st));
    else
        MXP_CUDA(cudaLaunchCooperativeKernel((const void *)diag_factor_kernel<false>, dim3(grid), dim3(kCT), args,
                                             kSmemPlain, st));
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
