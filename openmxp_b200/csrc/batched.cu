// Batched solve: many independent systems of uneven orders factored (FP32
// panels, FP16 Schur update on tcgen05 with FP32 accumulation) and refined in
// FP64 in ONE persistent launch.
//
// The reference solves one system per job (main.cpp:617-657); this is the
// batched form of that path.  Design:
//  * one CTA (256 threads) per SM, each taking whole systems from a ticket in
//    descending order of size (longest first), so a CTA runs one system's
//    LU and refinement start to finish with no grid-wide synchronisation;
//  * per block step of B columns: the B x B diagonal block and the two panel
//    strips are factored with the SIMT FP32 pieces of dense_tile.cuh (same
//    algorithm as the single-system path: no-pivot LU, TRSM against the
//    diagonal triangles, sgetrf_nopiv_naive order); the strips are then cast
//    to FP16 into a per-CTA staging area laid out as the shared-memory image
//    of a 128-byte-swizzled K-major tile (16 KB per 128 rows x 64 columns), so
//    the Schur phase moves each operand tile with one plain bulk copy
//    (cp.async.bulk, no tensor map) into a ring of shared-memory stages;
//  * the trailing update C -= L R^T runs warp-specialised on the CTA's own
//    tensor core: warp 0 issues the bulk copies, warp 1 the tcgen05.mma
//    (M = 128, N = TN, K = 16) into one of two TMEM accumulators, warps 4-7
//    drain the accumulator and apply it to C in HBM;
//  * refinement follows iterative_refinement.hpp:141-171 per system: x0 = b/d,
//    r = b - A x with A regenerated in FP64 from the LCG (otf_gemv), stop at
//    scaled residual < 16, else x += U^{-1} L^{-1} r (block substitution with
//    r in shared memory).
// Every wait is bounded; a timeout records MXP_TIMEOUT, stops all roles, frees
// TMEM and returns.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "dense_tile.cuh"
#include "mxp_internal.cuh"
#include "tc_ptx.cuh"

namespace mxp {

namespace {

using namespace dt;
using namespace tc;

constexpr int kBatchThreads = 256;
static_assert(kBatchThreads == kCT, "the SIMT pieces assume kCT threads");
constexpr int kSliceK = 64;                  // K per smem stage (one 128-byte swizzle atom of FP16)
constexpr int kRowTile = 128;                // MMA M
constexpr uint32_t kBlockBytes = 16384;      // 128 rows x 64 FP16, swizzled
constexpr int kMaxStages = 4;

struct BatchSys {
    int n;          // order (multiple of 128)
    int pad;
    uint64_t seed;  // generator seed
    int64_t a_off;  // first element of the matrix in the packed FP32 array
    int64_t v_off;  // first element of the vectors in the packed FP64 arrays
};

struct BatchOut {
    int iterations;  // refinement steps taken
    int converged;   // 1 when the scaled residual went below 16
    int info;        // first zero pivot (1-based) or 0
    int pad;
    double hpl;      // final scaled residual
    double resid;    // final ||b - A x||_inf
};

struct BatchArgs {
    const BatchSys *sys;
    const int *order;      // ticket -> system index (descending n)
    int count;
    int b;                 // block size (multiple of 64, <= 256)
    int stages;            // smem ring depth
    int maxit;
    float *A;
    const double *d;
    const double *rhs;
    double *x;
    BatchOut *out;
    uint8_t *staging;      // per-CTA FP16 operand staging
    int64_t staging_stride;  // bytes per CTA
    int64_t rstage_off;    // offset of the R staging inside a CTA's area
    unsigned int *ticket;
    DevStatus *dst;
};

// Byte offset of FP16 element (r, k) of a 128-row block in the 128-byte
// swizzled K-major layout (8-row groups of 1024 bytes; the 16-byte chunk
// index is XOR-ed with the row within the group).
__device__ __forceinline__ uint32_t sw128_offset(int r, int chunk) {
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((chunk ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// Cast one operand row (bk values, v(k) for k in [0, bk)) into the staging area:
// slice s = k / 64 of row-block rt lives at base + (s * nblk + rt) * 16 KB.
template <typename Get>
__device__ __forceinline__ void stage_row(uint8_t *base, int nblk, int row, int bk, Get v) {
    const int rt = row >> 7, r = row & 127;
    for (int s = 0; s < bk / kSliceK; ++s) {
        uint8_t *blk = base + ((int64_t)s * nblk + rt) * kBlockBytes;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int k = s * kSliceK + c * 8;
            uint4 q;
            q.x = pack_h2(v(k + 0), v(k + 1));
            q.y = pack_h2(v(k + 2), v(k + 3));
            q.z = pack_h2(v(k + 4), v(k + 5));
            q.w = pack_h2(v(k + 6), v(k + 7));
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r, c)) = q;
        }
    }
}

// The same for a row whose bk values are contiguous and 16-byte aligned in
// memory (a column of the U strip, i.e. a row of R = U^T): eight values per
// chunk as two 16-byte loads (a whole 32-byte sector per thread; the scalar
// form read 4 bytes of a sector per load across 32 columns per warp).
__device__ __forceinline__ void stage_row_contig(uint8_t *base, int nblk, int row, int bk, const float *src) {
    const int rt = row >> 7, r = row & 127;
    for (int s = 0; s < bk / kSliceK; ++s) {
        uint8_t *blk = base + ((int64_t)s * nblk + rt) * kBlockBytes;
        float4 lo[8], hi[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 *p4 = reinterpret_cast<const float4 *>(src + s * kSliceK + c * 8);
            lo[c] = __ldcg(p4);
            hi[c] = __ldcg(p4 + 1);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            uint4 q;
            q.x = pack_h2(lo[c].x, lo[c].y);
            q.y = pack_h2(lo[c].z, lo[c].w);
            q.z = pack_h2(hi[c].x, hi[c].y);
            q.w = pack_h2(hi[c].z, hi[c].w);
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r, c)) = q;
        }
    }
}

// Four consecutive rows r4 .. r4 + 3 of a column-major panel (row i, value k at
// src[(i - r4) + k * ld], src 16-byte aligned, ld % 4 == 0): each k read as one
// 16-byte load of the four rows (a warp covers 128 consecutive rows, 512
// contiguous bytes), instead of a 4-byte load per row.  Not inlined (the
// persistent kernel around it is at the register limit).
__device__ __noinline__ void stage_rows4(uint8_t *base, int nblk, int r4, int bk, const float *src, int64_t ld) {
    const int rt = r4 >> 7, r = r4 & 127;
    for (int s = 0; s < bk / kSliceK; ++s) {
        uint8_t *blk = base + ((int64_t)s * nblk + rt) * kBlockBytes;
#pragma unroll 2
        for (int c = 0; c < 8; ++c) {
            const int k = s * kSliceK + c * 8;
            float4 v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) v[e] = __ldcg(reinterpret_cast<const float4 *>(src + (int64_t)(k + e) * ld));
            uint4 q0, q1, q2, q3;
            q0.x = pack_h2(v[0].x, v[1].x); q0.y = pack_h2(v[2].x, v[3].x); q0.z = pack_h2(v[4].x, v[5].x); q0.w = pack_h2(v[6].x, v[7].x);
            q1.x = pack_h2(v[0].y, v[1].y); q1.y = pack_h2(v[2].y, v[3].y); q1.z = pack_h2(v[4].y, v[5].y); q1.w = pack_h2(v[6].y, v[7].y);
            q2.x = pack_h2(v[0].z, v[1].z); q2.y = pack_h2(v[2].z, v[3].z); q2.z = pack_h2(v[4].z, v[5].z); q2.w = pack_h2(v[6].z, v[7].z);
            q3.x = pack_h2(v[0].w, v[1].w); q3.y = pack_h2(v[2].w, v[3].w); q3.z = pack_h2(v[4].w, v[5].w); q3.w = pack_h2(v[6].w, v[7].w);
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r + 0, c)) = q0;
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r + 1, c)) = q1;
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r + 2, c)) = q2;
            *reinterpret_cast<uint4 *>(blk + sw128_offset(r + 3, c)) = q3;
        }
    }
}

__device__ __forceinline__ void stage_zero_row(uint8_t *base, int nblk, int row, int bk) {
    const int rt = row >> 7, r = row & 127;
    for (int s = 0; s < bk / kSliceK; ++s) {
        uint8_t *blk = base + ((int64_t)s * nblk + rt) * kBlockBytes;
#pragma unroll
        for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4 *>(blk + sw128_offset(r, c)) = make_uint4(0, 0, 0, 0);
    }
}

// U-strip columns [c0, c0 + 256) of B (nb x ncols): X = L^{-1} B with L the unit
// lower part of the diagonal block (load_tri).  The 64 x 256 block goes
// through shared memory (stage: 256 x 65 floats) with coalesced 16-byte loads
// and stores, all of a thread's loads in flight at once; thread j solves
// column j.  Not inlined: the persistent kernel around it is at the register
// limit, and the sixteen loads in flight spilled there.
constexpr size_t kColStageOff = 65536;  // after the Smem union
constexpr size_t kColStageBytes = sizeof(float) * kCT * (kNB + 1);

__device__ __noinline__ void trsm_cols_staged(Smem &sm, float *stage, int ncols, int nb, float *B, int64_t ldb,
                                              int c0) {
    // 16-byte loads, all sixteen of a thread in flight at once, when the
    // columns allow them (nb = 64, B and ldb 16-byte aligned)
    const bool vec = nb == kNB && ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb & 3) == 0;
    if (vec) {
        float4 v[kNB * kCT / 4 / kCT];
#pragma unroll
        for (int q = 0; q < kNB * kCT / 4 / kCT; ++q) {
            const int idx = threadIdx.x + kCT * q;
            const int k4 = idx % (kNB / 4), j = idx / (kNB / 4);
            v[q] = c0 + j < ncols ? __ldcg(reinterpret_cast<const float4 *>(B + (int64_t)(c0 + j) * ldb) + k4)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < kNB * kCT / 4 / kCT; ++q) {
            const int idx = threadIdx.x + kCT * q;
            const int k4 = idx % (kNB / 4), j = idx / (kNB / 4);
            float *st = stage + j * (kNB + 1) + 4 * k4;
            st[0] = v[q].x;
            st[1] = v[q].y;
            st[2] = v[q].z;
            st[3] = v[q].w;
        }
    } else {
#pragma unroll 16
        for (int idx = threadIdx.x; idx < kNB * kCT; idx += kCT) {
            const int k = idx % kNB, j = idx / kNB;
            stage[j * (kNB + 1) + k] = (k < nb && c0 + j < ncols) ? __ldcg(B + (int64_t)(c0 + j) * ldb + k) : 0.0f;
        }
    }
    __syncthreads();
    {  // right-looking: x_r -= l_rk x_k for r > k, rotated (trsm_col)
        const int j = threadIdx.x;
        float x[kNB];
#pragma unroll
        for (int k = 0; k < kNB; ++k) x[k] = stage[j * (kNB + 1) + k];
        trsm_col(sm, x, nb, stage + j * (kNB + 1));
    }
    __syncthreads();
    if (vec) {
#pragma unroll
        for (int q = 0; q < kNB * kCT / 4 / kCT; ++q) {
            const int idx = threadIdx.x + kCT * q;
            const int k4 = idx % (kNB / 4), j = idx / (kNB / 4);
            if (c0 + j < ncols) {
                const float *st = stage + j * (kNB + 1) + 4 * k4;
                reinterpret_cast<float4 *>(B + (int64_t)(c0 + j) * ldb)[k4] = make_float4(st[0], st[1], st[2], st[3]);
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < kNB * kCT; idx += kCT) {
            const int k = idx % kNB, j = idx / kNB;
            if (k < nb && c0 + j < ncols) B[(int64_t)(c0 + j) * ldb + k] = stage[j * (kNB + 1) + k];
        }
    }
    __syncthreads();
}

// one accumulating rank-64 tile of the panel (its own register allocation: the
// persistent kernel around it is at the register limit); MI / NJ = 4 for the
// 64-row / 64-column remainders of the strips, whose padding half is skipped
template <int MI, int NJ>
__device__ __noinline__ void panel_tile_v(SmemGV &sv, int m, int n, const float *A, const float *B, float *C,
                                          int64_t ld, int m0, int n0) {
    gemm_tile_v<MI, NJ>(sv, m, n, 0, kNB, -1.0f, A, ld, B, ld, true, C, ld, m0, n0);
}

// ---- panel factorisation of one block step (SIMT FP32, whole CTA) -----------
// D = A(k0, k0) (bk x bk), L strip = A(k0+bk.., k0..) (m x bk), U strip =
// A(k0.., k0+bk..) (bk x m); lda = n.
__device__ void factor_step(Smem &sm, float *stage, float *A, int n, int k0, int bk, DevStatus *dst) {
    const int64_t lda = n;
    // the rank-64 updates as cp.async-staged tiles when the system allows
    // 16-byte copies (its base 16-byte aligned, n a multiple of 4)
    SmemGV &sv = *reinterpret_cast<SmemGV *>(&sm);
    const bool vec = gemm_tile_v_ok(A, lda, A, lda, A, lda, 0);
    auto tile = [&](int tm_, int tn_, const float *Ap, const float *Bp, float *Cp, int m0, int n0) {
        if (vec) {
            const bool hm = tm_ - m0 <= kNB, hn = tn_ - n0 <= kNB;
            if (hm && hn) panel_tile_v<4, 4>(sv, tm_, tn_, Ap, Bp, Cp, lda, m0, n0);
            else if (hm) panel_tile_v<4, 8>(sv, tm_, tn_, Ap, Bp, Cp, lda, m0, n0);
            else if (hn) panel_tile_v<8, 4>(sv, tm_, tn_, Ap, Bp, Cp, lda, m0, n0);
            else panel_tile_v<8, 8>(sv, tm_, tn_, Ap, Bp, Cp, lda, m0, n0);
        }
        else gemm_tile(sm, tm_, tn_, 0, kNB, -1.0f, Ap, lda, Bp, lda, true, Cp, lda, m0, n0);
    };
    float *D = A + k0 + (int64_t)k0 * lda;
    const int m = n - k0 - bk;
    // diagonal block: blocked by 64, whole CTA
    for (int jb = 0; jb < bk; jb += kNB) {
        float *Dj = D + jb + (int64_t)jb * lda;
        getrf64(sm, kNB, Dj, lda, dst, k0 + jb);
        const int rem = bk - jb - kNB;
        if (rem <= 0) break;
        load_tri(sm, kNB, Dj, lda);
        for (int r0 = 0; r0 < rem; r0 += kCT) trsm_rows(sm, rem, kNB, Dj + kNB, lda, r0);
        for (int c0 = 0; c0 < rem; c0 += kCT) trsm_cols_staged(sm, stage, rem, kNB, Dj + (int64_t)kNB * lda, lda, c0);
        __syncthreads();
        const int tm = (rem + GBM - 1) / GBM;
        for (int t = 0; t < tm * tm; ++t)
            tile(rem, rem, Dj + kNB, Dj + (int64_t)kNB * lda, Dj + kNB + (int64_t)kNB * lda, (t % tm) * GBM,
                 (t / tm) * GBN);
    }
    if (m <= 0) return;
    float *Ls = D + bk;                     // m x bk
    float *Us = D + (int64_t)bk * lda;      // bk x m
    // L strip: X U = B, one 64-column block at a time
    for (int c = 0; c < bk; c += kNB) {
        load_tri(sm, kNB, D + c + (int64_t)c * lda, lda);
        for (int r0 = 0; r0 < m; r0 += kCT) trsm_rows(sm, m, kNB, Ls + (int64_t)c * lda, lda, r0);
        __syncthreads();
        const int rest = bk - c - kNB;
        if (rest > 0) {
            const int tm = (m + GBM - 1) / GBM, tn = (rest + GBN - 1) / GBN;
            for (int t = 0; t < tm * tn; ++t)
                tile(m, rest, Ls + (int64_t)c * lda, D + c + (int64_t)(c + kNB) * lda, Ls + (int64_t)(c + kNB) * lda,
                     (t % tm) * GBM, (t / tm) * GBN);
        }
    }
    // U strip: L X = B, one 64-row block at a time, one group of 256 columns
    // after another.  Its columns are independent, so every element receives
    // the same operations in the same order as with the row blocks outermost;
    // but a column's 64-row slices (256 bytes each) are then read while the
    // group is still in L2, instead of four passes over the whole strip from
    // DRAM (2048 systems of orders 256..4096: U strip 163 -> 135 ms per CTA;
    // the diagonal triangle reloaded per group costs little).
    for (int g0 = 0; g0 < m; g0 += kCT) {
        const int ge = min(m, g0 + kCT);
        for (int c = 0; c < bk; c += kNB) {
            load_tri(sm, kNB, D + c + (int64_t)c * lda, lda);
            trsm_cols_staged(sm, stage, m, kNB, Us + c, lda, g0);
            __syncthreads();
            const int rest = bk - c - kNB;
            if (rest > 0) {
                const int tm = (rest + GBM - 1) / GBM, tn = (ge - g0 + GBN - 1) / GBN;
                for (int t = 0; t < tm * tn; ++t)
                    tile(rest, ge, D + c + kNB + (int64_t)c * lda, Us + c, Us + c + kNB, (t % tm) * GBM,
                         g0 + (t / tm) * GBN);
            }
        }
    }
}

// ---- tcgen05 trailing update of one block step --------------------------------
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

struct Ring {
    float *cbuf;            // epilogue staging of C: 128 columns x 128 rows
    uint8_t *sA;            // stages x 16 KB
    uint8_t *sB;            // stages x TN x 128 B
    uint64_t *full, *empty; // per stage
    uint64_t *tfull, *tempty;  // per accumulator
    uint32_t tmem;
    int stages;
};

// Barrier positions carried across steps and systems (each role owns its own).
struct RoleState {
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
};

template <int TN>
__device__ bool schur_step(const Ring &rg, RoleState &rs, volatile int *abort_flag, float *C, int64_t ldc,
                           int m, int bk, const uint8_t *Lst, int nblkL, const uint8_t *Rst, int nblkR,
                           DevStatus *dst) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_m = (m + kRowTile - 1) / kRowTile, tiles_n = (m + TN - 1) / TN;
    const int ntiles = tiles_m * tiles_n;
    const int nslice = bk / kSliceK;
    constexpr uint32_t kBBytes = (uint32_t)TN * 128;
    bool ok = true;
    if (warp == 0) {
        if (lane == 0) {  // ---- bulk-copy producer ----
            for (int t = 0; t < ntiles && ok; ++t) {
                const int rt = t / tiles_n, ct = t % tiles_n;
                for (int s = 0; s < nslice; ++s) {
                    if (!mbar_wait(smem_u32(&rg.empty[rs.stage]), rs.phase ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&rg.full[rs.stage]);
                    mbar_expect_tx(fb, kBlockBytes + kBBytes);
                    bulk_copy_g2s(smem_u32(rg.sA + (size_t)rs.stage * kBlockBytes),
                                  Lst + ((int64_t)s * nblkL + rt) * kBlockBytes, kBlockBytes, fb);
                    bulk_copy_g2s(smem_u32(rg.sB + (size_t)rs.stage * kBBytes),
                                  Rst + ((int64_t)s * nblkR + (int64_t)ct * (TN / 128)) * kBlockBytes, kBBytes, fb);
                    if (++rs.stage == rg.stages) {
                        rs.stage = 0;
                        rs.phase ^= 1u;
                    }
                }
            }
            if (!ok) report(dst, MXP_TIMEOUT, 31, blockIdx.x);
        }
    } else if (warp == 1) {
        if (lane == 0) {  // ---- MMA issuer ----
            constexpr uint32_t idesc = idesc_f16_mn(0u, kRowTile, TN);
            for (int t = 0; t < ntiles && ok; ++t) {
                if (!mbar_wait(smem_u32(&rg.tempty[rs.acc]), rs.acc_phase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = rg.tmem + (uint32_t)(rs.acc * TN);
                for (int s = 0; s < nslice; ++s) {
                    if (!mbar_wait(smem_u32(&rg.full[rs.stage]), rs.phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(rg.sA + (size_t)rs.stage * kBlockBytes);
                    const uint32_t b0 = smem_u32(rg.sB + (size_t)rs.stage * kBBytes);
#pragma unroll
                    for (int k = 0; k < kSliceK / 16; ++k)
                        tc_mma_f16(d_tmem, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k), idesc,
                                   (s > 0 || k > 0) ? 1u : 0u);
                    tc_commit(smem_u32(&rg.empty[rs.stage]));
                    if (++rs.stage == rg.stages) {
                        rs.stage = 0;
                        rs.phase ^= 1u;
                    }
                }
                if (!ok) break;
                tc_commit(smem_u32(&rg.tfull[rs.acc]));
                if (++rs.acc == 2) {
                    rs.acc = 0;
                    rs.acc_phase ^= 1u;
                }
            }
            if (!ok) report(dst, MXP_TIMEOUT, 32, blockIdx.x);
        }
    } else if (warp >= 4) {  // ---- epilogue: TMEM lane quarter = warp % 4 ----
        const int quarter = warp & 3;
        for (int t = 0; t < ntiles && ok; ++t) {
            const int rt = t / tiles_n, ct = t % tiles_n;
            if (!mbar_wait(smem_u32(&rg.tfull[rs.acc]), rs.acc_phase, abort_flag)) {
                ok = false;
                break;
            }
            __syncwarp();
            tc_fence_after();
            const int r = quarter * 32 + lane;  // row within the tile
            const int row = rt * kRowTile + r;
            const uint32_t tbase = rg.tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(rs.acc * TN);
#pragma unroll 1
            for (int h = 0; h < TN / 128; ++h) {
                // C for 128 columns of this row -> shared memory with async copies (the
                // bytes in flight are not bounded by registers), then subtract the
                // accumulator column by column and store
                const int colh = ct * TN + h * 128;
                if (row < m) {
                    const float *cp = C + (int64_t)colh * ldc + row;
#pragma unroll 8
                    for (int j = 0; j < 128; ++j)
                        if (colh + j < m)
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(rg.cbuf + j * 128 + r)),
                                         "l"(cp + (int64_t)j * ldc)
                                         : "memory");
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
                asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll 1
                for (int c = 0; c < 4; ++c) {
                    uint32_t v[32];
                    tmem_ld_32x32b_x32(tbase + h * 128 + c * 32, v);
                    if (h == TN / 128 - 1 && c == 3) {  // accumulator drained: the next tile may use it
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(smem_u32(&rg.tempty[rs.acc]));
                    }
                    if (row < m) {
                        float *cp = C + (int64_t)(colh + c * 32) * ldc + row;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (colh + c * 32 + j < m)
                                __stcs(cp + (int64_t)j * ldc, rg.cbuf[(c * 32 + j) * 128 + r] - __uint_as_float(v[j]));
                    }
                }
            }
            if (++rs.acc == 2) {
                rs.acc = 0;
                rs.acc_phase ^= 1u;
            }
        }
        if (!ok && lane == 0) report(dst, MXP_TIMEOUT, 33, blockIdx.x);
    }
    if (!ok) *abort_flag = 1;
    __syncthreads();
    return *abort_flag == 0;
}

// ---- per-system refinement (whole CTA) -----------------------------------------
__device__ double block_max(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = red[0];
#pragma unroll
    for (int w = 1; w < kBatchThreads / 32; ++w) m = fmax(m, red[w]);
    return m;
}

// r = b - A x with a_ij regenerated in FP64 from the LCG (otf_gemv,
// panel_gemv.hpp:13-81) and the diagonal taken from d; x and r in shared memory.
// Rows are processed two per thread; the sum over j runs in increasing j.
__device__ void otf_residual(int n, uint64_t seed, const double *__restrict__ d, const double *__restrict__ b,
                             const double *xs, double *rs) {
    const uint64_t s00 = lcg_stat00(seed);
    const Aff inc1 = lcg_inc1();
    const Aff jn = aff_pow(inc1, (uint64_t)n);
    const Aff step2 = aff_pow(inc1, (uint64_t)kBatchThreads);
    constexpr double kScale = 0x1.fffffffffffffP-65;
    for (int i0 = threadIdx.x; i0 < n; i0 += 2 * kBatchThreads) {
        const int i1 = i0 + kBatchThreads;
        uint64_t s0 = aff_apply(aff_pow(inc1, (uint64_t)i0), s00);  // element (i0, 0)
        uint64_t s1 = aff_apply(step2, s0);                          // element (i1, 0)
        double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
            const double xj = xs[j];
            double v0 = i64_to_double_rn(s0) * kScale;
            double v1 = i64_to_double_rn(s1) * kScale;
            v0 = (j == i0) ? 0.0 : v0;
            v1 = (j == i1) ? 0.0 : v1;
            acc0 = __fma_rn(v0, xj, acc0);
            acc1 = __fma_rn(v1, xj, acc1);
            s0 = aff_apply(jn, s0);
            s1 = aff_apply(jn, s1);
        }
        rs[i0] = b[i0] - (acc0 + d[i0] * xs[i0]);
        if (i1 < n) rs[i1] = b[i1] - (acc1 + d[i1] * xs[i1]);
    }
    __syncthreads();
}

// r <- U^{-1} L^{-1} r with the FP32 factors (lda = n) and r in shared memory:
// 64-row blocks, the diagonal block solved in FP64 by one warp, the block's
// column panel applied to the remaining rows by all threads (the block
// substitution of panel_trsv.hpp:601-747).
// r[i] -= sum_k LU(i, c0 + k) r[c0 + k] (k = 0..63, in order) for the rows i in
// [i_begin, i_end): a thread takes four consecutive rows and reads the block
// column with 16-byte loads (sixteen in flight), instead of one row at a time
// with 4-byte loads; each row's sum is the same.  Its own register allocation
// (the persistent kernel around it is at the register limit).
__device__ __noinline__ void block_column_update(const float *__restrict__ LU, int64_t lda, int c0, double *r,
                                                 int i_begin, int i_end) {
    const bool vec = ((reinterpret_cast<uintptr_t>(LU) & 15) == 0) && (lda & 3) == 0 && (i_begin & 3) == 0;
    if (vec) {
        for (int i = i_begin + 4 * threadIdx.x; i < i_end; i += 4 * kBatchThreads) {
            if (i + 4 <= i_end) {
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll 16
                for (int k = 0; k < kNB; ++k) {
                    const float4 v = __ldg(reinterpret_cast<const float4 *>(LU + (int64_t)(c0 + k) * lda + i));
                    const double rk = r[c0 + k];
                    a0 = __fma_rn((double)v.x, rk, a0);
                    a1 = __fma_rn((double)v.y, rk, a1);
                    a2 = __fma_rn((double)v.z, rk, a2);
                    a3 = __fma_rn((double)v.w, rk, a3);
                }
                r[i] -= a0;
                r[i + 1] -= a1;
                r[i + 2] -= a2;
                r[i + 3] -= a3;
            } else {
                for (int e = i; e < i_end; ++e) {
                    double acc = 0.0;
                    for (int k = 0; k < kNB; ++k) acc = __fma_rn((double)__ldg(LU + (int64_t)(c0 + k) * lda + e), r[c0 + k], acc);
                    r[e] -= acc;
                }
            }
        }
    } else {
        for (int i = i_begin + threadIdx.x; i < i_end; i += kBatchThreads) {
            double acc = 0.0;
#pragma unroll 16
            for (int k = 0; k < kNB; ++k) acc = __fma_rn((double)__ldg(LU + (int64_t)(c0 + k) * lda + i), r[c0 + k], acc);
            r[i] -= acc;
        }
    }
}

__device__ void lu_solve_shared(int n, const float *__restrict__ LU, double *r, float (*tri)[kNB + 1]) {
    const int64_t lda = n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nb = n / kNB;
    auto load_diag = [&](int c0) {  // tri[col][row] of the 64 x 64 diagonal block, coalesced
        for (int idx = threadIdx.x; idx < kNB * kNB; idx += kBatchThreads) {
            const int rr = idx % kNB, cc = idx / kNB;
            tri[cc][rr] = LU[(int64_t)(c0 + cc) * lda + c0 + rr];
        }
        __syncthreads();
    };
    for (int blk = 0; blk < nb; ++blk) {  // forward, unit lower
        const int c0 = blk * kNB;
        load_diag(c0);
        if (warp == 0) {
            double z0 = r[c0 + lane], z1 = r[c0 + 32 + lane];
            for (int k = 0; k < kNB; ++k) {
                const double zk = __shfl_sync(0xffffffffu, k < 32 ? z0 : z1, k & 31);
                if (lane > k) z0 -= (double)tri[k][lane] * zk;
                if (lane + 32 > k) z1 -= (double)tri[k][lane + 32] * zk;
            }
            r[c0 + lane] = z0;
            r[c0 + 32 + lane] = z1;
        }
        __syncthreads();
        block_column_update(LU, lda, c0, r, c0 + kNB, n);
        __syncthreads();
    }
    for (int blk = nb - 1; blk >= 0; --blk) {  // backward, upper non-unit
        const int c0 = blk * kNB;
        load_diag(c0);
        if (warp == 0) {
            double z0 = r[c0 + lane], z1 = r[c0 + 32 + lane];
            for (int k = kNB - 1; k >= 0; --k) {
                const double rdk = 1.0 / (double)tri[k][k];
                if (k < 32) {
                    if (lane == k) z0 = z0 * rdk;
                } else if (lane + 32 == k) {
                    z1 = z1 * rdk;
                }
                const double zk = __shfl_sync(0xffffffffu, k < 32 ? z0 : z1, k & 31);
                if (lane < k) z0 -= (double)tri[k][lane] * zk;
                if (lane + 32 < k) z1 -= (double)tri[k][lane + 32] * zk;
            }
            r[c0 + lane] = z0;
            r[c0 + 32 + lane] = z1;
        }
        __syncthreads();
        block_column_update(LU, lda, c0, r, 0, c0);
        __syncthreads();
    }
}

// Classic refinement of iterative_refinement.hpp:141-171 for one system whose
// factors are in A; returns the number of corrections applied.
__device__ void refine_system(int n, uint64_t seed, const float *A, const double *d, const double *b, double *x,
                              int maxit, double *xs, double *rs, double *red, float (*tri)[kNB + 1], BatchOut *out) {
    double mb = 0.0, md = 0.0;
    for (int i = threadIdx.x; i < n; i += kBatchThreads) {
        mb = fmax(mb, fabs(b[i]));
        md = fmax(md, d[i]);
        xs[i] = b[i] / d[i];
    }
    const double normb = block_max(mb, red);
    const double norma = 2.0 * block_max(md, red);  // hpl_infnorm(d), panel_norm.hpp:129-135
    const double eps = 0x1p-53;
    int it = 0;
    bool conv = false;
    double hpl = -1.0, normr = -1.0;
    for (it = 0; it < maxit; ++it) {
        otf_residual(n, seed, d, b, xs, rs);
        double mr = 0.0, mx = 0.0;
        for (int i = threadIdx.x; i < n; i += kBatchThreads) {
            mr = fmax(mr, fabs(rs[i]));
            mx = fmax(mx, fabs(xs[i]));
        }
        normr = block_max(mr, red);
        const double normx = block_max(mx, red);
        hpl = normr / (norma * normx + normb) * 1.0 / ((double)n * eps);
        if (!(hpl < 16.0) && isfinite(hpl)) {
            lu_solve_shared(n, A, rs, tri);
            for (int i = threadIdx.x; i < n; i += kBatchThreads) xs[i] += rs[i];
            __syncthreads();
            continue;
        }
        conv = hpl < 16.0;
        break;
    }
    for (int i = threadIdx.x; i < n; i += kBatchThreads) x[i] = xs[i];
    if (threadIdx.x == 0) {
        out->iterations = it;
        out->converged = conv ? 1 : 0;
        out->hpl = hpl;
        out->resid = normr;
    }
    __syncthreads();
}

// ---- the persistent kernel ------------------------------------------------------
struct BatchKernelArgs {
    BatchArgs a;
    DevStatus *sys_status;  // per system (zero pivots)
};

template <int TN>
__global__ void __launch_bounds__(kBatchThreads, 1) batched_kernel(BatchKernelArgs ka) {
    const BatchArgs &a = ka.a;
    extern __shared__ uint8_t batch_smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(batch_smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t bar_full[kMaxStages], bar_empty[kMaxStages], bar_tfull[2], bar_tempty[2];
    __shared__ uint32_t tmem_holder;
    __shared__ int abort_flag;
    __shared__ int s_ticket;
    __shared__ double red[kBatchThreads / 32];
    constexpr uint32_t kTmemCols = 2 * TN;
    const int warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < a.stages; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int c = 0; c < 2; ++c) {
            mbar_init(smem_u32(&bar_tfull[c]), 1);
            mbar_init(smem_u32(&bar_tempty[c]), 4);  // the four epilogue warps
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    Ring rg;
    rg.sA = smem;
    rg.sB = smem + (size_t)a.stages * kBlockBytes;
    rg.cbuf = reinterpret_cast<float *>(rg.sB + (size_t)a.stages * TN * 128);
    rg.full = bar_full;
    rg.empty = bar_empty;
    rg.tfull = bar_tfull;
    rg.tempty = bar_tempty;
    rg.tmem = tmem_holder;
    rg.stages = a.stages;
    RoleState rs;
    Smem &sm = *reinterpret_cast<Smem *>(smem);  // SIMT phases reuse the ring's memory
    float *colstage = reinterpret_cast<float *>(smem + kColStageOff);
    static_assert(sizeof(Smem) <= kColStageOff, "column stage overlaps the SIMT scratch");
    uint8_t *Lst = a.staging + (int64_t)blockIdx.x * a.staging_stride;
    uint8_t *Rst = Lst + a.rstage_off;

    while (true) {
        if (threadIdx.x == 0) s_ticket = (int)atomicAdd(a.ticket, 1u);
        __syncthreads();
        const int tk = s_ticket;
        if (tk >= a.count || abort_flag) break;
        const int si = a.order[tk];
        const BatchSys S = a.sys[si];
        const int n = S.n;
        float *A = a.A + S.a_off;
        const int64_t lda = n;
        DevStatus *sst = ka.sys_status + si;
        // ---------------- LU ----------------
        for (int k0 = 0; k0 < n && !abort_flag; k0 += a.b) {
            const int bk = min(a.b, n - k0);
            factor_step(sm, colstage, A, n, k0, bk, sst);
            const int m = n - k0 - bk;
            if (m <= 0) break;
            const int mp = (m + kRowTile - 1) / kRowTile * kRowTile;
            const int np = (m + TN - 1) / TN * TN;
            const float *Ls = A + (k0 + bk) + (int64_t)k0 * lda;
            const float *Us = A + k0 + (int64_t)(k0 + bk) * lda;
            const bool lvec = ((reinterpret_cast<uintptr_t>(Ls) & 15) == 0) && (lda & 3) == 0;
            if (lvec) {
                for (int r4 = 4 * threadIdx.x; r4 < mp; r4 += 4 * kBatchThreads) {
                    if (r4 + 4 <= m) {
                        stage_rows4(Lst, mp / 128, r4, bk, Ls + r4, lda);
                    } else {
                        for (int row = r4; row < r4 + 4 && row < mp; ++row) {
                            if (row < m)
                                stage_row(Lst, mp / 128, row, bk,
                                          [&](int k) { return __ldcg(Ls + row + (int64_t)k * lda); });
                            else
                                stage_zero_row(Lst, mp / 128, row, bk);
                        }
                    }
                }
            } else {
                for (int row = threadIdx.x; row < mp; row += kBatchThreads) {
                    if (row < m)
                        stage_row(Lst, mp / 128, row, bk, [&](int k) { return __ldcg(Ls + row + (int64_t)k * lda); });
                    else
                        stage_zero_row(Lst, mp / 128, row, bk);
                }
            }
            const bool rvec = ((reinterpret_cast<uintptr_t>(Us) & 15) == 0) && (lda & 3) == 0;
            for (int j = threadIdx.x; j < np; j += kBatchThreads) {
                if (j < m && rvec)
                    stage_row_contig(Rst, np / 128, j, bk, Us + (int64_t)j * lda);
                else if (j < m)
                    stage_row(Rst, np / 128, j, bk, [&](int k) { return __ldcg(Us + k + (int64_t)j * lda); });
                else
                    stage_zero_row(Rst, np / 128, j, bk);
            }
            asm volatile("fence.proxy.async.global;" ::: "memory");  // staging -> bulk copies
            __syncthreads();
            schur_step<TN>(rg, rs, &abort_flag, A + (k0 + bk) + (int64_t)(k0 + bk) * lda, lda, m, bk, Lst, mp / 128,
                           Rst, np / 128, a.dst);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // ring memory back to generic use
            __syncthreads();
        }
        if (abort_flag) break;
        // ---------------- refinement ----------------
        double *xs = reinterpret_cast<double *>(smem);
        double *rsv = xs + n;
        refine_system(n, S.seed, A, a.d + S.v_off, a.rhs + S.v_off, a.x + S.v_off, a.maxit, xs, rsv, red,
                      reinterpret_cast<float(*)[kNB + 1]>(rsv + n), a.out + si);
        if (threadIdx.x == 0) a.out[si].info = sst->code == MXP_ZERO_PIVOT ? sst->info0 : 0;
    }

    __syncthreads();
    if (abort_flag && threadIdx.x == 0) {  // let copies still in flight land before TMEM is freed
        const unsigned long long t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < 50000ull) {
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_holder), "r"(kTmemCols)
                     : "memory");
    }
}

}  // namespace

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
struct BatchConfig {
    int b = 128, tile_n = 256, stages = 3;
};

}  // namespace mxp

using namespace mxp;

struct mxp_batch {
    int count = 0, device = 0, nmax = 0, grid = 0;
    std::vector<int> n;
    std::vector<uint64_t> seed;
    std::vector<int64_t> a_off, v_off;
    std::vector<int> order;          // descending n (longest first)
    int64_t matrix_floats = 0, vector_doubles = 0;
    BatchSys *d_sys = nullptr;
    int *d_order = nullptr;
    BatchOut *d_out = nullptr;
    DevStatus *d_sys_status = nullptr;
    DevStatus *d_status = nullptr;
    unsigned int *d_ticket = nullptr;
    uint8_t *d_staging = nullptr;
    int64_t staging_stride = 0, rstage_off = 0;
    BatchConfig cfg;
    int autotuned = 0;
    // captured launch (captured on a private stream, replayed on the caller's)
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void *g_A = nullptr, *g_d = nullptr, *g_rhs = nullptr, *g_x = nullptr;
    int g_maxit = -1, g_b = -1, g_tn = -1, g_st = -1, g_count = -1;
    const int *g_order = nullptr;
};

namespace {

constexpr int kBatchMaxN = 8192;

size_t ring_bytes(int tile_n, int stages) { return (size_t)stages * (kBlockBytes + (size_t)tile_n * 128); }

constexpr size_t kCbufBytes = 128 * 128 * 4;  // epilogue staging of C

size_t smem_bytes(const mxp_batch *bt, const BatchConfig &c) {
    size_t s = ring_bytes(c.tile_n, c.stages) + kCbufBytes;
    s = std::max(s, (size_t)16 * bt->nmax + sizeof(float) * kNB * (kNB + 1));  // x, r (FP64) + a 64 x 64 block
    s = std::max(s, kColStageOff + kColStageBytes);
    s = std::max(s, sizeof(SmemGV));  // the panel's cp.async-staged update tiles
    return s + 1024;                          // 1024-byte alignment of the ring
}

bool config_ok(const mxp_batch *bt, const BatchConfig &c) {
    if (c.b != 64 && c.b != 128 && c.b != 256) return false;
    if (c.tile_n != 128 && c.tile_n != 256) return false;
    if (c.stages < 2 || c.stages > kMaxStages) return false;
    return smem_bytes(bt, c) <= 227 * 1024;
}

mxp_status launch_batch(mxp_batch *bt, const BatchConfig &c, int count, const int *d_order, float *A,
                        const double *d, const double *rhs, double *x, int maxit, cudaStream_t st) {
    BatchKernelArgs ka;
    ka.a.sys = bt->d_sys;
    ka.a.order = d_order;
    ka.a.count = count;
    ka.a.b = c.b;
    ka.a.stages = c.stages;
    ka.a.maxit = maxit;
    ka.a.A = A;
    ka.a.d = d;
    ka.a.rhs = rhs;
    ka.a.x = x;
    ka.a.out = bt->d_out;
    ka.a.staging = bt->d_staging;
    ka.a.staging_stride = bt->staging_stride;
    ka.a.rstage_off = bt->rstage_off;
    ka.a.ticket = bt->d_ticket;
    ka.a.dst = bt->d_status;
    ka.sys_status = bt->d_sys_status;
    const size_t smem = smem_bytes(bt, c);
    MXP_CUDA(cudaMemsetAsync(bt->d_ticket, 0, sizeof(unsigned int), st));
    MXP_CUDA(cudaMemsetAsync(bt->d_sys_status, 0, sizeof(DevStatus) * bt->count, st));
    MXP_CUDA(cudaMemsetAsync(bt->d_status, 0, sizeof(DevStatus), st));
    const int grid = std::min(bt->grid, count);
    if (c.tile_n == 256)
        batched_kernel<256><<<grid, kBatchThreads, smem, st>>>(ka);
    else
        batched_kernel<128><<<grid, kBatchThreads, smem, st>>>(ka);
    MXP_CUDA(cudaGetLastError());
    MXP_LAUNCHED();
    return MXP_OK;
}

// Shared-memory opt-in of the kernel instance a configuration uses (set outside
// any stream capture).
mxp_status set_smem_attr(const mxp_batch *bt, const BatchConfig &c) {
    const int smem = (int)smem_bytes(bt, c);
    if (c.tile_n == 256)
        MXP_CUDA(cudaFuncSetAttribute(batched_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    else
        MXP_CUDA(cudaFuncSetAttribute(batched_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return MXP_OK;
}

mxp_status batch_status(mxp_batch *bt, cudaStream_t st) {
    DevStatus h;
    MXP_CUDA(cudaMemcpyAsync(&h, bt->d_status, sizeof(h), cudaMemcpyDeviceToHost, st));
    MXP_CUDA(cudaStreamSynchronize(st));
    if (h.code == MXP_TIMEOUT) return fail(MXP_TIMEOUT, "batch solve: a bounded wait timed out");
    if (h.code != 0) return fail((mxp_status)h.code, "batch solve: device error");
    return MXP_OK;
}

void drop_graph(mxp_batch *bt) {
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    bt->exec = nullptr;
}

}  // namespace

extern "C" mxp_status mxp_batch_sizes(int count, uint64_t size_seed, int *h_n) {
    if (count <= 0 || !h_n) return fail(MXP_INVALID_ARG, "batch_sizes: bad arguments");
    // value i of the generator stream from size_seed, v in [-0.5, 0.5], mapped
    // to N = 128 * (2 + floor((v + 0.5) * 31)), clamped to 128 * [2, 32]
    uint64_t s = lcg_stat00(size_seed);
    const Aff inc1 = lcg_inc1();
    for (int i = 0; i < count; ++i) {
        const double v = (double)(int64_t)s * 0x1.fffffffffffffP-65;
        int u = 2 + (int)std::floor((v + 0.5) * 31.0);
        u = std::min(32, std::max(2, u));
        h_n[i] = 128 * u;
        s = aff_apply(inc1, s);
    }
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_partition(int count, const int *h_n, int nparts, int *h_part) {
    if (count <= 0 || !h_n || !h_part || nparts <= 0) return fail(MXP_INVALID_ARG, "batch_partition: bad arguments");
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) {
        if (h_n[i] <= 0) return fail(MXP_INVALID_ARG, "batch_partition: every n must be positive");
        order[i] = i;
    }
    // largest first (stable: equal orders keep their index order)
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h_n[a] > h_n[b]; });
    std::vector<double> load(nparts, 0.0);
    for (int i : order) {
        int best = 0;
        for (int p = 1; p < nparts; ++p)
            if (load[p] < load[best]) best = p;
        const double n = h_n[i];
        load[best] += n * n * n;
        h_part[i] = best;
    }
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_create(int count, const int *h_n, const uint64_t *h_seed, int device,
                                       mxp_batch **out) {
    if (!out || count <= 0 || !h_n || !h_seed) return fail(MXP_INVALID_ARG, "batch_create: bad arguments");
    for (int i = 0; i < count; ++i)
        if (h_n[i] < 128 || h_n[i] > kBatchMaxN || h_n[i] % 128)
            return fail(MXP_INVALID_ARG, "batch_create: every n must be a multiple of 128 in [128, 8192]");
    int cur = 0;
    MXP_CUDA(cudaGetDevice(&cur));
    MXP_CUDA(cudaSetDevice(device));
    mxp_batch *bt = new mxp_batch();
    bt->count = count;
    bt->device = device;
    bt->n.assign(h_n, h_n + count);
    bt->seed.assign(h_seed, h_seed + count);
    bt->a_off.resize(count);
    bt->v_off.resize(count);
    for (int i = 0; i < count; ++i) {
        bt->a_off[i] = bt->matrix_floats;
        bt->v_off[i] = bt->vector_doubles;
        bt->matrix_floats += (int64_t)h_n[i] * h_n[i];
        bt->vector_doubles += h_n[i];
        bt->nmax = std::max(bt->nmax, h_n[i]);
    }
    bt->order.resize(count);
    for (int i = 0; i < count; ++i) bt->order[i] = i;
    std::stable_sort(bt->order.begin(), bt->order.end(), [&](int x, int y) { return bt->n[x] > bt->n[y]; });
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    bt->grid = std::max(1, sms);
    // staging for the largest block (256) and widest tile (256): L rows padded to
    // 128, R rows to 256, 256 FP16 per row
    const int64_t lrows = ((int64_t)bt->nmax + 127) / 128 * 128, rrows = ((int64_t)bt->nmax + 255) / 256 * 256;
    bt->rstage_off = lrows * 256 * 2;
    bt->staging_stride = (bt->rstage_off + rrows * 256 * 2 + 1023) / 1024 * 1024;
    std::vector<BatchSys> hs(count);
    for (int i = 0; i < count; ++i) hs[i] = BatchSys{h_n[i], 0, h_seed[i], bt->a_off[i], bt->v_off[i]};
    bool ok = cudaMalloc(&bt->d_sys, sizeof(BatchSys) * count) == cudaSuccess &&
              cudaMalloc(&bt->d_order, sizeof(int) * count) == cudaSuccess &&
              cudaMalloc(&bt->d_out, sizeof(BatchOut) * count) == cudaSuccess &&
              cudaMalloc(&bt->d_sys_status, sizeof(DevStatus) * count) == cudaSuccess &&
              cudaMalloc(&bt->d_status, sizeof(DevStatus)) == cudaSuccess &&
              cudaMalloc(&bt->d_ticket, 256) == cudaSuccess &&
              cudaMalloc(&bt->d_staging, (size_t)bt->staging_stride * bt->grid) == cudaSuccess &&
              cudaStreamCreateWithFlags(&bt->cap, cudaStreamNonBlocking) == cudaSuccess;
    if (ok)
        ok = cudaMemcpy(bt->d_sys, hs.data(), sizeof(BatchSys) * count, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(bt->d_order, bt->order.data(), sizeof(int) * count, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemset(bt->d_out, 0, sizeof(BatchOut) * count) == cudaSuccess;
    cudaSetDevice(cur);
    if (!ok) {
        cudaGetLastError();
        mxp_batch_destroy(bt);
        return fail(MXP_NO_MEMORY, "batch_create: device allocation failed");
    }
    *out = bt;
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_destroy(mxp_batch *bt) {
    if (!bt) return MXP_OK;
    drop_graph(bt);
    cudaFree(bt->d_sys);
    cudaFree(bt->d_order);
    cudaFree(bt->d_out);
    cudaFree(bt->d_sys_status);
    cudaFree(bt->d_status);
    cudaFree(bt->d_ticket);
    cudaFree(bt->d_staging);
    if (bt->cap) cudaStreamDestroy(bt->cap);
    delete bt;
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_layout(const mxp_batch *bt, int64_t *matrix_floats, int64_t *vector_doubles,
                                       int64_t *h_a_off, int64_t *h_v_off) {
    if (!bt) return fail(MXP_INVALID_ARG, "batch_layout: batch is NULL");
    if (matrix_floats) *matrix_floats = bt->matrix_floats;
    if (vector_doubles) *vector_doubles = bt->vector_doubles;
    for (int i = 0; i < bt->count; ++i) {
        if (h_a_off) h_a_off[i] = bt->a_off[i];
        if (h_v_off) h_v_off[i] = bt->v_off[i];
    }
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_matgen(mxp_batch *bt, float *d_A, double *d_d, double *d_rhs, void *stream) {
    if (!bt || !d_A || !d_d || !d_rhs) return fail(MXP_INVALID_ARG, "batch_matgen: NULL argument");
    cudaStream_t st = as_stream(stream);
    for (int i = 0; i < bt->count; ++i) {
        mxp_status s = launch_matgen(bt->n[i], bt->seed[i], MXP_DIAG_ROWSUM, d_A + bt->a_off[i], bt->n[i],
                                     d_d + bt->v_off[i], nullptr, d_rhs + bt->v_off[i], st);
        if (s != MXP_OK) return s;
    }
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_set_config(mxp_batch *bt, int b, int tile_n, int stages) {
    if (!bt) return fail(MXP_INVALID_ARG, "batch_set_config: batch is NULL");
    BatchConfig c{b, tile_n, stages};
    if (!config_ok(bt, c))
        return fail(MXP_INVALID_ARG, "batch_set_config: b in {64,128,256}, tile_n in {128,256}, stages 2..4 "
                                     "within 227 KB of shared memory");
    bt->cfg = c;
    drop_graph(bt);
    return MXP_OK;
}

extern "C" mxp_status mxp_batch_solve(mxp_batch *bt, float *d_A, const double *d_d, const double *d_rhs,
                                      double *d_x, int maxit, void *stream, mxp_batch_stats *stats) {
    if (!bt || !d_A || !d_d || !d_rhs || !d_x) return fail(MXP_INVALID_ARG, "batch_solve: NULL argument");
    if (maxit < 1) return fail(MXP_INVALID_ARG, "batch_solve: maxit < 1");
    cudaStream_t st = as_stream(stream);
    const BatchConfig &c = bt->cfg;
    // the launch (counter resets + the persistent kernel) is captured once per
    // set of buffers / configuration and replayed as a CUDA graph
    if (!bt->exec || bt->g_A != d_A || bt->g_d != d_d || bt->g_rhs != d_rhs || bt->g_x != d_x ||
        bt->g_maxit != maxit || bt->g_b != c.b || bt->g_tn != c.tile_n || bt->g_st != c.stages ||
        bt->g_count != bt->count || bt->g_order != bt->d_order) {
        drop_graph(bt);
        mxp_status sa = set_smem_attr(bt, c);
        if (sa != MXP_OK) return sa;
        cudaGraph_t g = nullptr;
        MXP_CUDA(cudaStreamBeginCapture(bt->cap, cudaStreamCaptureModeThreadLocal));
        mxp_status s = launch_batch(bt, c, bt->count, bt->d_order, d_A, d_d, d_rhs, d_x, maxit, bt->cap);
        cudaError_t e = cudaStreamEndCapture(bt->cap, &g);
        if (s != MXP_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_fail(e, "batch_solve: stream capture");
        e = cudaGraphInstantiate(&bt->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            bt->exec = nullptr;
            return cuda_fail(e, "batch_solve: graph instantiation");
        }
        bt->g_A = d_A;
        bt->g_d = d_d;
        bt->g_rhs = d_rhs;
        bt->g_x = d_x;
        bt->g_maxit = maxit;
        bt->g_b = c.b;
        bt->g_tn = c.tile_n;
        bt->g_st = c.stages;
        bt->g_count = bt->count;
        bt->g_order = bt->d_order;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    cudaError_t e = cudaGraphLaunch(bt->exec, st);
    cudaEventRecord(e1, st);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return cuda_fail(e, "batch_solve: graph launch");
    }
    MXP_LAUNCHED();
    mxp_status s = batch_status(bt, st);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->ms_total = ms;
        stats->b = c.b;
        stats->tile_n = c.tile_n;
        stats->stages = c.stages;
        stats->autotuned = bt->autotuned;
        stats->grid = std::min(bt->grid, bt->count);
    }
    return s;
}

extern "C" mxp_status mxp_batch_results(const mxp_batch *bt, mxp_batch_result *h_results) {
    if (!bt || !h_results) return fail(MXP_INVALID_ARG, "batch_results: NULL argument");
    static_assert(sizeof(mxp_batch_result) == sizeof(BatchOut), "result layout");
    MXP_CUDA(cudaMemcpy(h_results, bt->d_out, sizeof(BatchOut) * bt->count, cudaMemcpyDeviceToHost));
    return MXP_OK;
}

// Autotuner: times every admissible (b, tile_n, stages) on a sample of the
// batch (every stride-th system in size order, regenerated before each run)
// and keeps the fastest per credited FLOP.
extern "C" mxp_status mxp_batch_autotune(mxp_batch *bt, float *d_A, double *d_d, double *d_rhs, double *d_x,
                                         int sample, void *stream, mxp_batch_stats *stats) {
    if (!bt || !d_A || !d_d || !d_rhs || !d_x) return fail(MXP_INVALID_ARG, "batch_autotune: NULL argument");
    cudaStream_t st = as_stream(stream);
    if (sample <= 0 || sample > bt->count) sample = std::min(bt->count, std::max(bt->grid, bt->count / 8));
    std::vector<int> sub;
    const double stride = (double)bt->count / sample;
    for (int i = 0; i < sample; ++i) sub.push_back(bt->order[(int)(i * stride)]);
    int *d_sub = nullptr;
    MXP_CUDA(cudaMalloc(&d_sub, sizeof(int) * sub.size()));
    MXP_CUDA(cudaMemcpy(d_sub, sub.data(), sizeof(int) * sub.size(), cudaMemcpyHostToDevice));
    auto regen = [&]() -> mxp_status {
        for (int i : sub) {
            mxp_status s = launch_matgen(bt->n[i], bt->seed[i], MXP_DIAG_ROWSUM, d_A + bt->a_off[i], bt->n[i],
                                         d_d + bt->v_off[i], nullptr, d_rhs + bt->v_off[i], st);
            if (s != MXP_OK) return s;
        }
        return MXP_OK;
    };
    BatchConfig best = bt->cfg;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    mxp_status s = MXP_OK;
    for (int b : {64, 128, 256})
        for (int tn : {128, 256})
            for (int stg : {2, 3, 4}) {
                BatchConfig c{b, tn, stg};
                if (!config_ok(bt, c) || s != MXP_OK) continue;
                s = set_smem_attr(bt, c);
                if (s != MXP_OK) break;
                float tot = 0.0f;
                for (int rep = 0; rep < 2 && s == MXP_OK; ++rep) {
                    s = regen();
                    if (s != MXP_OK) break;
                    cudaEventRecord(e0, st);
                    s = launch_batch(bt, c, (int)sub.size(), d_sub, d_A, d_d, d_rhs, d_x, 50, st);
                    cudaEventRecord(e1, st);
                    if (s == MXP_OK) s = batch_status(bt, st);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep == 1) tot = ms;  // the first run warms up
                }
                if (s == MXP_OK && tot < best_ms) {
                    best_ms = tot;
                    best = c;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_sub);
    if (s != MXP_OK) return s;
    bt->cfg = best;
    bt->autotuned = 1;
    drop_graph(bt);
    if (stats) {
        stats->ms_total = best_ms;
        stats->b = best.b;
        stats->tile_n = best.tile_n;
        stats->stages = best.stages;
        stats->autotuned = 1;
        stats->grid = std::min(bt->grid, (int)sub.size());
    }
    return MXP_OK;
}
