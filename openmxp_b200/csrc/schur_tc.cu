// Schur update C -= L * R^T on the 5th-generation tensor cores (tcgen05).
//
// Reference: the FP16 gemm_ex calls of the LU loop (GPUBLAS_SGEMM_EX with
// OP_N, OP_T, alpha = -1, beta = 1, FP16 inputs, FP32 C and compute;
// panel_trf.hpp:661-665, 710-715, 734-740, 828-834; rocm_device_macros.h:
// 267-268).  The reference reaches matrix cores only through that library
// call; this is a hand-written sm_100a kernel.
//
// Design (one CTA per SM, persistent over output tiles):
//   * tile 128 (rows of L) x 256 (rows of R), K step 64 (2-byte types),
//     4-stage shared-memory ring filled by TMA (cp.async.bulk.tensor, 128-byte
//     swizzle, single-destination loads), synchronised with mbarriers;
//   * warp 0: TMA producer; warp 1: allocates 512 TMEM columns and issues
//     tcgen05.mma (kind::f16, M=128, N=256, K=16) from one lane, committing
//     each stage back to the producer and each finished accumulator to the
//     epilogue;
//   * warps 2..9: epilogue.  Two TMEM accumulators (2 x 256 columns) let the
//     epilogue of tile t overlap the main loop of tile t+1.  Each epilogue
//     warp reads its 32-lane quarter of the accumulator (tcgen05.ld 32x32b),
//     and applies C -= acc to FP32 C in place with 128-byte coalesced
//     accesses (lanes = consecutive rows of the column-major C);
//   * every mbarrier wait is bounded (%globaltimer); on timeout the kernel
//     records MXP_TIMEOUT in the status word, drains, frees TMEM and returns.
//
// Operands are K-major (row i of the panel holds its K values contiguously),
// as written by the panel-cast kernels.  Out-of-range rows / K columns are
// zero-filled by TMA; C is masked in the epilogue.
#include <cudaTypedefs.h>

#include <mutex>

#include "fp8_quant.cuh"
#include "mxp_internal.cuh"
#include "tc_ptx.cuh"

namespace mxp {

namespace {

using namespace tc;

constexpr int kBM = 128;
constexpr int kBN = 256;
constexpr int kStages = 4;
constexpr int kStageBytesA = kBM * 128;  // 128 rows x 128 bytes of K
constexpr int kStageBytesB = kBN * 128;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;  // 2 control warps + epilogue
constexpr int kTmemCols = 512;
constexpr int kRing = 8;  // tile-index ring between the producer and the consumers
constexpr int kSmemBytes = 1024 /*align slack*/ + kStages * (kStageBytesA + kStageBytesB) + 512;

__host__ __device__ constexpr uint32_t idesc_f16(uint32_t ab_fmt) { return idesc_f16_mn(ab_fmt, kBM, kBN); }

struct TileMap {
    int tiles_m, tiles_n, group_m;
    __device__ __forceinline__ void get(int t, int &tm, int &tn) const {
        const int per_group = group_m * tiles_n;
        const int g = t / per_group;
        const int local = t - g * per_group;
        const int gm = min(group_m, tiles_m - g * group_m);
        tm = g * group_m + local % gm;
        tn = local / gm;
    }
};

// Where a CTA's tiles come from.  counter == nullptr: static round robin
// (blockIdx.x, + gridDim.x, ...).  Otherwise every tile is claimed from a
// device counter (zeroed before the first launch that uses it), so several
// launches with the same arguments can share one pass: a launch whose CTAs
// start late simply claims fewer tiles.  Tiles with tm < skip_m and
// tn < skip_n are not computed (a corner updated by another launch).
struct TileSrc {
    int *counter;
    int skip_m, skip_n;
};

// Producer side: the next tile of this CTA, or -1 when the pass is done.
__device__ __forceinline__ int fetch_tile(const TileMap &tiles, const TileSrc &src, int total,
                                          int &t_static) {
    for (;;) {
        int t;
        if (src.counter) {
            t = atomicAdd(src.counter, 1);
        } else {
            t = t_static;
            t_static += gridDim.x;
        }
        if (t >= total) return -1;
        if (src.skip_m > 0) {
            int tm, tn;
            tiles.get(t, tm, tn);
            if (tm < src.skip_m && tn < src.skip_n) continue;
        }
        return t;
    }
}

// The ring: slot s holds a tile index; sfull[s] (count 1) is arrived by the
// producer after writing it, sempty[s] (count 1 + kEpiWarps) by the MMA lane
// and each epilogue warp after reading it.
struct TileRing {
    uint64_t *sfull, *sempty;
    volatile int *ids;
};

__device__ __forceinline__ bool ring_put(const TileRing &r, int &slot, uint32_t &phase, int t,
                                         volatile int *abort_flag) {
    if (!mbar_wait(smem_u32(&r.sempty[slot]), phase ^ 1u, abort_flag)) return false;
    r.ids[slot] = t;
    mbar_arrive(smem_u32(&r.sfull[slot]));
    if (++slot == kRing) {
        slot = 0;
        phase ^= 1u;
    }
    return true;
}

// Single-thread consumer (the MMA lane).
__device__ __forceinline__ bool ring_take1(const TileRing &r, int &slot, uint32_t &phase, int &t,
                                           volatile int *abort_flag) {
    if (!mbar_wait(smem_u32(&r.sfull[slot]), phase, abort_flag)) return false;
    t = r.ids[slot];
    mbar_arrive(smem_u32(&r.sempty[slot]));
    if (++slot == kRing) {
        slot = 0;
        phase ^= 1u;
    }
    return true;
}

// Whole-warp consumer (an epilogue warp): every lane waits and reads, the
// warp agrees on success, lane 0 releases the slot.
__device__ __forceinline__ bool ring_take_warp(const TileRing &r, int &slot, uint32_t &phase, int &t,
                                               volatile int *abort_flag) {
    const bool got = mbar_wait(smem_u32(&r.sfull[slot]), phase, abort_flag);
    if (!__all_sync(0xffffffffu, got)) return false;
    t = r.ids[slot];
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(smem_u32(&r.sempty[slot]));
    if (++slot == kRing) {
        slot = 0;
        phase ^= 1u;
    }
    return true;
}

__device__ __forceinline__ void ring_init(const TileRing &r) {
    for (int s = 0; s < kRing; ++s) {
        mbar_init(smem_u32(&r.sfull[s]), 1);
        mbar_init(smem_u32(&r.sempty[s]), 1 + kEpiWarps);
    }
}

template <bool F8>
__global__ void __launch_bounds__(kThreads, 1)
schur_tc_f16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int M, int N, int K, float *__restrict__ C, int64_t ldc, uint32_t idesc,
                    TileMap tiles, TileSrc src, int store, int tri_mode, int seg, F8Out f8, DevStatus *dst) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                ~uintptr_t(1023));
    uint8_t *sA = smem;
    uint8_t *sB = smem + kStages * kStageBytesA;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + kStages * kStageBytesB);
    uint64_t *full = bars;                     // [kStages]
    uint64_t *empty = bars + kStages;          // [kStages]
    uint64_t *tfull = bars + 2 * kStages;      // [2]
    uint64_t *tempty = bars + 2 * kStages + 2; // [2]
    const TileRing ring{bars + 2 * kStages + 4, bars + 2 * kStages + 4 + kRing,
                        reinterpret_cast<volatile int *>(bars + 2 * kStages + 4 + 2 * kRing)};
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 4 + 2 * kRing) + kRing;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);
    // FP8 copy of the output (store mode): per column half, the four epilogue
    // warps meet at amax_bar (count 4) to combine their 32-row amax partials
    // (double-buffered by tile parity)
    uint64_t *amax_bar = bars + 40;                                    // [2]
    float *amax_part = reinterpret_cast<float *>(bars + 42);           // [2 parity][2 half][4 quarter]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total_tiles = tiles.tiles_m * tiles.tiles_n;
    const int nk = (K + 63) / 64;
    // Triangular operand (panel solves against a triangular inverse): a tile
    // only needs the K stages, within each of the K segments of length seg,
    // below its column (tri_mode 1) or row (tri_mode 2) extent.
    // In each K segment of seg_st stages a tile needs the first stage_count
    // of them.  The stage loops walk the segments with a position counter and
    // jump over the rest of a segment: testing every skipped stage with a
    // runtime modulo cost ~0.15 us per stage on the issuing thread, ~5 us for
    // a tile that needs 4 of 40 stages, and held back the producer's next tile.
    const int seg_st = tri_mode ? seg / 64 : nk;
    auto stage_count = [&](int tm, int tn) -> int {
        if (tri_mode == 0) return nk;
        return min(seg_st, (tri_mode == 1 ? (tn + 1) * kBN : (tm + 1) * kBM) / 64);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&tfull[a]), 1);
            mbar_init(smem_u32(&tempty[a]), kEpiWarps);
        }
        ring_init(ring);
        mbar_init(smem_u32(&amax_bar[0]), 4);
        mbar_init(smem_u32(&amax_bar[1]), 4);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int rslot = 0, t_static = blockIdx.x;
            uint32_t rphase = 0;
            bool ok = true;
            while (ok) {
                const int t = fetch_tile(tiles, src, total_tiles, t_static);
                if (!ring_put(ring, rslot, rphase, t, abort_flag)) {
                    ok = false;
                    break;
                }
                if (t < 0) break;
                int tm, tn;
                tiles.get(t, tm, tn);
                const int cnt = stage_count(tm, tn);
                int pos = -1;
                for (int kb = 0; kb < nk; ++kb) {
                    if (++pos == seg_st) pos = 0;
                    if (pos >= cnt) {  // the rest of this segment is not needed
                        kb += seg_st - 1 - pos;
                        pos = seg_st - 1;
                        continue;
                    }
                    if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[stage]);
                    mbar_expect_tx(fb, kStageBytesA + kStageBytesB);
                    tma_load_2d(smem_u32(sA + stage * kStageBytesA), &tmA, kb * 64, tm * kBM, fb);
                    tma_load_2d(smem_u32(sB + stage * kStageBytesB), &tmB, kb * 64, tn * kBN, fb);
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (!ok) {
                *abort_flag = 1;
                report(dst, MXP_TIMEOUT, 1, blockIdx.x);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t it = 0;
            int rslot = 0;
            uint32_t rphase = 0;
            bool ok = true;
            for (;; ++it) {
                int t;
                if (!ring_take1(ring, rslot, rphase, t, abort_flag)) {
                    ok = false;
                    break;
                }
                if (t < 0) break;
                int tm, tn;
                tiles.get(t, tm, tn);
                const uint32_t acc = it & 1u, acc_phase = (it >> 1) & 1u;
                if (!mbar_wait(smem_u32(&tempty[acc]), acc_phase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + acc * kBN;
                bool first = true;
                const int cnt = stage_count(tm, tn);
                int pos = -1;
                for (int kb = 0; kb < nk; ++kb) {
                    if (++pos == seg_st) pos = 0;
                    if (pos >= cnt) {
                        kb += seg_st - 1 - pos;
                        pos = seg_st - 1;
                        continue;
                    }
                    if (!mbar_wait(smem_u32(&full[stage]), phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(sA + stage * kStageBytesA);
                    const uint32_t b0 = smem_u32(sB + stage * kStageBytesB);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        tc_mma_f16(d_tmem, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k),
                                   idesc, (!first || k > 0) ? 1u : 0u);
                    }
                    first = false;
                    tc_commit(smem_u32(&empty[stage]));
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                tc_commit(smem_u32(&tfull[acc]));
            }
            if (!ok) {
                *abort_flag = 1;
                report(dst, MXP_TIMEOUT, 2, blockIdx.x);
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int ew = warp - 2;             // 0..7
        const int quarter = warp & 3;        // TMEM lane quarter this warp may access
        const int col_half = ew >> 2;        // which 128 columns of the 256
        uint32_t it = 0;
        int rslot = 0;
        uint32_t rphase = 0;
        bool ok = true;
        for (;; ++it) {
            int t;
            if (!ring_take_warp(ring, rslot, rphase, t, abort_flag)) {
                ok = false;
                break;
            }
            if (t < 0) break;
            int tm, tn;
            tiles.get(t, tm, tn);
            const uint32_t acc = it & 1u, acc_phase = (it >> 1) & 1u;
            if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&tfull[acc]), acc_phase, abort_flag))) {
                ok = false;
                break;
            }
            __syncwarp();
            tc_fence_after();
            const int64_t row = (int64_t)tm * kBM + quarter * 32 + lane;
            const bool row_ok = row < M;
            const float sg = store == 2 ? -1.0f : 1.0f;
            float rmax = 0.0f;  // |C| over this thread's 128 columns (FP8 copy)
#pragma unroll 1
            for (int c0 = col_half * 128; c0 < col_half * 128 + 128; c0 += 32) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quarter * 32) << 16) + acc * kBN + c0, r);
                const int64_t col0 = (int64_t)tn * kBN + c0;
                if (row_ok) {
                    float *cp = C + col0 * ldc + row;
                    float cv[32];
                    const int ncol = (int)imin64(32, (int64_t)N - col0);
                    if (store) {  // C = acc (panel solves), or C = -acc (store == 2)
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < ncol) __stcs(cp + j * ldc, sg * __uint_as_float(r[j]));
                        if (F8) {
#pragma unroll
                            for (int j = 0; j < 32; ++j) rmax = fmaxf(rmax, fabsf(sg * __uint_as_float(r[j])));
                        }
                    } else if (ncol >= 32) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) cv[j] = __ldcs(cp + j * ldc);
#pragma unroll
                        for (int j = 0; j < 32; ++j) __stcs(cp + j * ldc, cv[j] - __uint_as_float(r[j]));
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < ncol) cp[j * ldc] = cp[j * ldc] - __uint_as_float(r[j]);
                    }
                }
            }
            if (F8) {
                // E4M3 copy of this 128 x 128 block of C with one power-of-two
                // scale from its amax, as cast_left_fp8_kernel makes from C in
                // memory (same values, same rounding, same bytes)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
                const uint32_t par = it & 1u;
                float *part = amax_part + (par * 2 + col_half) * 4;
                if (lane == 0) {
                    part[quarter] = rmax;
                    mbar_arrive(smem_u32(&amax_bar[col_half]));
                }
                const bool met = mbar_wait(smem_u32(&amax_bar[col_half]), par, abort_flag);
                if (!__all_sync(0xffffffffu, met)) {
                    ok = false;
                    break;
                }
                const float amax = fmaxf(fmaxf(part[0], part[1]), fmaxf(part[2], part[3]));
                const int e = e4m3_scale_exp(amax);
                const float up = e4m3_scale_up(e);
#pragma unroll 1
                for (int c0 = col_half * 128; c0 < col_half * 128 + 128; c0 += 32) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quarter * 32) << 16) + acc * kBN + c0, r);
                    if (row_ok && f8.trans) {
                        // R layout: row j of the panel holds its k contiguously, so for
                        // each column j the 32 lanes (32 consecutive k) store one
                        // 32-byte run
                        uint8_t *dp = f8.out + ((int64_t)tn * kBN + c0) * f8.ldk + row;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            dp[j * f8.ldk] = to_e4m3(__fmul_rn(sg * __uint_as_float(r[j]), up));
                    } else if (row_ok) {
                        uint32_t w[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            uint32_t v = 0u;
#pragma unroll
                            for (int b4 = 0; b4 < 4; ++b4)
                                v |= (uint32_t)to_e4m3(__fmul_rn(sg * __uint_as_float(r[4 * q + b4]), up)) << (8 * b4);
                            w[q] = v;
                        }
                        uint4 *dp = reinterpret_cast<uint4 *>(f8.out + row * f8.ldk + (int64_t)tn * kBN + c0);
                        dp[0] = make_uint4(w[0], w[1], w[2], w[3]);
                        dp[1] = make_uint4(w[4], w[5], w[6], w[7]);
                    }
                }
                if (lane == 0 && quarter == 0) {
                    if (f8.trans) f8.sc[(int64_t)(2 * tn + col_half) * f8.sc_ld + tm] = (uint8_t)(127 - e);
                    else f8.sc[(int64_t)tm * f8.sc_ld + 2 * tn + col_half] = (uint8_t)(127 - e);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&tempty[acc]));
        }
        if (!ok && lane == 0) {
            *abort_flag = 1;
            report(dst, MXP_TIMEOUT, 3, blockIdx.x);
        }
    }

    __syncthreads();
    if (*abort_flag) {
        // Let any TMA copy / MMA still in flight land before TMEM and shared
        // memory are released.  The abort is raised only by a role whose wait
        // ran out (2 s); every other role leaves at its next bounded wait, so
        // the producer issues nothing after it sees the flag and at most
        // kStages stages of loads (and the MMAs of as many stages) can still
        // be in flight.  Each completes within the memory latency and one
        // stage's MMA time, a few microseconds even under the full load of
        // the GPU (the per-stage traces of these kernels show ~1-2 us from a
        // load's issue to its data); 50 us is an order of magnitude above
        // that.  A wait on the stages' own barriers is not used here because
        // a barrier whose phase was never completed would make this path
        // wait out another timeout.
        if (threadIdx.x == 0) {
            const unsigned long long t0 = globaltimer_ns();
            while (globaltimer_ns() - t0 < 50000ull) {
            }
        }
        __syncthreads();
    }
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

// ---- FP8 E4M3, block-scaled (kind::mxf8f6f4.block_scale) ---------------------
//
// Same pipeline with 128-byte K stages (128 FP8 values).  Each 128 x 128 tile
// of a panel carries one UE8M0 scale (2^-e, e from the tile amax); a stage of
// K = 128 covers exactly one scale tile, so the stage's scale factors are
// uniform per 128 rows.  Once per four stages warp 0 writes them to shared
// memory in the MX scale-factor atom layout (32 rows x 16 bytes; row r's
// 32-bit word for its lane quarter at byte (r%32)*16 + (r/32)*4), byte g of
// the word holding the scale of the group's stage g, next to the TMA tiles;
// the MMA lane moves them to TMEM with tcgen05.cp (32x128b, replicated to the
// four lane quarters) and issues tcgen05.mma ... kind::mxf8f6f4.block_scale
// with sf_id = the stage's byte, which applies the scales inside the MMA.
// Copying per group rather than per stage issues a quarter of the copies
// (measured neutral in throughput: the kernel is power-bound).  TMEM: one
// 256-column accumulator (cols 0..255) plus
// two scale-factor slots (cols 256..287).  The epilogue copies the whole
// accumulator to registers first and releases TMEM, so its C update overlaps
// the next tile's main loop.
constexpr int kF8BN = 256;
constexpr int kF8StageA = kBM * 128;
constexpr int kF8StageB = kF8BN * 128;
constexpr int kF8StageSF = 2048;  // SFA 512 B + SFB 1024 B, padded
constexpr int kF8StageBytes = kF8StageA + kF8StageB + kF8StageSF;
constexpr int kF8Stages = 4;
constexpr int kF8SmemBytes = 1024 + kF8Stages * kF8StageBytes + 512;
constexpr int kF8SfCol0 = 256;
// Stages whose scale factors share one TMEM copy: a tile's scale is uniform
// over its 128 x 128 block, so the four K blocks of a stage use one byte of
// the 32-bit scale word and one word carries four stages (byte = stage % 4,
// selected by sf_id).  Two TMEM slots (16 columns each) alternate by group.
constexpr int kF8SfGroup = 4;

__device__ __forceinline__ void tc_cp_32x128b_x4(uint32_t taddr, uint64_t sdesc) {
    asm volatile("tcgen05.cp.cta_group::1.32x128b.warpx4 [%0], %1;" ::"r"(taddr), "l"(sdesc)
                 : "memory");
}

__device__ __forceinline__ void tc_mma_mxf8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t sfa, uint32_t sfb,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::mxf8f6f4.block_scale [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(
            d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
        : "memory");
}

// Scale-factor tile: 32 rows x 16 bytes, no swizzle; 8-row core matrices 128 B apart.
__device__ __forceinline__ uint64_t smem_desc_sf(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;           // LBO: a single core matrix along K
    d |= (uint64_t)(128 >> 4) << 32;  // SBO
    d |= (uint64_t)1 << 46;           // version
    return d;                         // layout type 0 = no swizzle
}

// Block-scaled instruction descriptor: A, B = E4M3, K-major, UE8M0 scales,
// M = 128, N = 256, dense K = 32; sf_id picks the byte (k-block) of the scale words.
__host__ __device__ constexpr uint32_t idesc_mxf8(uint32_t sf_id) {
    return (sf_id << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(kF8BN >> 3) << 17) | (1u << 23) |
           ((uint32_t)(kBM >> 4) << 24) | (sf_id << 29);
}

__global__ void __launch_bounds__(kThreads, 1)
schur_tc_fp8_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int M, int N, int K, const uint8_t *__restrict__ lsc,
                    const uint8_t *__restrict__ rsc, int lsc_ld, int rsc_ld, float *__restrict__ C,
                    int64_t ldc, TileMap tiles, TileSrc src, DevStatus *dst) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kF8Stages * kF8StageBytes);
    uint64_t *full = bars;
    uint64_t *empty = bars + kF8Stages;
    uint64_t *tfull = bars + 2 * kF8Stages;
    uint64_t *tempty = bars + 2 * kF8Stages + 1;
    const TileRing ring{bars + 2 * kF8Stages + 2, bars + 2 * kF8Stages + 2 + kRing,
                        reinterpret_cast<volatile int *>(bars + 2 * kF8Stages + 2 + 2 * kRing)};
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + 2 * kF8Stages + 2 + 2 * kRing) + kRing;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);
    auto stA = [&](int s) { return smem + s * kF8StageBytes; };
    auto stB = [&](int s) { return smem + s * kF8StageBytes + kF8StageA; };
    auto stSF = [&](int s) { return smem + s * kF8StageBytes + kF8StageA + kF8StageB; };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total_tiles = tiles.tiles_m * tiles.tiles_n;
    const int nk = (K + 127) / 128;
    const int rtiles = (N + 127) / 128;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kF8Stages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(tfull), 1);
        mbar_init(smem_u32(tempty), kEpiWarps);
        ring_init(ring);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;

    if (warp == 0) {
        // ---------------- producer: scale factors (whole warp) + TMA (lane 0) ----------------
        int stage = 0;
        uint32_t phase = 0;
        int rslot = 0, t_static = blockIdx.x;
        uint32_t rphase = 0;
        bool ok = true;
        while (ok) {
            int t = 0, put = 1;
            if (lane == 0) {
                t = fetch_tile(tiles, src, total_tiles, t_static);
                put = ring_put(ring, rslot, rphase, t, abort_flag) ? 1 : 0;
            }
            t = __shfl_sync(0xffffffffu, t, 0);
            if (!__shfl_sync(0xffffffffu, put, 0)) {
                ok = false;
                break;
            }
            if (t < 0) break;
            int tm, tn;
            tiles.get(t, tm, tn);
            // Scale bytes of 64 stages at a time, lane i holding stages i and
            // 32 + i: loaded before the slot wait, so the global-load latency
            // stays off the per-stage path to the TMA issue.
            uint32_t ra[2] = {0u, 0u}, rb0[2] = {0u, 0u}, rb1[2] = {127u, 127u};
            const bool has_b1 = 2 * tn + 1 < rtiles;
            for (int kb = 0; kb < nk; ++kb) {
                if ((kb & 63) == 0) {
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int kx = kb + 32 * j + lane;
                        if (kx < nk) {
                            ra[j] = lsc[(int64_t)tm * lsc_ld + kx];
                            rb0[j] = rsc[(int64_t)(2 * tn) * rsc_ld + kx];
                            rb1[j] = has_b1 ? rsc[(int64_t)(2 * tn + 1) * rsc_ld + kx] : 127u;
                        }
                    }
                }
                int got = 1;
                if (lane == 0) got = mbar_wait(smem_u32(&empty[stage]), phase ^ 1u, abort_flag) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                // operand tiles first (the barrier expects their bytes), then, at
                // the first stage of a group, the group's scale factors; the
                // single arrival comes after both
                const uint32_t fb = smem_u32(&full[stage]);
                if (lane == 0) {
                    mbar_expect_tx_only(fb, kF8StageA + kF8StageB);
                    tma_load_2d(smem_u32(stA(stage)), &tmA, kb * 128, tm * kBM, fb);
                    tma_load_2d(smem_u32(stB(stage)), &tmB, kb * 128, tn * kF8BN, fb);
                }
                if ((kb & (kF8SfGroup - 1)) == 0) {
                    // byte g of each scale word = the scale of stage kb + g (2^0 past K)
                    uint32_t wa = 0u, wb0 = 0u, wb1 = 0u;
#pragma unroll
                    for (int g = 0; g < kF8SfGroup; ++g) {
                        const int kx = kb + g;
                        const bool hi = (kx & 32) != 0;
                        const int src_lane = kx & 31;
                        uint32_t va = __shfl_sync(0xffffffffu, hi ? ra[1] : ra[0], src_lane);
                        uint32_t v0 = __shfl_sync(0xffffffffu, hi ? rb0[1] : rb0[0], src_lane);
                        uint32_t v1 = __shfl_sync(0xffffffffu, hi ? rb1[1] : rb1[0], src_lane);
                        if (kx >= nk) va = v0 = v1 = 127u;
                        wa |= va << (8 * g);
                        wb0 |= v0 << (8 * g);
                        wb1 |= v1 << (8 * g);
                    }
                    uint4 *sf = reinterpret_cast<uint4 *>(stSF(stage));
                    sf[lane] = make_uint4(wa, wa, wa, wa);             // SFA: rows 0..127
                    sf[32 + lane] = make_uint4(wb0, wb0, wb0, wb0);    // SFB atom 0: rows 0..127
                    sf[64 + lane] = make_uint4(wb1, wb1, wb1, wb1);    // SFB atom 1: rows 128..255
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(fb);
                if (++stage == kF8Stages) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
        }
        if (!ok && lane == 0) {
            *abort_flag = 1;
            report(dst, MXP_TIMEOUT, 4, blockIdx.x);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t it = 0;
            uint32_t groups = 0;  // scale-factor groups copied so far (their TMEM slot alternates)
            int rslot = 0;
            uint32_t rphase = 0;
            bool ok = true;
            for (;; ++it) {
                int t;
                if (!ring_take1(ring, rslot, rphase, t, abort_flag)) {
                    ok = false;
                    break;
                }
                if (t < 0) break;
                if (!mbar_wait(smem_u32(tempty), (it & 1u) ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(smem_u32(&full[stage]), phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t gpos = (uint32_t)(kb & (kF8SfGroup - 1));
                    if (gpos == 0) ++groups;
                    const uint32_t sfa_t = tmem_base + kF8SfCol0 + 16u * (groups & 1u);
                    const uint32_t sfb_t = sfa_t + 4u;
                    if (gpos == 0) {  // the group's scales, written with its first stage
                        const uint32_t sf0 = smem_u32(stSF(stage));
                        tc_cp_32x128b_x4(sfa_t, smem_desc_sf(sf0));
                        tc_cp_32x128b_x4(sfb_t, smem_desc_sf(sf0 + 512));
                        tc_cp_32x128b_x4(sfb_t + 4u, smem_desc_sf(sf0 + 1024));
                    }
                    const uint32_t a0 = smem_u32(stA(stage));
                    const uint32_t b0 = smem_u32(stB(stage));
                    // the stage's four K blocks share its tile scale: byte gpos
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        tc_mma_mxf8(tmem_base, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k),
                                    idesc_mxf8(gpos), sfa_t, sfb_t, (kb > 0 || k > 0) ? 1u : 0u);
                    }
                    tc_commit(smem_u32(&empty[stage]));
                    if (++stage == kF8Stages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                tc_commit(smem_u32(tfull));
            }
            if (!ok) {
                *abort_flag = 1;
                report(dst, MXP_TIMEOUT, 5, blockIdx.x);
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int ew = warp - 2;
        const int quarter = warp & 3;
        const int col_half = ew >> 2;
        uint32_t it = 0;
        int rslot = 0;
        uint32_t rphase = 0;
        bool ok = true;
        for (;; ++it) {
            int t;
            if (!ring_take_warp(ring, rslot, rphase, t, abort_flag)) {
                ok = false;
                break;
            }
            if (t < 0) break;
            int tm, tn;
            tiles.get(t, tm, tn);
            if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(tfull), it & 1u, abort_flag))) {
                ok = false;
                break;
            }
            __syncwarp();
            tc_fence_after();
            uint32_t r[4][32];
#pragma unroll
            for (int c = 0; c < 4; ++c)
                tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quarter * 32) << 16) + col_half * 128 + 32 * c, r[c]);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(tempty));  // accumulator free: next tile may start
            const int64_t row = (int64_t)tm * kBM + quarter * 32 + lane;
            if (row < M) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int64_t col0 = (int64_t)tn * kF8BN + col_half * 128 + 32 * c;
                    const int ncol = (int)imin64(32, (int64_t)N - col0);
                    float *cp = C + col0 * ldc + row;
                    if (ncol >= 32) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            float cv[16];
#pragma unroll
                            for (int j = 0; j < 16; ++j) cv[j] = __ldcs(cp + (16 * h + j) * ldc);
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                __stcs(cp + (16 * h + j) * ldc, cv[j] - __uint_as_float(r[c][16 * h + j]));
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < ncol) cp[j * ldc] = cp[j * ldc] - __uint_as_float(r[c][j]);
                    }
                }
            }
        }
        if (!ok && lane == 0) {
            *abort_flag = 1;
            report(dst, MXP_TIMEOUT, 6, blockIdx.x);
        }
    }

    __syncthreads();
    if (*abort_flag) {
        if (threadIdx.x == 0) {
            const unsigned long long t0 = globaltimer_ns();
            while (globaltimer_ns() - t0 < 50000ull) {
            }
        }
        __syncthreads();
    }
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

// ---- host side ---------------------------------------------------------------

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 2-D K-major map: dim0 = K (contiguous), dim1 = rows; box = box_k x box_rows.
mxp_status make_kmajor_map(CUtensorMap *map, CUtensorMapDataType dt, int esize, const void *base,
                           int64_t K, int64_t rows, int64_t ld, int box_k, int box_rows) {
    auto fn = get_encode_fn();
    if (!fn) return fail(MXP_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0)
        return fail(MXP_INVALID_ARG, "schur: panel base must be 16-byte aligned");
    if ((ld * esize) % 16 != 0) return fail(MXP_INVALID_ARG, "schur: panel ld*esize must be a multiple of 16");
    cuuint64_t gdim[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)(ld * esize)};
    cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, dt, 2, const_cast<void *>(base), gdim, gstride, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MXP_CUDA_ERROR, "cuTensorMapEncodeTiled failed");
    return MXP_OK;
}

mxp_status launch_schur2(int form, int m, int n, int k, const void *L, int64_t ldl, const uint8_t *lsc,
                         const void *R, int64_t ldr, const uint8_t *rsc, float *C, int64_t ldc,
                         DevStatus *dst, cudaStream_t st, int store, int lsc_ld, int rsc_ld, int tri_mode);

mxp_status launch_schur(int form, int m, int n, int k, const void *L, int64_t ldl,
                        const uint8_t *lsc, const void *R, int64_t ldr, const uint8_t *rsc,
                        float *C, int64_t ldc, DevStatus *dst, cudaStream_t st, int store,
                        int lsc_ld, int rsc_ld, int tri_mode, int pair, const SchurSched *sched,
                        const F8Out *f8out) {
    if (pair) {
        if (f8out && f8out->out) return fail(MXP_UNSUPPORTED, "schur: the FP8 copy is single-SM only");
        if (sched) return fail(MXP_UNSUPPORTED, "schur: tile schedules are single-SM only");
        return launch_schur2(form, m, n, k, L, ldl, lsc, R, ldr, rsc, C, ldc, dst, st, store, lsc_ld,
                             rsc_ld, tri_mode);
    }
    if (m < 0 || n < 0 || k < 0) return fail(MXP_INVALID_ARG, "schur: negative size");
    if (m == 0 || n == 0 || k == 0) return MXP_OK;
    if (ldc < m) return fail(MXP_INVALID_ARG, "schur: ldc < m");
    if (form != MXP_FORM_FP16 && form != MXP_FORM_BF16X2 && form != MXP_FORM_FP8 && form != kFormBf16)
        return fail(MXP_INVALID_ARG, "schur: unknown form");
    if (m > (1 << 30) || n > (1 << 30)) return fail(MXP_INVALID_ARG, "schur: size too large");
    const int64_t K = (form == MXP_FORM_BF16X2) ? 3 * (int64_t)k : k;
    if (ldl < K || ldr < K) return fail(MXP_INVALID_ARG, "schur: panel ld smaller than K");
    TileMap tiles;
    tiles.tiles_m = (int)cdiv(m, kBM);
    tiles.tiles_n = (int)cdiv(n, form == MXP_FORM_FP8 ? kF8BN : kBN);
    tiles.group_m = 16;
    const int64_t total = (int64_t)tiles.tiles_m * tiles.tiles_n;
    if (total > (int64_t)1 << 30) return fail(MXP_INVALID_ARG, "schur: too many tiles");
    const int bn = form == MXP_FORM_FP8 ? kF8BN : kBN;
    TileSrc src{nullptr, 0, 0};
    int grid = (int)(total < num_sms() ? total : num_sms());
    if (sched) {
        if (sched->grid < 0 || sched->skip_rows < 0 || sched->skip_cols < 0)
            return fail(MXP_INVALID_ARG, "schur: bad tile schedule");
        if (sched->skip_rows % kBM != 0 || sched->skip_cols % bn != 0)
            return fail(MXP_INVALID_ARG, "schur: skipped corner must be whole tiles");
        if (sched->grid > 0) grid = (int)imin64(grid, sched->grid);
        src.counter = sched->counter;
        src.skip_m = sched->skip_rows / kBM;
        src.skip_n = sched->skip_cols / bn;
    }
    CUtensorMap mapA, mapB;
    if (form == MXP_FORM_FP8) {
        if (!lsc || !rsc) return fail(MXP_INVALID_ARG, "schur: FP8 form needs both scale tables");
        if (store || tri_mode) return fail(MXP_UNSUPPORTED, "schur: store / triangular modes are FP16/BF16 only");
        mxp_status s = make_kmajor_map(&mapA, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L, K, m, ldl, 128, kBM);
        if (s != MXP_OK) return s;
        s = make_kmajor_map(&mapB, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, R, K, n, ldr, 128, kF8BN);
        if (s != MXP_OK) return s;
        static bool attr8 = false;
        if (!attr8) {
            MXP_CUDA(cudaFuncSetAttribute(schur_tc_fp8_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, kF8SmemBytes));
            attr8 = true;
        }
        const int kt = (int)cdiv(K, 128);
        schur_tc_fp8_kernel<<<grid, kThreads, kF8SmemBytes, st>>>(
            mapA, mapB, m, n, (int)K, lsc, rsc, lsc_ld > 0 ? lsc_ld : kt, rsc_ld > 0 ? rsc_ld : kt, C,
            ldc, tiles, src, dst);
        MXP_LAUNCHED();
        return MXP_OK;
    }
    const CUtensorMapDataType dt =
        form == MXP_FORM_FP16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    mxp_status s = make_kmajor_map(&mapA, dt, 2, L, K, m, ldl, 64, kBM);
    if (s != MXP_OK) return s;
    s = make_kmajor_map(&mapB, dt, 2, R, K, n, ldr, 64, kBN);
    if (s != MXP_OK) return s;
    static bool attr_done = false;
    if (!attr_done) {
        MXP_CUDA(cudaFuncSetAttribute(schur_tc_f16_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kSmemBytes));
        MXP_CUDA(cudaFuncSetAttribute(schur_tc_f16_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kSmemBytes));
        attr_done = true;
    }
    const uint32_t idesc = idesc_f16(form == MXP_FORM_FP16 ? 0u : 1u);
    // the triangular skip needs whole stages inside one K segment
    if (tri_mode != 0 && (k % 64 != 0)) tri_mode = 0;
    F8Out f8{nullptr, 0, nullptr, 0, 0};
    if (f8out && f8out->out) {
        if (!store || n % kBN != 0 || !f8out->sc ||
            (!f8out->trans && (f8out->ldk % 16 != 0 || (reinterpret_cast<uintptr_t>(f8out->out) & 15u))))
            return fail(MXP_INVALID_ARG, "schur: FP8 copy needs store mode, n % 256 == 0 and 16-byte rows");
        f8 = *f8out;
    }
    if (f8.out)
        schur_tc_f16_kernel<true><<<grid, kThreads, kSmemBytes, st>>>(mapA, mapB, m, n, (int)K, C, ldc, idesc,
                                                                      tiles, src, store, tri_mode, k, f8, dst);
    else
        schur_tc_f16_kernel<false><<<grid, kThreads, kSmemBytes, st>>>(mapA, mapB, m, n, (int)K, C, ldc, idesc,
                                                                       tiles, src, store, tri_mode, k, f8, dst);
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
