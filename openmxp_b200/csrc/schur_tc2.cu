// Schur update C -= L * R^T with the 2-SM tensor-core MMA (tcgen05 cta_group::2).
//
// Same operation and operand layout as schur_tc.cu (reference: the FP16
// gemm_ex Schur calls, panel_trf.hpp:661-665, 710-740, 828-834), with a pair
// of CTAs (a cluster of two, one per SM) cooperating on a 256 x 256 output
// tile: CTA r holds rows [128r, 128r+128) of the L tile and rows
// [128r, 128r+128) of the R tile in its own shared memory, the leader CTA
// (rank 0) issues tcgen05.mma.cta_group::2 (M = 256, N = 256), and each CTA's
// tensor memory receives its 128 rows of the accumulator.  Each SM thus
// stages half of the R operand instead of all of it, which is what limits
// the one-SM 128 x 256 kernel (shared-memory bandwidth: TMA writes plus MMA
// operand reads).
//
// Synchronisation (every load has a single destination): both CTAs' TMA loads complete
// bytes on the leader's full barrier (cp.async.bulk.tensor ... cta_group::2,
// barrier address mapped to rank 0 with mapa); the leader posts the
// expected byte count for both; the leader's MMA commits arrive on each
// CTA's empty / accumulator-full barriers with one unicast commit per CTA;
// both CTAs' epilogue warps arrive on the leader's accumulator-empty barrier
// (remote mbarrier.arrive for the peer).  All waits are bounded.
//
// FP8 (kind::mxf8f6f4.block_scale): each CTA writes the UE8M0 scale-factor
// atoms of its own L rows and of the whole R tile next to its stage; the
// leader copies them to tensor memory with tcgen05.cp.cta_group::2.
#include "tc_ptx.cuh"

namespace mxp {
namespace {

using namespace tc;

constexpr int kM2 = 256, kN2 = 256, kHalf = 128;
constexpr int kT2Epi = 8;
constexpr int kT2Threads = 64 + 32 * kT2Epi;
constexpr int kT2TmemCols = 512;

template <bool FP8>
struct Cfg2 {
    static constexpr int kStageA = kHalf * 128;  // 128 rows x 128 bytes of K
    static constexpr int kStageB = kHalf * 128;  // this CTA's half of the R tile
    static constexpr int kStageSF = FP8 ? 2048 : 0;
    static constexpr int kStageBytes = kStageA + kStageB + kStageSF;
    static constexpr int kStages = 6;
    static constexpr int kSmem = 1024 + kStages * kStageBytes + 512;
    static constexpr int kKPerStage = FP8 ? 128 : 64;
    static constexpr int kAccBufs = FP8 ? 1 : 2;
    static constexpr int kSfCol0 = 256;
};

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, int x, int y,
                                                 uint32_t bar_cluster) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
        : "memory");
}

__device__ __forceinline__ void tc_commit_pair(uint32_t bar_cluster) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_cluster)
                 : "memory");
}

__device__ __forceinline__ void tc_mma_f16_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                                uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_mma_mxf8_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                                 uint32_t sfa, uint32_t sfb, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::mxf8f6f4.block_scale [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(sfa), "r"(sfb)
        : "memory");
}

__device__ __forceinline__ void tc_cp_pair(uint32_t taddr, uint64_t sdesc) {
    asm volatile("tcgen05.cp.cta_group::2.32x128b.warpx4 [%0], %1;" ::"r"(taddr), "l"(sdesc) : "memory");
}

__device__ __forceinline__ uint64_t smem_desc_sf32(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(128 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__host__ __device__ constexpr uint32_t idesc_mxf8_mn(uint32_t sf_id, int M, int N) {
    return (sf_id << 4) | ((uint32_t)(N >> 3) << 17) | (1u << 23) | ((uint32_t)(M >> 4) << 24) |
           (sf_id << 29);
}

struct TileMap2 {
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

template <bool FP8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kT2Threads, 1)
schur_tc2_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M,
                 int N, int K, const uint8_t *__restrict__ lsc, const uint8_t *__restrict__ rsc, int lsc_ld,
                 int rsc_ld, float *__restrict__ C, int64_t ldc, uint32_t idesc_f16, TileMap2 tiles,
                 int store, int tri_mode, int seg, DevStatus *dst) {
    using Cfg = Cfg2<FP8>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + Cfg::kStages * Cfg::kStageBytes);
    uint64_t *full = bars;
    uint64_t *empty = bars + Cfg::kStages;
    uint64_t *tfull = bars + 2 * Cfg::kStages;
    uint64_t *tempty = bars + 2 * Cfg::kStages + 2;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + 2 * Cfg::kStages + 4);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);
    auto stA = [&](int s) { return smem + s * Cfg::kStageBytes; };
    auto stB = [&](int s) { return smem + s * Cfg::kStageBytes + Cfg::kStageA; };
    auto stSF = [&](int s) { return smem + s * Cfg::kStageBytes + Cfg::kStageA + Cfg::kStageB; };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const bool leader = rank == 0;
    const int cluster = blockIdx.x >> 1, nclusters = gridDim.x >> 1;
    const int total_tiles = tiles.tiles_m * tiles.tiles_n;
    const int nk = (K + Cfg::kKPerStage - 1) / Cfg::kKPerStage;
    const int rtiles = (N + 127) / 128;
    // needed K stages: the first stage_count of each segment of seg_st stages
    // (walked with a position counter, no per-stage modulo)
    const int seg_st = tri_mode ? seg / Cfg::kKPerStage : nk;
    auto stage_count = [&](int tm, int tn) -> int {
        if (tri_mode == 0) return nk;
        return min(seg_st, (tri_mode == 1 ? (tn + 1) * kN2 : (tm + 1) * kM2) / Cfg::kKPerStage);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cfg::kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&tfull[a]), 1);
            mbar_init(smem_u32(&tempty[a]), 2 * kT2Epi);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_holder)),
                     "r"(kT2TmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;

    if (warp == 0) {
        // ---------------- producer (both CTAs) ----------------
        int stage = 0;
        uint32_t phase = 0;
        bool ok = true;
        for (int t = cluster; t < total_tiles && ok; t += nclusters) {
            int tm, tn;
            tiles.get(t, tm, tn);
            const int cnt = stage_count(tm, tn);
            int pos = -1;
            for (int kb = 0; kb < nk; ++kb) {
                if (++pos == seg_st) pos = 0;
                if (pos >= cnt) {
                    kb += seg_st - 1 - pos;
                    pos = seg_st - 1;
                    continue;
                }
                int got = 1;
                if (lane == 0) got = mbar_wait(smem_u32(&empty[stage]), phase ^ 1u, abort_flag) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                if (FP8) {
                    const int arow = 2 * tm + (int)rank;  // this CTA's 128-row scale tile of L
                    const uint32_t sa = lsc[(int64_t)arow * lsc_ld + kb];
                    const uint32_t sb0 = rsc[(int64_t)(2 * tn) * rsc_ld + kb];
                    const uint32_t sb1 = (2 * tn + 1 < rtiles) ? rsc[(int64_t)(2 * tn + 1) * rsc_ld + kb] : 127u;
                    const uint32_t wa = sa * 0x01010101u, wb0 = sb0 * 0x01010101u, wb1 = sb1 * 0x01010101u;
                    uint4 *sf = reinterpret_cast<uint4 *>(stSF(stage));
                    sf[lane] = make_uint4(wa, wa, wa, wa);
                    sf[32 + lane] = make_uint4(wb0, wb0, wb0, wb0);
                    sf[64 + lane] = make_uint4(wb1, wb1, wb1, wb1);
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                }
                if (lane == 0) {
                    const uint32_t fb = smem_u32(&full[stage]);
                    if (leader) mbar_expect_tx(fb, 2 * (Cfg::kStageA + Cfg::kStageB));
                    const uint32_t fb0 = mapa_shared(fb, 0);
                    tma_load_2d_pair(smem_u32(stA(stage)), &tmA, kb * Cfg::kKPerStage, tm * kM2 + (int)rank * kHalf, fb0);
                    tma_load_2d_pair(smem_u32(stB(stage)), &tmB, kb * Cfg::kKPerStage, tn * kN2 + (int)rank * kHalf, fb0);
                }
                if (++stage == Cfg::kStages) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
        }
        if (!ok && lane == 0) {
            *abort_flag = 1;
            report(dst, MXP_TIMEOUT, 21, blockIdx.x);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (leader CTA, one lane) ----------------
        if (leader && lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t it = 0;
            bool ok = true;
            for (int t = cluster; t < total_tiles && ok; t += nclusters, ++it) {
                int tm, tn;
                tiles.get(t, tm, tn);
                const uint32_t acc = (Cfg::kAccBufs == 2) ? (it & 1u) : 0u;
                const uint32_t use = (Cfg::kAccBufs == 2) ? (it >> 1) : it;
                if (!mbar_wait(smem_u32(&tempty[acc]), (use & 1u) ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + acc * kN2;
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
                    const uint32_t a0 = smem_u32(stA(stage));
                    const uint32_t b0 = smem_u32(stB(stage));
                    if (FP8) {
                        const uint32_t sfa_t = tmem_base + Cfg::kSfCol0 + 16u * stage;
                        const uint32_t sfb_t = sfa_t + 4u;
                        const uint32_t sf0 = smem_u32(stSF(stage));
                        tc_cp_pair(sfa_t, smem_desc_sf32(sf0));
                        tc_cp_pair(sfb_t, smem_desc_sf32(sf0 + 512));
                        tc_cp_pair(sfb_t + 4u, smem_desc_sf32(sf0 + 1024));
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            tc_mma_mxf8_pair(d_tmem, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k),
                                             idesc_mxf8_mn((uint32_t)k, kM2, kN2), sfa_t, sfb_t,
                                             (!first || k > 0) ? 1u : 0u);
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            tc_mma_f16_pair(d_tmem, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k),
                                            idesc_f16, (!first || k > 0) ? 1u : 0u);
                    }
                    first = false;
                    const uint32_t eb = smem_u32(&empty[stage]);
                    tc_commit_pair(mapa_shared(eb, 0));
                    tc_commit_pair(mapa_shared(eb, 1));
                    if (++stage == Cfg::kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                const uint32_t fb = smem_u32(&tfull[acc]);
                tc_commit_pair(mapa_shared(fb, 0));
                tc_commit_pair(mapa_shared(fb, 1));
            }
            if (!ok) {
                *abort_flag = 1;
                report(dst, MXP_TIMEOUT, 22, blockIdx.x);
            }
        }
    } else {
        // ---------------- epilogue (both CTAs) ----------------
        const int ew = warp - 2;
        const int quarter = warp & 3;
        const int col_half = ew >> 2;
        uint32_t it = 0;
        bool ok = true;
        for (int t = cluster; t < total_tiles; t += nclusters, ++it) {
            int tm, tn;
            tiles.get(t, tm, tn);
            const uint32_t acc = (Cfg::kAccBufs == 2) ? (it & 1u) : 0u;
            const uint32_t use = (Cfg::kAccBufs == 2) ? (it >> 1) : it;
            if (!mbar_wait(smem_u32(&tfull[acc]), use & 1u, abort_flag)) {
                ok = false;
                break;
            }
            __syncwarp();
            tc_fence_after();
            const int64_t row = (int64_t)tm * kM2 + (int)rank * kHalf + quarter * 32 + lane;
            const bool row_ok = row < M;
            const uint32_t tbase = tmem_base + ((uint32_t)(quarter * 32) << 16) + acc * kN2 + col_half * 128;
            const uint32_t tempty0 = mapa_shared(smem_u32(&tempty[acc]), 0);
            if (FP8) {
                uint32_t r[4][32];
#pragma unroll
                for (int c = 0; c < 4; ++c) tmem_ld_32x32b_x32(tbase + 32 * c, r[c]);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(tempty0);
                if (row_ok) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int64_t col0 = (int64_t)tn * kN2 + col_half * 128 + 32 * c;
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
            } else {
#pragma unroll 1
                for (int c = 0; c < 4; ++c) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tbase + 32 * c, r);
                    const int64_t col0 = (int64_t)tn * kN2 + col_half * 128 + 32 * c;
                    if (row_ok) {
                        float *cp = C + col0 * ldc + row;
                        const int ncol = (int)imin64(32, (int64_t)N - col0);
                        if (store) {  // C = acc, or C = -acc (store == 2)
                            const float sg = store == 2 ? -1.0f : 1.0f;
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (j < ncol) __stcs(cp + j * ldc, sg * __uint_as_float(r[j]));
                        } else if (ncol >= 32) {
                            float cv[32];
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
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(tempty0);
            }
        }
        if (!ok && lane == 0) {
            *abort_flag = 1;
            report(dst, MXP_TIMEOUT, 23, blockIdx.x);
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
    cluster_sync();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kT2TmemCols)
                     : "memory");
    }
}

}  // namespace

mxp_status make_kmajor_map(CUtensorMap *map, CUtensorMapDataType dt, int esize, const void *base,
                           int64_t K, int64_t rows, int64_t ld, int box_k, int box_rows);

// 2-SM variant of launch_schur (same arguments and semantics).
mxp_status launch_schur2(int form, int m, int n, int k, const void *L, int64_t ldl, const uint8_t *lsc,
                         const void *R, int64_t ldr, const uint8_t *rsc, float *C, int64_t ldc,
                         DevStatus *dst, cudaStream_t st, int store, int lsc_ld, int rsc_ld, int tri_mode) {
    if (m < 0 || n < 0 || k < 0) return fail(MXP_INVALID_ARG, "schur: negative size");
    if (m == 0 || n == 0 || k == 0) return MXP_OK;
    if (ldc < m) return fail(MXP_INVALID_ARG, "schur: ldc < m");
    const bool fp8 = form == MXP_FORM_FP8;
    const int64_t K = (form == MXP_FORM_BF16X2) ? 3 * (int64_t)k : k;
    if (ldl < K || ldr < K) return fail(MXP_INVALID_ARG, "schur: panel ld smaller than K");
    if (fp8 && (!lsc || !rsc)) return fail(MXP_INVALID_ARG, "schur: FP8 form needs both scale tables");
    if (fp8 && (store || tri_mode)) return fail(MXP_UNSUPPORTED, "schur: store / triangular modes are FP16/BF16 only");
    TileMap2 tiles;
    tiles.tiles_m = (int)cdiv(m, kM2);
    tiles.tiles_n = (int)cdiv(n, kN2);
    tiles.group_m = 8;
    const int64_t total = (int64_t)tiles.tiles_m * tiles.tiles_n;
    if (total > (int64_t)1 << 30) return fail(MXP_INVALID_ARG, "schur: too many tiles");
    const int pairs = (int)imin64(total, num_sms() / 2);
    const int grid = 2 * pairs;
    CUtensorMap mapA, mapB;
    const CUtensorMapDataType dt = fp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                       : (form == MXP_FORM_FP16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16);
    const int es = fp8 ? 1 : 2;
    const int boxk = fp8 ? 128 : 64;
    mxp_status s = make_kmajor_map(&mapA, dt, es, L, K, m, ldl, boxk, kHalf);
    if (s != MXP_OK) return s;
    s = make_kmajor_map(&mapB, dt, es, R, K, n, ldr, boxk, kHalf);
    if (s != MXP_OK) return s;
    if (tri_mode != 0 && (k % boxk != 0)) tri_mode = 0;
    const int kt = (int)cdiv(K, 128);
    if (fp8) {
        static bool attr = false;
        if (!attr) {
            MXP_CUDA(cudaFuncSetAttribute(schur_tc2_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          Cfg2<true>::kSmem));
            attr = true;
        }
        schur_tc2_kernel<true><<<grid, kT2Threads, Cfg2<true>::kSmem, st>>>(
            mapA, mapB, m, n, (int)K, lsc, rsc, lsc_ld > 0 ? lsc_ld : kt, rsc_ld > 0 ? rsc_ld : kt, C, ldc, 0u,
            tiles, 0, 0, k, dst);
    } else {
        static bool attr = false;
        if (!attr) {
            MXP_CUDA(cudaFuncSetAttribute(schur_tc2_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          Cfg2<false>::kSmem));
            attr = true;
        }
        const uint32_t idesc = idesc_f16_mn(form == MXP_FORM_FP16 ? 0u : 1u, kM2, kN2);
        schur_tc2_kernel<false><<<grid, kT2Threads, Cfg2<false>::kSmem, st>>>(
            mapA, mapB, m, n, (int)K, nullptr, nullptr, 0, 0, C, ldc, idesc, tiles, store, tri_mode, k, dst);
    }
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
