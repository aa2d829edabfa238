// FP32 -> low-precision panel casts.
//
// Reference: convert_left_panels_wGPU / convert_right_panels_wGPU
// (panel_trf.hpp:258-277, 305-325) with copyCoalesced / transposeCoalesced
// (fp16_gpu_kernels.cpp:11-36, 158-211).  The reference writes the L panel
// column-major and the U panel transposed (R = U^T, column-major) for a
// library GEMM with OP_N, OP_T.  Here the panels are written K-major (row i
// of the panel holds its b values contiguously), the layout the TMA-fed
// tcgen05 Schur kernel reads with 128-byte swizzle.  The reference layouts
// are also provided (mxp_half_conversion_left / _right_trans) as drop-ins.
//
// Forms:
//   FP16    : round to nearest even (__float2half_rn), as the reference.
//   BF16X2  : hi = bf16(x), lo = bf16(x - hi); the K-major row is laid out
//             as three K segments (left: hi|hi|lo, right: hi|lo|hi) so one
//             GEMM with K' = 3b accumulates hi*hi + hi*lo + lo*hi.
//   BF16    : (internal, kFormBf16) bf16(x) only, K = b: the operands of the
//             single-product TRSM by inverse.
//   FP8     : E4M3 (satfinite) of x * 2^e with one power-of-two scale per
//             128 x 128 tile of the panel, e the largest exponent keeping the
//             tile's amax <= 448; the UE8M0 byte 127 - e (value 2^-e) is
//             stored per tile for the block-scaled MMA.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "fp8_quant.cuh"

#include "mxp_internal.cuh"

namespace mxp {

namespace {

constexpr int kTile = 64;
constexpr int kCastThreads = 256;

template <int FORM>
__device__ __forceinline__ void store_lowp(void *out, int64_t ldk, int64_t row, int k, int b,
                                           float x, bool is_right) {
    if (FORM == MXP_FORM_FP16) {
        reinterpret_cast<__half *>(out)[row * ldk + k] = __float2half_rn(x);
    } else if (FORM == kFormBf16) {
        reinterpret_cast<__nv_bfloat16 *>(out)[row * ldk + k] = __float2bfloat16_rn(x);
    } else {  // BF16X2
        __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(out) + row * ldk;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(x, __bfloat162float(hi)));
        o[k] = hi;
        o[b + k] = is_right ? lo : hi;
        o[2 * b + k] = is_right ? hi : lo;
    }
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t pack_bf2(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// 8 consecutive k of one row as one 16-byte store per K segment (requires the
// row start, k0 and b to keep every segment 16-byte aligned; checked by the
// launcher).
template <int FORM>
__device__ __forceinline__ void store8(void *out, int64_t ldk, int64_t row, int k0, int b,
                                       const float *v, bool is_right) {
    if (FORM == MXP_FORM_FP16) {
        uint4 w = make_uint4(pack_h2(v[0], v[1]), pack_h2(v[2], v[3]), pack_h2(v[4], v[5]),
                             pack_h2(v[6], v[7]));
        *reinterpret_cast<uint4 *>(reinterpret_cast<__half *>(out) + row * ldk + k0) = w;
    } else if (FORM == kFormBf16) {
        __nv_bfloat16 h[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16_rn(v[q]);
        *reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) + row * ldk + k0) =
            make_uint4(pack_bf2(h[0], h[1]), pack_bf2(h[2], h[3]), pack_bf2(h[4], h[5]), pack_bf2(h[6], h[7]));
    } else {
        __nv_bfloat16 hi[8], lo[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            hi[q] = __float2bfloat16_rn(v[q]);
            lo[q] = __float2bfloat16_rn(__fsub_rn(v[q], __bfloat162float(hi[q])));
        }
        const uint4 H = make_uint4(pack_bf2(hi[0], hi[1]), pack_bf2(hi[2], hi[3]), pack_bf2(hi[4], hi[5]),
                                   pack_bf2(hi[6], hi[7]));
        const uint4 Lw = make_uint4(pack_bf2(lo[0], lo[1]), pack_bf2(lo[2], lo[3]), pack_bf2(lo[4], lo[5]),
                                    pack_bf2(lo[6], lo[7]));
        __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(out) + row * ldk + k0;
        *reinterpret_cast<uint4 *>(o) = H;
        *reinterpret_cast<uint4 *>(o + b) = is_right ? Lw : H;
        *reinterpret_cast<uint4 *>(o + 2 * b) = is_right ? H : Lw;
    }
}

template <int FORM>
__device__ __forceinline__ void store16(void *out, int64_t ldk, int64_t row, int k0, int b,
                                        const float *v, bool is_right) {
    store8<FORM>(out, ldk, row, k0, b, v, is_right);
    store8<FORM>(out, ldk, row, k0 + 8, b, v + 8, is_right);
}

// L column panel: FP32 m x b column-major -> K-major rows (transpose through
// shared memory: reads coalesced along rows, writes coalesced along k).
template <int FORM>
__global__ void __launch_bounds__(kCastThreads)
cast_left_kernel(int m, int b, const float *__restrict__ A, int64_t lda, void *out, int64_t ldk,
                 bool vec) {
    __shared__ float tile[kTile][kTile + 1];
    const int i0 = blockIdx.x * kTile;
    const int k0 = blockIdx.y * kTile;
    const int t = threadIdx.x;
    const int ii = t % kTile;
#pragma unroll
    for (int q = 0; q < kTile * kTile / kCastThreads; ++q) {
        const int kk = t / kTile + q * (kCastThreads / kTile);
        const int i = i0 + ii, k = k0 + kk;
        tile[kk][ii] = (i < m && k < b) ? A[(int64_t)k * lda + i] : 0.0f;
    }
    __syncthreads();
    const int ri = t / 4;          // row within tile
    const int kc = (t % 4) * 16;   // 16 k per thread
    const int64_t row = i0 + ri;
    if (row >= m) return;
    if (vec && k0 + kc + 16 <= b) {
        float v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = tile[kc + q][ri];
        store16<FORM>(out, ldk, row, k0 + kc, b, v, false);
        return;
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int k = k0 + kc + q;
        if (k < b) store_lowp<FORM>(out, ldk, row, k, b, tile[kc + q][ri], false);
    }
}

// U row panel: FP32 b x m column-major (element (k, j) at A[k + j*lda]) ->
// K-major rows j (= U^T).  No transpose: column j of U is already contiguous
// in k.
template <int FORM>
__global__ void __launch_bounds__(kCastThreads)
cast_right_kernel(int m, int b, const float *__restrict__ A, int64_t lda, void *out, int64_t ldk,
                  bool vec, bool vec_in) {
    const int64_t gid = (int64_t)blockIdx.x * kCastThreads + threadIdx.x;
    const int kchunks = (b + 7) / 8;
    const int64_t j = gid / kchunks;
    const int k0 = (int)(gid % kchunks) * 8;
    if (j >= m) return;
    const float *src = A + j * lda;
    if (vec && k0 + 8 <= b) {
        float v[8];
        if (vec_in) {  // two 16-byte loads (column start 16-byte aligned, k0 % 8 == 0)
            const float4 a = *reinterpret_cast<const float4 *>(src + k0);
            const float4 c = *reinterpret_cast<const float4 *>(src + k0 + 4);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
            v[4] = c.x; v[5] = c.y; v[6] = c.z; v[7] = c.w;
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = src[k0 + q];
        }
        store8<FORM>(out, ldk, j, k0, b, v, true);
        return;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = k0 + q;
        if (k < b) store_lowp<FORM>(out, ldk, j, k, b, src[k], true);
    }
}

// ---- FP8 E4M3 with per-128x128-tile power-of-two scales -----------------

// e4m3_scale_exp, e4m3_scale_up and to_e4m3: fp8_quant.cuh

__device__ __forceinline__ float block_max_256(float v, float *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float r = red[0];
#pragma unroll
    for (int w = 1; w < kCastThreads / 32; ++w) r = fmaxf(r, red[w]);
    return r;
}

constexpr int kF8Tile = 128;

// L panel, FP8: one CTA per 128 (rows) x 128 (k) tile.
__global__ void __launch_bounds__(kCastThreads)
cast_left_fp8_kernel(int m, int b, const float *__restrict__ A, int64_t lda, uint8_t *out,
                     int64_t ldk, uint8_t *scales, int sc_ld) {
    __shared__ uint32_t tile[kF8Tile][kF8Tile / 4 + 1];
    __shared__ float red[kCastThreads / 32];
    const int i0 = blockIdx.x * kF8Tile, k0 = blockIdx.y * kF8Tile;
    const int t = threadIdx.x;
    const int ii = t % kF8Tile, kh = t / kF8Tile;  // kh in {0,1}: 64 k each
    float v[64];
    float amax = 0.0f;
    const int i = i0 + ii;
#pragma unroll
    for (int q = 0; q < 64; ++q) {
        const int k = k0 + kh * 64 + q;
        v[q] = (i < m && k < b) ? A[(int64_t)k * lda + i] : 0.0f;
        amax = fmaxf(amax, fabsf(v[q]));
    }
    amax = block_max_256(amax, red);
    const int e = e4m3_scale_exp(amax);
    const float up = e4m3_scale_up(e);
#pragma unroll
    for (int q = 0; q < 64; q += 4) {
        uint32_t w = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) w |= (uint32_t)to_e4m3(__fmul_rn(v[q + r], up)) << (8 * r);
        tile[ii][(kh * 64 + q) / 4] = w;
    }
    if (t == 0) scales[(int64_t)blockIdx.x * sc_ld + blockIdx.y] = (uint8_t)(127 - e);
    __syncthreads();
    // write out: row ri = t / 2, 64 bytes (16 words) per thread
    const int ri = t / 2, half = t % 2;
    const int64_t row = i0 + ri;
    if (row >= m) return;
    uint8_t *dst = out + row * ldk + k0 + half * 64;
    const int kvalid = min(64, b - (k0 + half * 64));
    if (kvalid <= 0) return;
    if (kvalid == 64) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 w;
            w.x = tile[ri][half * 16 + 4 * q + 0];
            w.y = tile[ri][half * 16 + 4 * q + 1];
            w.z = tile[ri][half * 16 + 4 * q + 2];
            w.w = tile[ri][half * 16 + 4 * q + 3];
            reinterpret_cast<uint4 *>(dst)[q] = w;
        }
    } else {
        for (int q = 0; q < kvalid; ++q)
            dst[q] = (uint8_t)(tile[ri][(half * 64 + q) / 4] >> (8 * (q % 4)));
    }
}

// R panel (U^T rows), FP8: one CTA per 128 (rows j) x 128 (k) tile.  Column j
// of U holds the 128 k of the tile contiguously, and so does row j of R: warp
// w takes the 16 columns j0 + 16w .. +15, reading each as one 512-byte float4
// load across its lanes (lane l: k = 4l .. 4l+3) and writing it as one
// 128-byte row of E4M3 (one 32-bit word per lane).  vec4: A and lda keep
// every column start 16-byte aligned and out rows 4-byte aligned.
__global__ void __launch_bounds__(kCastThreads)
cast_right_fp8_kernel(int m, int b, const float *__restrict__ A, int64_t lda, uint8_t *out,
                      int64_t ldk, uint8_t *scales, int sc_ld, bool vec4) {
    __shared__ float red[kCastThreads / 32];
    const int j0 = blockIdx.x * kF8Tile, k0 = blockIdx.y * kF8Tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kl = k0 + 4 * lane;  // first of this lane's 4 k
    float4 v[16];
    float amax = 0.0f;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        const int64_t j = j0 + 16 * warp + c;
        const float *src = A + j * lda + kl;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < m) {
            if (vec4 && kl + 4 <= b) {
                x = *reinterpret_cast<const float4 *>(src);
            } else {
                if (kl + 0 < b) x.x = src[0];
                if (kl + 1 < b) x.y = src[1];
                if (kl + 2 < b) x.z = src[2];
                if (kl + 3 < b) x.w = src[3];
            }
        }
        v[c] = x;
        amax = fmaxf(amax, fmaxf(fmaxf(fabsf(x.x), fabsf(x.y)), fmaxf(fabsf(x.z), fabsf(x.w))));
    }
    amax = block_max_256(amax, red);
    const int e = e4m3_scale_exp(amax);
    const float up = e4m3_scale_up(e);
    if (threadIdx.x == 0) scales[(int64_t)blockIdx.x * sc_ld + blockIdx.y] = (uint8_t)(127 - e);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        const int64_t j = j0 + 16 * warp + c;
        if (j >= m || kl >= b) continue;
        const float4 x = v[c];
        const uint32_t w = (uint32_t)to_e4m3(__fmul_rn(x.x, up)) | ((uint32_t)to_e4m3(__fmul_rn(x.y, up)) << 8) |
                           ((uint32_t)to_e4m3(__fmul_rn(x.z, up)) << 16) |
                           ((uint32_t)to_e4m3(__fmul_rn(x.w, up)) << 24);
        uint8_t *dst = out + j * ldk + kl;
        if (vec4 && kl + 4 <= b) {
            *reinterpret_cast<uint32_t *>(dst) = w;
        } else {
            for (int q = 0; q < 4 && kl + q < b; ++q) dst[q] = (uint8_t)(w >> (8 * q));
        }
    }
}

// ---- reference layouts (bit-exact drop-ins) --------------------------------

__global__ void half_left_ref_kernel(const float *__restrict__ C, int m, int b, int64_t plda,
                                     __half *lp, int64_t lplda) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t k = blockIdx.y;
    if (i < m && k < b) lp[k * lplda + i] = __float2half_rn(C[k * plda + i]);
}

__global__ void __launch_bounds__(kCastThreads)
half_right_trans_ref_kernel(const float *__restrict__ C, int b, int m, int64_t plda, __half *rp,
                            int64_t rplda) {
    __shared__ float tile[kTile][kTile + 1];
    const int k0 = blockIdx.x * kTile;  // rows of the U block (K)
    const int j0 = blockIdx.y * kTile;  // columns of the U block
    const int t = threadIdx.x;
    const int x = t % kTile;
#pragma unroll
    for (int q = 0; q < kTile * kTile / kCastThreads; ++q) {
        const int y = t / kTile + q * (kCastThreads / kTile);
        const int k = k0 + x, j = j0 + y;
        tile[y][x] = (k < b && j < m) ? C[(int64_t)j * plda + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kTile * kTile / kCastThreads; ++q) {
        const int y = t / kTile + q * (kCastThreads / kTile);
        const int j = j0 + x, k = k0 + y;
        if (k < b && j < m) rp[(int64_t)k * rplda + j] = __float2half_rn(tile[x][y]);
    }
}

}  // namespace

// 16-byte stores need a 16-byte aligned base, row stride and segment offset.
static bool vec_ok(const void *out, int64_t ldk, int b) {
    return (reinterpret_cast<uintptr_t>(out) % 16 == 0) && (ldk % 8 == 0) && (b % 8 == 0);
}

static mxp_status check_cast_args(int form, int m, int b, int64_t lda, int64_t ldk) {
    if (m < 0 || b <= 0) return fail(MXP_INVALID_ARG, "panel cast: bad m/b");
    if (lda < 1) return fail(MXP_INVALID_ARG, "panel cast: bad lda");
    const int64_t K = (form == MXP_FORM_BF16X2) ? 3 * (int64_t)b : b;
    if (ldk < K) return fail(MXP_INVALID_ARG, "panel cast: ldk smaller than the K extent");
    if (form != MXP_FORM_FP16 && form != MXP_FORM_BF16X2 && form != MXP_FORM_FP8 && form != kFormBf16)
        return fail(MXP_INVALID_ARG, "panel cast: unknown form");
    return MXP_OK;
}

mxp_status launch_cast_left(int form, int m, int b, const float *A, int64_t lda, void *out,
                            int64_t ldk, uint8_t *scales, cudaStream_t st, int sc_ld) {
    mxp_status s = check_cast_args(form, m, b, lda, ldk);
    if (s != MXP_OK) return s;
    if (m == 0) return MXP_OK;
    if (form == MXP_FORM_FP8) {
        if (!scales) return fail(MXP_INVALID_ARG, "FP8 cast needs a scale buffer");
        dim3 grid((unsigned)cdiv(m, kF8Tile), (unsigned)cdiv(b, kF8Tile));
        cast_left_fp8_kernel<<<grid, kCastThreads, 0, st>>>(m, b, A, lda, (uint8_t *)out, ldk,
                                                            scales, sc_ld > 0 ? sc_ld : (int)grid.y);
    } else {
        const bool vec = vec_ok(out, ldk, b);
        dim3 grid((unsigned)cdiv(m, kTile), (unsigned)cdiv(b, kTile));
        if (form == MXP_FORM_FP16)
            cast_left_kernel<MXP_FORM_FP16><<<grid, kCastThreads, 0, st>>>(m, b, A, lda, out, ldk, vec);
        else if (form == kFormBf16)
            cast_left_kernel<kFormBf16><<<grid, kCastThreads, 0, st>>>(m, b, A, lda, out, ldk, vec);
        else
            cast_left_kernel<MXP_FORM_BF16X2><<<grid, kCastThreads, 0, st>>>(m, b, A, lda, out, ldk, vec);
    }
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_cast_right(int form, int m, int b, const float *A, int64_t lda, void *out,
                             int64_t ldk, uint8_t *scales, cudaStream_t st, int sc_ld) {
    mxp_status s = check_cast_args(form, m, b, lda, ldk);
    if (s != MXP_OK) return s;
    if (m == 0) return MXP_OK;
    if (form == MXP_FORM_FP8) {
        if (!scales) return fail(MXP_INVALID_ARG, "FP8 cast needs a scale buffer");
        dim3 grid((unsigned)cdiv(m, kF8Tile), (unsigned)cdiv(b, kF8Tile));
        const bool vec4 = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (lda % 4 == 0) &&
                          (reinterpret_cast<uintptr_t>(out) % 4 == 0) && (ldk % 4 == 0);
        cast_right_fp8_kernel<<<grid, kCastThreads, 0, st>>>(m, b, A, lda, (uint8_t *)out, ldk,
                                                             scales, sc_ld > 0 ? sc_ld : (int)grid.y, vec4);
    } else {
        const bool vec = vec_ok(out, ldk, b);
        const bool vec_in = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (lda % 4 == 0);
        const int64_t threads = (int64_t)m * ((b + 7) / 8);
        const unsigned blocks = (unsigned)cdiv(threads, kCastThreads);
        if (form == MXP_FORM_FP16)
            cast_right_kernel<MXP_FORM_FP16><<<blocks, kCastThreads, 0, st>>>(m, b, A, lda, out, ldk, vec,
                                                                              vec_in);
        else if (form == kFormBf16)
            cast_right_kernel<kFormBf16><<<blocks, kCastThreads, 0, st>>>(m, b, A, lda, out, ldk, vec, vec_in);
        else
            cast_right_kernel<MXP_FORM_BF16X2><<<blocks, kCastThreads, 0, st>>>(m, b, A, lda, out,
                                                                                 ldk, vec, vec_in);
    }
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_half_left_ref(const float *C, int m, int b, int64_t plda, uint16_t *lp,
                                int64_t lplda, cudaStream_t st) {
    if (m < 0 || b < 0 || plda < m || lplda < m) return fail(MXP_INVALID_ARG, "half_conversion_left: bad sizes");
    if (m == 0 || b == 0) return MXP_OK;
    dim3 grid((unsigned)cdiv(m, 256), (unsigned)b);
    half_left_ref_kernel<<<grid, 256, 0, st>>>(C, m, b, plda, reinterpret_cast<__half *>(lp), lplda);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_half_right_trans_ref(const float *C, int b, int m, int64_t plda, uint16_t *rp,
                                       int64_t rplda, cudaStream_t st) {
    if (m < 0 || b < 0 || plda < b || rplda < m)
        return fail(MXP_INVALID_ARG, "half_conversion_right_trans: bad sizes");
    if (m == 0 || b == 0) return MXP_OK;
    dim3 grid((unsigned)cdiv(b, kTile), (unsigned)cdiv(m, kTile));
    half_right_trans_ref_kernel<<<grid, kCastThreads, 0, st>>>(C, b, m, plda,
                                                               reinterpret_cast<__half *>(rp), rplda);
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
