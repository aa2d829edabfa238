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
    union {
        float t[kNB][kNB + 4];   // t[col][row] of a 64 x 64 block (16-byte rows)
        float ub[kNB][kNB + 1];  // staging of 64 U-strip columns, ub[col][row] (t is dead by then)
    };
    float us[kNB][kNB];      // us[k][c] = U(k, k + 1 + c): row k of U right of the diagonal, zero past the block
    float ls[kNB][kNB];      // ls[k][c] = L(k + 1 + c, k): column k of L below the diagonal, zero past the block
    float dinv[kNB];
    int ready[32];           // 64 x 64 factor: multipliers of pivot k published (getrf64)
};
struct __align__(16) SmemG64 {  // one 64 x 64 x 64 product staged whole
    float As[kNB][kNB];       // As[k][row]
    float Bs[kNB][kNB + 4];   // Bs[k][col]
};
union __align__(16) Smem {
    SmemGemm g;
    SmemTri t;
    SmemG64 g64;
};

// A 64 x 64 block (rows r < nb, columns c < nb; zero elsewhere) from global
// memory through L2 into registers: 16 values per thread, element q at
// column (threadIdx.x + 256 q) / 64, row (threadIdx.x + 256 q) % 64.  All 16
// loads are issued before any is used, so the block costs one L2 round trip.
static_assert(kCT * 16 == kNB * kNB, "64 x 64 block = 16 values per thread");
template <int N>
__device__ __forceinline__ void load_block64(float (&v)[N], const float *D, int64_t ld, int nr, int nc) {
    static_assert(N >= 16, "16 values per thread");
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int idx = threadIdx.x + kCT * q;
        const int r = idx % kNB, c = idx / kNB;
        v[q] = (r < nr && c < nc) ? __ldcg(D + (int64_t)c * ld + r) : 0.0f;
    }
}

// One pivot of a right-looking elimination on a row held in registers that
// moves left by one column per pivot: x[c] = x[c + 1] - s[c] * v for c < W - 1,
// x[W - 1] = 0.  With x[0] the pivot column and s the pivot row (or column)
// right of the diagonal, this is x_j -= s_j v for j > k in the same operation
// (one fmaf) as the unrotated loop, but every pivot runs the same code, so the
// pivot loop stays rolled: fully unrolled 64-pivot eliminations are thousands
// of straight-line instructions, and their instruction fetch, not the FMA
// pipe, set their speed (~8-10 cycles per instruction in a per-step trace).
// W (the live width, 64 - 16 p in phase p of a 64-wide elimination) skips the
// columns the rotation has already emptied.  s is 16-byte aligned.
template <int W>
__device__ __forceinline__ void rot_axpy(float (&x)[kNB], const float *s, float v) {
#pragma unroll
    for (int c4 = 0; c4 < W / 4; ++c4) {
        const float4 u = *reinterpret_cast<const float4 *>(s + 4 * c4);
        x[4 * c4 + 0] = fmaf(-u.x, v, x[4 * c4 + 1]);
        x[4 * c4 + 1] = fmaf(-u.y, v, x[4 * c4 + 2]);
        x[4 * c4 + 2] = fmaf(-u.z, v, x[4 * c4 + 3]);
        x[4 * c4 + 3] = (4 * c4 + 4 < W) ? fmaf(-u.w, v, x[4 * c4 + 4]) : 0.0f;
    }
}


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

// ---- 128 x 128 SIMT GEMM tile staged by cp.async -----------------------------
// The same tile as gemm_tile with the same per-element operation order (each
// output is one fmaf chain over k ascending from 0, then times alpha, then
// plus C), so the two give identical bits; only the data movement differs.
// gemm_tile moves 16-deep slices through registers with two CTA barriers
// each and reads C by scattered scalar loads after the products, which puts
// four L2 round trips and 64 uncoalesced requests per thread on every
// 128 x 128 x 64 tile.  Here 16-byte cp.async copies (L2 only, .cg: the data
// may come from other CTAs behind a grid barrier) bring a whole 64-deep
// slice of both operands and, for an accumulating tile, the C tile into
// shared memory at once, the next slice streams into the second buffer
// while the current one is multiplied, and C is written back by float4
// stores.  Needs 16-byte aligned bases, leading dimensions that are
// multiples of 4 floats and kb % 4 == 0 (gemm_tile_v_ok); ragged edges are
// zero-filled through cp.async's source size.
struct __align__(16) SmemGVBuf {
    float As[kNB][GBM];      // As[k][row]
    float Bs[GBN][kNB + 4];  // Bs[col][k]
};
struct __align__(16) SmemGV {
    SmemGVBuf buf[2];  // two 64-deep operand slices; a C tile Cs[col][row] (pitch 132) in buf[1]
};
static_assert(sizeof(SmemGVBuf) == sizeof(float) * GBN * (GBM + 4), "the C tile fills one operand buffer");

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }
__device__ __forceinline__ bool gemm_tile_v_ok(const float *A, int64_t lda, const float *B, int64_t ldb,
                                               const float *C, int64_t ldc, int kb) {
    return aligned16(A) && aligned16(B) && aligned16(C) && ((lda | ldb | ldc) & 3) == 0 && (kb & 3) == 0;
}

// bytes of a 4-float group starting at index i of an extent e (0 .. 16)
__device__ __forceinline__ int grp_bytes(int i, int e) { return 4 * max(0, min(4, e - i)); }

// one 64-deep slice [k0, k0 + 64) ∩ [k0, ke) of A(m0:m0+128, :) and B(:, n0:n0+128)
__device__ __forceinline__ void gv_load_slice(SmemGVBuf &b, int m, int n, int k0, int ke, const float *A,
                                              int64_t lda, const float *B, int64_t ldb, int m0, int n0) {
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 8; ++q) {  // A: 64 k x 32 row groups
        const int idx = t + kCT * q;
        const int kk = idx >> 5, r = (idx & 31) * 4;
        const int gk = k0 + kk, gr = m0 + r;
        const int by = gk < ke ? grp_bytes(gr, m) : 0;
        cp_async16(&b.As[kk][r], by ? A + (int64_t)gk * lda + gr : A, by);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {  // B: 128 columns x 16 k groups
        const int idx = t + kCT * q;
        const int c = idx >> 4, kk = (idx & 15) * 4;
        const int gc = n0 + c, gk = k0 + kk;
        const int by = gc < n ? grp_bytes(gk, ke) : 0;
        cp_async16(&b.Bs[c][kk], by ? B + (int64_t)gc * ldb + gk : B, by);
    }
}

// MI = 4 (NJ = 4): the tile's live rows (columns) are its first 64 only, the
// caller guarantees m - m0 <= 64 (n - n0 <= 64), and the padding half is
// neither multiplied nor stored (the live elements' operations unchanged).
template <int MI = 8, int NJ = 8>
__device__ void gemm_tile_v(SmemGV &sv, int m, int n, int kb, int ke, float alpha, const float *__restrict__ A,
                            int64_t lda, const float *__restrict__ B, int64_t ldb, bool accumulate, float *C,
                            int64_t ldc, int m0, int n0, int skip = 0) {
    static_assert((MI == 4 || MI == 8) && (NJ == 4 || NJ == 8), "full or half tile sides");
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    float(*Cs)[GBM + 4] = reinterpret_cast<float(*)[GBM + 4]>(&sv.buf[1]);
    const int nch = ke > kb ? (ke - kb + kNB - 1) / kNB : 0;
    const bool c_early = accumulate && nch <= 1;  // C shares buf[1] with the second slice
    __syncthreads();  // the caller's previous use of this memory is over
    if (nch > 0) gv_load_slice(sv.buf[0], m, n, kb, ke, A, lda, B, ldb, m0, n0);
    cp_async_commit();
    auto load_c = [&]() {
#pragma unroll
        for (int q = 0; q < 16; ++q) {  // 128 columns x 32 row groups
            const int idx = t + kCT * q;
            const int c = idx >> 5, r = (idx & 31) * 4;
            const int gc = n0 + c, gr = m0 + r;
            const int by = gc < n ? grp_bytes(gr, m) : 0;
            cp_async16(&Cs[c][r], by ? C + (int64_t)gc * ldc + gr : C, by);
        }
        cp_async_commit();
    };
    if (c_early) load_c();

    float acc[MI][NJ];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[i][j] = 0.0f;

    for (int ch = 0; ch < nch; ++ch) {
        const int k0 = kb + ch * kNB;
        if (ch + 1 < nch) {
            gv_load_slice(sv.buf[(ch + 1) & 1], m, n, k0 + kNB, ke, A, lda, B, ldb, m0, n0);
            cp_async_commit();
            cp_async_wait<1>();  // slice ch has landed, ch + 1 may be in flight
        } else if (c_early) {
            cp_async_wait<1>();  // slice ch has landed, C may be in flight
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const SmemGVBuf &b = sv.buf[ch & 1];
        const int nk4 = (min(kNB, ke - k0) + 3) / 4;
#pragma unroll 1
        for (int k4 = 0; k4 < nk4; ++k4) {
            float4 bq[NJ];
#pragma unroll
            for (int j = 0; j < NJ; ++j)
                bq[j] = *reinterpret_cast<const float4 *>(&b.Bs[j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4)][4 * k4]);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                float av[MI];
                {
                    const float4 a0 = *reinterpret_cast<const float4 *>(&b.As[4 * k4 + s][tx * 4]);
                    av[0] = a0.x;
                    av[1] = a0.y;
                    av[2] = a0.z;
                    av[3] = a0.w;
                }
                if constexpr (MI == 8) {
                    const float4 a1 = *reinterpret_cast<const float4 *>(&b.As[4 * k4 + s][64 + tx * 4]);
                    av[MI - 4] = a1.x;
                    av[MI - 3] = a1.y;
                    av[MI - 2] = a1.z;
                    av[MI - 1] = a1.w;
                }
                float bv[NJ];
#pragma unroll
                for (int j = 0; j < NJ; ++j) bv[j] = s == 0 ? bq[j].x : s == 1 ? bq[j].y : s == 2 ? bq[j].z : bq[j].w;
#pragma unroll
                for (int i = 0; i < MI; ++i)
#pragma unroll
                    for (int j = 0; j < NJ; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
            }
        }
        __syncthreads();  // buf[ch & 1] is refilled two slices on (or holds C)
    }
    if (accumulate) {
        if (!c_early) load_c();
        cp_async_wait<0>();
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
        const int cl = j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4);
        const int gc = n0 + cl;
        if (gc >= n) continue;
#pragma unroll
        for (int h = 0; h < MI / 4; ++h) {
            const int rl = h * 64 + tx * 4, gr = m0 + rl;
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) v[e] = acc[4 * h + e][j] * alpha;
            if (accumulate) {
                const float4 c4 = *reinterpret_cast<const float4 *>(&Cs[cl][rl]);
                v[0] += c4.x;
                v[1] += c4.y;
                v[2] += c4.z;
                v[3] += c4.w;
            }
            // element (rl + e, cl) of the tile is left alone when rl + e < skip and cl < skip
            float *dst = C + (int64_t)gc * ldc + gr;
            if (gr + 3 < m && (cl >= skip || rl >= skip)) {
                *reinterpret_cast<float4 *>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                continue;
            }
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (gr + e < m && !(cl < skip && rl + e < skip)) dst[e] = v[e];
        }
    }
    __syncthreads();  // shared memory is reused by the caller's next item
}

// C[0:m, 0:n] += alpha * A(:, 0:k) B(0:k, :) for m, n <= 64 (one 64 x 64 tile,
// 4 x 4 outputs per thread): the look-ahead update of the next diagonal block.
// C is read together with the first operand slice (one L2 round trip for
// all three).  to_smem: the result goes to sm.t.t[col][row] instead of C, for
// getrf64(..., in_smem = true) to factor without a global round trip (the
// caller then owns writing it back; getrf64 does).
__device__ void gemm_tile64(Smem &sm, int m, int n, int k, float alpha, const float *__restrict__ A, int64_t lda,
                            const float *__restrict__ B, int64_t ldb, float *C, int64_t ldc, bool to_smem = false) {
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    float acc[4][4], cv[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[i][j] = 0.0f;
            const int gr = tx * 4 + i, gc = ty * 4 + j;
            cv[i][j] = (gr < m && gc < n) ? __ldcg(C + (int64_t)gc * ldc + gr) : 0.0f;
        }
    for (int k0 = 0; k0 < k; k0 += kNB) {
        // the whole 64-deep slice of both operands in one L2 round trip
        const int kc = min(kNB, k - k0);
        float va[16], vb[16];
        load_block64(va, A + (int64_t)k0 * lda, lda, m, kc);  // va: A(r, k0 + c)
#pragma unroll
        for (int q = 0; q < 16; ++q) {  // vb: B(k0 + kk, c), kk fastest
            const int idx = t + kCT * q;
            const int kk = idx % kNB, c = idx / kNB;
            vb[q] = (kk < kc && c < n) ? __ldcg(B + (int64_t)c * ldb + k0 + kk) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int idx = t + kCT * q;
            sm.g64.As[idx / kNB][idx % kNB] = va[q];
            sm.g64.Bs[idx % kNB][idx / kNB] = vb[q];
        }
        __syncthreads();
#pragma unroll 16
        for (int kk = 0; kk < kNB; ++kk) {
            const float4 a = *reinterpret_cast<const float4 *>(&sm.g64.As[kk][tx * 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&sm.g64.Bs[kk][ty * 4]);
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
            if (gr < m && gc < n) acc[i][j] += cv[i][j];
        }
    }
    if (to_smem) __syncthreads();  // the operand slices share memory with t
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int gc = ty * 4 + j;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gr = tx * 4 + i;
            if (to_smem) sm.t.t[gc][gr] = acc[i][j];
            else if (gr < m && gc < n) C[(int64_t)gc * ldc + gr] = acc[i][j];
        }
    }
    __syncthreads();
}

// ---- 64 x 64 no-pivot LU of D (nb <= 64), warps 0 and 1 ---------------------
// sgetrf_nopiv_naive order (sgetrf_nopiv.cpp:27-61): scale by the reciprocal
// pivot, then the rank-1 update.  Lane l of each warp keeps rows l and l + 32;
// warp 0 holds columns 0..31, warp 1 columns 32..63.
//  pivots 0..31: warp 0 factors its columns, each row rotated (rot_axpy's
//    scheme: at pivot k an active row holds A(r, k ..) from index 0), the
//    pivot row by register shuffles, the next pivot's reciprocal
//    (rcp_rn_f32, branch-free) issued as soon as that pivot is final; it
//    publishes each pivot's multipliers (column k of L) in shared memory and
//    raises ready[k].  Warp 1 follows pivot by pivot: it waits for ready[k]
//    (bounded), takes the multipliers and the pivot row's right half (row k
//    is in its own registers, by shuffles) and updates its columns;
//  pivots 32..63: warp 1 alone on rows 32..63 of its columns, rotated.
// Every element receives the same fmaf updates in the same order as in the
// one-warp form, so the factors are bit-identical; splitting the columns
// halves the shuffles on the pivot chain (~4 issue cycles each).  Rows stop
// rotating at their own pivot, so at the end each lane holds its rows of U;
// the factor goes through shared memory (T = t[col][row]) to one coalesced
// store (scattered global stores stalled it under the L2 traffic of the
// trailing update running beside it).  Warps 2..7 wait at the barriers.
template <int W>
__device__ __forceinline__ void getrf64_left(float (*T)[kNB + 4], volatile int *ready, float (&a0)[32],
                                             float (&a1)[32], float &pv, float &rp, int k0, int k1, int nb,
                                             DevStatus *dst, int pivot_base) {
    const int ln = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        if (ln == 0 && (!(pv != 0.0f) || !isfinite(pv))) report(dst, MXP_ZERO_PIVOT, pivot_base + k + 1, 0);
        const bool act0 = ln > k && ln < nb, act1 = ln + 32 < nb;
        const float l0 = act0 ? a0[0] * rp : 0.0f;
        const float l1 = act1 ? a1[0] * rp : 0.0f;
        if (act0) T[k][ln] = l0;
        if (act1) T[k][ln + 32] = l1;
        __threadfence_block();
        __syncwarp();
        if (ln == 0) ready[k] = 1;
        const float u0 = __shfl_sync(full, a0[1], k);
        if (act0) a0[0] = fmaf(-u0, l0, a0[1]);
        if (act1) a1[0] = fmaf(-u0, l1, a1[1]);
        if (k + 1 < 32) {  // uniform: the next pivot is final now
            pv = __shfl_sync(full, a0[0], k + 1);
            rp = rcp_rn_f32(pv);
        }
#pragma unroll
        for (int c = 1; c < W - 1; ++c) {
            const float u = __shfl_sync(full, a0[c + 1], k);
            if (act0) a0[c] = fmaf(-u, l0, a0[c + 1]);
            if (act1) a1[c] = fmaf(-u, l1, a1[c + 1]);
        }
        if (act0) a0[W - 1] = 0.0f;
        if (act1) a1[W - 1] = 0.0f;
    }
}

template <int W>
__device__ __forceinline__ void getrf64_lower_right(float (*T)[kNB + 4], float (&b1)[32], float &pv, float &rp,
                                                    int k0, int k1, int nb, DevStatus *dst, int pivot_base) {
    const int ln = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        if (ln == 0 && (!(pv != 0.0f) || !isfinite(pv))) report(dst, MXP_ZERO_PIVOT, pivot_base + k + 1, 0);
        const int src = k - 32;  // row k: b1 of lane k - 32
        const bool act1 = ln + 32 > k && ln + 32 < nb;
        const float l1 = act1 ? b1[0] * rp : 0.0f;
        const float u0 = __shfl_sync(full, b1[1], src);
        if (act1) b1[0] = fmaf(-u0, l1, b1[1]);
        {  // the next pivot (past the last one the value is not used)
            pv = __shfl_sync(full, b1[0], (k + 1) & 31);
            rp = rcp_rn_f32(pv);
        }
        if (act1) T[k][ln + 32] = l1;
#pragma unroll
        for (int c = 1; c < W - 1; ++c) {
            const float u = __shfl_sync(full, b1[c + 1], src);
            if (act1) b1[c] = fmaf(-u, l1, b1[c + 1]);
        }
        if (act1) b1[W - 1] = 0.0f;
    }
}

// in_smem: the block to factor is already in sm.t.t[col][row] (gemm_tile64's
// to_smem output), not read from D; either way the factors are written to D.
__device__ __noinline__ void getrf64(Smem &sm, int nb, float *D, int64_t lda, DevStatus *dst, int pivot_base,
                                     bool in_smem = false) {
    float(*T)[kNB + 4] = sm.t.t;  // T[c][r]: the factored block, written out at the end
    volatile int *ready = sm.t.ready;
    if (threadIdx.x < 32) ready[threadIdx.x] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    if (warp == 0) {
        float a0[32], a1[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            a0[j] = (j < nb && ln < nb) ? (in_smem ? T[j][ln] : __ldcg(D + (int64_t)j * lda + ln)) : 0.0f;
            a1[j] = (j < nb && ln + 32 < nb) ? (in_smem ? T[j][ln + 32] : __ldcg(D + (int64_t)j * lda + ln + 32))
                                             : 0.0f;
        }
        float pv = __shfl_sync(full, a0[0], 0);
        float rp = rcp_rn_f32(pv);
        getrf64_left<32>(T, ready, a0, a1, pv, rp, 0, min(nb, 16), nb, dst, pivot_base);
        getrf64_left<16>(T, ready, a0, a1, pv, rp, 16, min(nb, 32), nb, dst, pivot_base);
        // rows 0..31 of U in columns 0..31: a0[c] = U(l, l + c)
#pragma unroll
        for (int c = 0; c < 32; ++c)
            if (ln < nb && ln + c < min(nb, 32)) T[ln + c][ln] = a0[c];
    } else if (warp == 1) {
        float b0[32], b1[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            b0[j] = (32 + j < nb && ln < nb) ? (in_smem ? T[32 + j][ln] : __ldcg(D + (int64_t)(32 + j) * lda + ln))
                                             : 0.0f;
            b1[j] = (32 + j < nb && ln + 32 < nb)
                        ? (in_smem ? T[32 + j][ln + 32] : __ldcg(D + (int64_t)(32 + j) * lda + ln + 32))
                        : 0.0f;
        }
        if (nb > 32) {
#pragma unroll 1
            for (int k = 0; k < 32; ++k) {
                // warp 0's multipliers of pivot k (bounded wait)
                const unsigned long long t0 = globaltimer_ns();
                while (ready[k] == 0) {
                    if (globaltimer_ns() - t0 > kWaitTimeoutNs) {
                        if (ln == 0) report(dst, MXP_TIMEOUT, 40, blockIdx.x);
                        break;
                    }
                }
                __threadfence_block();
                const bool act0 = ln > k && ln < nb, act1 = ln + 32 < nb;
                const float l0 = act0 ? T[k][ln] : 0.0f;
                const float l1 = act1 ? T[k][ln + 32] : 0.0f;
#pragma unroll
                for (int c = 0; c < 32; ++c) {  // row k's right half: b0 of lane k
                    const float u = __shfl_sync(full, b0[c], k);
                    if (act0) b0[c] = fmaf(-u, l0, b0[c]);
                    if (act1) b1[c] = fmaf(-u, l1, b1[c]);
                }
            }
            // rows 0..31 of U in columns 32..63
#pragma unroll
            for (int c = 0; c < 32; ++c)
                if (ln < nb && 32 + c < nb) T[32 + c][ln] = b0[c];
            float pv = __shfl_sync(full, b1[0], 0);
            float rp = rcp_rn_f32(pv);
            getrf64_lower_right<32>(T, b1, pv, rp, 32, min(nb, 48), nb, dst, pivot_base);
            getrf64_lower_right<16>(T, b1, pv, rp, 48, nb, nb, dst, pivot_base);
#pragma unroll
            for (int c = 0; c < 32; ++c)
                if (ln + 32 < nb && ln + 32 + c < nb) T[ln + 32 + c][ln + 32] = b1[c];
        }
    }
    __syncthreads();
    // the whole block in one coalesced pass
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int idx = threadIdx.x + kCT * q;
        const int r = idx % kNB, c = idx / kNB;
        if (r < nb && c < nb) D[(int64_t)c * lda + r] = T[c][r];
    }
    __syncthreads();
}

// D (nb x nb, factored) into shared memory: t[col][row], the skewed rows of U
// and columns of L the rotated strip solves read (us, ls), and the reciprocal
// diagonal.
__device__ void load_tri(Smem &sm, int nb, const float *D, int64_t lda) {
    float v[16];
    load_block64(v, D, lda, nb, nb);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int idx = threadIdx.x + kCT * q;
        sm.t.t[idx / kNB][idx % kNB] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int idx = threadIdx.x + kCT * q;
        const int k = idx / kNB, c = idx % kNB, j = k + 1 + c;
        sm.t.us[k][c] = j < nb ? sm.t.t[j][k] : 0.0f;
        sm.t.ls[k][c] = j < nb ? sm.t.t[k][j] : 0.0f;
    }
    if (threadIdx.x < nb) sm.t.dinv[threadIdx.x] = 1.0f / sm.t.t[threadIdx.x][threadIdx.x];
    __syncthreads();
}

// L strip rows [r0, r0 + rows) of B (m x nb), rows <= kCT: X = B U^{-1}, U =
// upper part of the diagonal block (load_tri).  Right-looking, thread per row
// (x_k final, then x_c -= u_kc x_k for c > k): per element the same
// operations in the same order as the dot-product form; the row rotates
// (rot_axpy) so the pivot loop stays rolled, and x_k is stored as soon as it
// is final.
template <int W>
__device__ __forceinline__ void trsm_rows_phase(Smem &sm, float (&x)[kNB], int k0, int k1, float *B, int64_t ldb,
                                                int i) {
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        const float xk = x[0] * sm.t.dinv[k];
        B[(int64_t)k * ldb + i] = xk;
        rot_axpy<W>(x, &sm.t.us[k][0], xk);
    }
}

// The row of B this thread solves (zero when it has none), and the solve of a
// row loaded that way: split so a caller can issue the loads before load_tri.
__device__ __forceinline__ void trsm_rows_load(float (&x)[kNB], int m, int nb, const float *B, int64_t ldb, int r0,
                                               int rows) {
    const int i = r0 + threadIdx.x;
    const bool act = threadIdx.x < rows && i < m;
#pragma unroll
    for (int c = 0; c < kNB; ++c) x[c] = (act && c < nb) ? __ldcg(B + (int64_t)c * ldb + i) : 0.0f;
}
__device__ __forceinline__ void trsm_rows_solve(Smem &sm, float (&x)[kNB], int m, int nb, float *B, int64_t ldb,
                                                int r0, int rows) {
    const int i = r0 + threadIdx.x;
    if (threadIdx.x >= rows || i >= m) return;
    trsm_rows_phase<64>(sm, x, 0, min(nb, 16), B, ldb, i);
    trsm_rows_phase<48>(sm, x, 16, min(nb, 32), B, ldb, i);
    trsm_rows_phase<32>(sm, x, 32, min(nb, 48), B, ldb, i);
    trsm_rows_phase<16>(sm, x, 48, nb, B, ldb, i);
}

__device__ void trsm_rows(Smem &sm, int m, int nb, float *B, int64_t ldb, int r0, int rows = kCT) {
    float x[kNB];
    trsm_rows_load(x, m, nb, B, ldb, r0, rows);
    trsm_rows_solve(sm, x, m, nb, B, ldb, r0, rows);
}

// One column of X = L^{-1} B (L unit lower, load_tri) in registers: x_r -=
// l_rk x_k for r > k, rotated; x_k goes to out[k] as soon as it is final.
template <int W>
__device__ __forceinline__ void trsm_col_phase(Smem &sm, float (&x)[kNB], int k0, int k1, float *out) {
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        const float xk = x[0];
        out[k] = xk;
        rot_axpy<W>(x, &sm.t.ls[k][0], xk);
    }
}

__device__ __forceinline__ void trsm_col(Smem &sm, float (&x)[kNB], int nb, float *out) {
    trsm_col_phase<64>(sm, x, 0, min(nb, 16), out);
    trsm_col_phase<48>(sm, x, 16, min(nb, 32), out);
    trsm_col_phase<32>(sm, x, 32, min(nb, 48), out);
    trsm_col_phase<16>(sm, x, 48, nb, out);
}

// U strip columns [c0, c0 + 64) of B (nb x ncols): X = L^{-1} B, L = unit lower
// part of the diagonal block (load_tri).  The 64 x 64 block moves through
// shared memory (ub, over the dead t) with coalesced loads and stores;
// threads 0..63 solve one column each.
// v[0..15]: the block, already loaded by load_block64(v, B + c0 ldb, ldb, nb, ncols - c0)
template <int N>
__device__ void trsm_cols64_loaded(Smem &sm, const float (&v)[N], int ncols, int nb, float *B, int64_t ldb,
                                   int c0) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int idx = threadIdx.x + kCT * q;
        sm.t.ub[idx / kNB][idx % kNB] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < kNB) {
        const int j = threadIdx.x;
        float x[kNB];
#pragma unroll
        for (int k = 0; k < kNB; ++k) x[k] = sm.t.ub[j][k];
        trsm_col(sm, x, nb, &sm.t.ub[j][0]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += kCT) {
        const int k = idx % kNB, j = idx / kNB;
        if (k < nb && c0 + j < ncols) B[(int64_t)(c0 + j) * ldb + k] = sm.t.ub[j][k];
    }
    __syncthreads();
}

__device__ void trsm_cols64(Smem &sm, int ncols, int nb, float *B, int64_t ldb, int c0) {
    float v[16];
    load_block64(v, B + (int64_t)c0 * ldb, ldb, nb, ncols - c0);
    trsm_cols64_loaded(sm, v, ncols, nb, B, ldb, c0);
}

// Inverse of the 64 x 64 diagonal block `blk` of an upper non-unit (upper = true)
// or unit-lower triangle; row i of the inverse solves x T = e_i.
__device__ void inv_diag_block(Smem &sm, int n, const float *T, int64_t ldt, float *X, int64_t ldx,
                               int blk, bool upper) {
    const int r0 = blk * kNB;
    const int nb = min(kNB, n - r0);
    {
        float v[16];
        load_block64(v, T + r0 + (int64_t)r0 * ldt, ldt, nb, nb);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int idx = threadIdx.x + kCT * q;
            sm.t.t[idx / kNB][idx % kNB] = v[q];
        }
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

// sv (when not null, with at least sizeof(SmemGV) bytes behind it): tiles
// whose operands allow it run as gemm_tile_v.
__device__ void run_jobs(Smem &sm, const Job *jobs, int njobs, int cta, int ncta, SmemGV *sv = nullptr) {
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
        const float *Az = J.A + J.sA * z, *Bz = J.B + J.sB * z;
        float *Cz = J.C + J.sC * z;
        if (sv && gemm_tile_v_ok(Az, J.lda, Bz, J.ldb, Cz, J.ldc, kb))
            gemm_tile_v(*sv, J.m, J.n, kb, ke, J.alpha, Az, J.lda, Bz, J.ldb, false, Cz, J.ldc, m0, n0);
        else
            gemm_tile(sm, J.m, J.n, kb, ke, J.alpha, Az, J.lda, Bz, J.ldb, false, Cz, J.ldc, m0, n0);
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
                             float *tmpU, float *tmpL, int cta, int G, Sync sync, int s_stop = 0,
                             SmemGV *sv = nullptr) {
    const int nsteps = (n + kNB - 1) / kNB;
    // invert the diagonal 64 x 64 blocks and zero the opposite block-triangle
    const int nblk = nsteps;
    for (int it = cta; it < 2 * nblk; it += G)
        inv_diag_block(sm, n, A, lda, it < nblk ? XU : XL, ldx, it % nblk, it < nblk);
    {   // zero the opposite block-triangles: a column per warp, rows by lanes
        // (a flat index split by 64-bit division cost ~30 us per 2560 block)
        constexpr int W = kCT / 32;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int c = cta * W + warp; c < n; c += G * W) {
            const int cb = c / kNB;
            float *xu = XU + (int64_t)c * ldx, *xl = XL + (int64_t)c * ldx;
            for (int r = lane; r < n; r += 32) {
                const int rb = r / kNB;
                if (rb > cb) xu[r] = 0.0f;
                if (rb < cb) xl[r] = 0.0f;
            }
        }
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
        run_jobs(sm, jb, nj, cta, G, sv);
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
        run_jobs(sm, jb, nj, cta, G, sv);
        if (!sync(25)) return false;
    }
    return true;
}

}  // namespace
}  // namespace dt
}  // namespace mxp
