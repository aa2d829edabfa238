/*
 * mxp_oracle.c -- CPU restatement of OpenMxP's single-process solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * openmxp_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product path never calls into it.
 *
 * Parity pinning: the generator functions below are checked bit-for-bit
 * against the reference's own hpl_rand.hpp compiled in place (the Makefile's
 * `ref` target -> oracle/_ref/libmxpref.so) and against the committed
 * fixtures in tests/golden/.  The LU/Schur/TRSM/IR restatements follow the
 * reference's algorithm; the reference's numbers at that boundary come from
 * rocBLAS/rocSOLVER, which are not part of the reference tree, so factor
 * parity is a tolerance check (relative Frobenius) rather than bitwise.
 *
 * Every function cites the reference file:line it restates.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* 64-bit LCG: x <- a*x + c (mod 2^64)                hpl_rand.hpp:12-78      */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint64_t a, c;
} orc_aff;

static const orc_aff ORC_INC1 = {6364136223846793005ULL, 1ULL}; /* hpl_rand.hpp:16 */

/* f o g : x -> f.a*(g.a*x+g.c)+f.c                     hpl_rand.hpp:18-20 */
static inline orc_aff aff_mul(orc_aff f, orc_aff g) {
    orc_aff r;
    r.a = f.a * g.a;
    r.c = f.a * g.c + f.c;
    return r;
}

/* f^n by binary powering                               hpl_rand.hpp:31-48 */
static orc_aff aff_pow(orc_aff f, uint64_t n) {
    orc_aff r = {1ULL, 0ULL};
    orc_aff t = f;
    while (n) {
        if (n & 1ULL) r = aff_mul(r, t);
        t = aff_mul(t, t);
        n >>= 1;
    }
    return r;
}

static inline uint64_t aff_apply(orc_aff f, uint64_t x) { return f.a * x + f.c; }

/* state -> double in [-0.5, 0.5]                       hpl_rand.hpp:64-73 */
static inline double state_to_double(uint64_t x) {
    return (double)(int64_t)x * 0x1.fffffffffffffP-65;
}

/* RandStat::initialize(seed) = INC1 * {seed}           hpl_rand.hpp:54-57 */
static inline uint64_t stat00(uint64_t seed) { return aff_apply(ORC_INC1, seed); }

/* Stream index of element (i, j) is i + n*j            hpl_rand.hpp:249-254 */
ORC_EXPORT double orc_elem(int n, uint64_t seed, int64_t i, int64_t j) {
    orc_aff jmp = aff_pow(ORC_INC1, (uint64_t)i + (uint64_t)n * (uint64_t)j);
    return state_to_double(aff_apply(jmp, stat00(seed)));
}

ORC_EXPORT uint64_t orc_state(int n, uint64_t seed, int64_t i, int64_t j) {
    orc_aff jmp = aff_pow(ORC_INC1, (uint64_t)i + (uint64_t)n * (uint64_t)j);
    return aff_apply(jmp, stat00(seed));
}

ORC_EXPORT void orc_aff_pow(uint64_t a, uint64_t c, uint64_t n, uint64_t *out_a, uint64_t *out_c) {
    orc_aff f = {a, c};
    orc_aff r = aff_pow(f, n);
    *out_a = r.a;
    *out_c = r.c;
}

/* ------------------------------------------------------------------------ */
/* Matrix generation                                                         */
/* ------------------------------------------------------------------------ */

/* Diagonal rules.  0 = the reference's rule (diag = off-diagonal row sum of
 * |a_ij|, matgen.hpp:26-62).  1 = 0.55*rowsum + 1 (weaker dominance stress
 * form; not a reference feature). */
enum { ORC_DIAG_ROWSUM = 0, ORC_DIAG_055_PLUS1 = 1 };

/* Row sum of |a_ij| (j != i) in the pinned GPU reduction order of
 * fill_panel_diag_dev (matgen.hpp:26-62): 512 strided partials, thread t
 * summing columns t, t+512, ... in ascending order; tree 512 -> 4
 * (matgen.hpp:39-57); then ((s0+s1)+s2)+s3 (matgen.hpp:61). */
static double rowsum_gpu_order(int n, uint64_t seed, int64_t row, const orc_aff *pn_t,
                               orc_aff j512) {
    double part[512];
    uint64_t s00 = stat00(seed);
    orc_aff ri = aff_pow(ORC_INC1, (uint64_t)row);
    uint64_t srow = aff_apply(ri, s00);
    for (int t = 0; t < 512; ++t) {
        double acc = 0.0;
        if (t < n) {
            uint64_t s = aff_apply(pn_t[t], srow); /* element (row, t) */
            for (int64_t j = t; j < n; j += 512) {
                if (j != row) acc += fabs(state_to_double(s));
                s = aff_apply(j512, s);
            }
        }
        part[t] = acc;
    }
    for (int w = 256; w >= 4; w >>= 1)
        for (int t = 0; t < w; ++t) part[t] += part[t + w];
    return ((part[0] + part[1]) + part[2]) + part[3];
}

/* Full N x N FP32 matrix, FP64 diagonal d, FP64 row sums, FP64 RHS.
 *   A(i,j) = float(elem(i,j))                  matgen.hpp:67-82 (fill_panel_dev)
 *   A(i,i) = float(d_i)                        matgen.hpp:59-63
 *   rhs_i  = elem(i, n)  (stream column n)     matgen.hpp:419-436 -> hpl_rand.hpp:80-129
 * Any of d / rowsum / rhs may be NULL. */
ORC_EXPORT void orc_matgen(int n, uint64_t seed, int diag_rule, float *A, int64_t lda, double *d,
                           double *rowsum, double *rhs) {
    uint64_t s00 = stat00(seed);
    orc_aff jn = aff_pow(ORC_INC1, (uint64_t)n);
    if (A) {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < n; ++j) {
            uint64_t s = aff_apply(aff_pow(ORC_INC1, (uint64_t)n * (uint64_t)j), s00);
            float *col = A + j * lda;
            for (int64_t i = 0; i < n; ++i) {
                col[i] = (float)state_to_double(s);
                s = aff_apply(ORC_INC1, s);
            }
        }
    }
    orc_aff pn_t[512];
    pn_t[0].a = 1;
    pn_t[0].c = 0;
    for (int t = 1; t < 512; ++t) pn_t[t] = aff_mul(jn, pn_t[t - 1]);
    orc_aff j512 = aff_pow(jn, 512);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        double s = rowsum_gpu_order(n, seed, i, pn_t, j512);
        double dv = (diag_rule == ORC_DIAG_055_PLUS1) ? (0.55 * s + 1.0) : s;
        if (rowsum) rowsum[i] = s;
        if (d) d[i] = dv;
        if (A) A[i * lda + i] = (float)dv;
    }
    if (rhs) {
        uint64_t s = aff_apply(aff_pow(ORC_INC1, (uint64_t)n * (uint64_t)n), s00);
        for (int64_t i = 0; i < n; ++i) {
            rhs[i] = state_to_double(s);
            s = aff_apply(ORC_INC1, s);
        }
    }
}

/* One row sum in the pinned GPU order (for spot checks at large n). */
ORC_EXPORT double orc_rowsum_row(int n, uint64_t seed, int64_t i) {
    orc_aff jn = aff_pow(ORC_INC1, (uint64_t)n);
    orc_aff pn_t[512];
    pn_t[0].a = 1;
    pn_t[0].c = 0;
    for (int t = 1; t < 512; ++t) pn_t[t] = aff_mul(jn, pn_t[t - 1]);
    return rowsum_gpu_order(n, seed, i, pn_t, aff_pow(jn, 512));
}

/* FP64 matrix with the FP64 generator values off the diagonal and d on it:
 * the matrix the refinement's residual uses (otf_gemv_d regenerates a_ij in
 * FP64, panel_gemv.hpp:49-81; the diagonal comes from d, :13-47).  Used for
 * the FP64 forward-error oracle. */
ORC_EXPORT void orc_matgen_f64(int n, uint64_t seed, const double *d, double *A, int64_t lda) {
    uint64_t s00 = stat00(seed);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j) {
        uint64_t s = aff_apply(aff_pow(ORC_INC1, (uint64_t)n * (uint64_t)j), s00);
        double *col = A + j * lda;
        for (int64_t i = 0; i < n; ++i) {
            col[i] = (i == j) ? d[i] : state_to_double(s);
            s = aff_apply(ORC_INC1, s);
        }
    }
}

/* Row sum in the reference CPU order (calc_diag, hpl_rand.hpp:200-214):
 * one sequential sum over j ascending.  Used only to document that the CPU
 * and GPU orders agree in FP32 and may differ in the last FP64 bit. */
ORC_EXPORT double orc_rowsum_cpu_order(int n, uint64_t seed, int64_t i) {
    uint64_t s = aff_apply(aff_pow(ORC_INC1, (uint64_t)i), stat00(seed));
    orc_aff jn = aff_pow(ORC_INC1, (uint64_t)n);
    double sum = 0.0;
    for (int64_t j = 0; j < n; ++j) {
        if (j != i) sum += fabs(state_to_double(s));
        s = aff_apply(jn, s);
    }
    return sum;
}

/* ------------------------------------------------------------------------ */
/* Low-precision conversions (bit-exact restatements)                        */
/* ------------------------------------------------------------------------ */
static inline uint32_t f2u(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
static inline float u2f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* FP32 -> FP16 round-to-nearest-even, subnormals kept, overflow -> inf.
 * Semantics of __float2half in copyCoalesced / transposeCoalesced
 * (fp16_gpu_kernels.cpp:11-36,158-176) and of _cvtss_sh(x, 0) in
 * fp16sim.hpp:119. */
ORC_EXPORT uint16_t orc_f2h(float f) {
    uint32_t x = f2u(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u | ((ax >> 13) & 0x3ffu));
    if (ax == 0x7f800000u) return (uint16_t)(sign | 0x7c00u);
    int e = (int)(ax >> 23) - 127 + 15;
    if (e >= 1) {
        uint32_t m = ax & 0x7fffffu;
        uint32_t h = ((uint32_t)e << 10) | (m >> 13);
        uint32_t rem = m & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;
        if (h >= 0x7c00u) h = 0x7c00u; /* overflow (also e >= 31) */
        return (uint16_t)(sign | h);
    }
    /* half subnormal or zero */
    int shift = 14 - e;
    if (shift > 40) return (uint16_t)sign;
    uint64_t mm = (uint64_t)((ax & 0x7fffffu) | ((ax >> 23) ? 0x800000u : 0u));
    uint64_t h = mm >> shift;
    uint64_t rem = mm & ((1ULL << shift) - 1ULL);
    uint64_t half = 1ULL << (shift - 1);
    if (rem > half || (rem == half && (h & 1ULL))) h += 1ULL;
    return (uint16_t)(sign | (uint32_t)h);
}

ORC_EXPORT float orc_h2f(uint16_t h) {
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu;
    uint32_t m = h & 0x3ffu;
    if (e == 0) {
        float v = (float)m * 0x1p-24f;
        return sign ? -v : v;
    }
    if (e == 31) return u2f(sign | 0x7f800000u | (m << 13));
    return u2f(sign | ((e - 15 + 127) << 23) | (m << 13));
}

/* FP32 -> BF16 round-to-nearest-even (split hi+lo form). */
ORC_EXPORT uint16_t orc_f2bf(float f) {
    uint32_t x = f2u(f);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
    uint32_t r = x + 0x7fffu + ((x >> 16) & 1u);
    return (uint16_t)(r >> 16);
}
ORC_EXPORT float orc_bf2f(uint16_t b) { return u2f((uint32_t)b << 16); }

/* FP32 -> FP8 E4M3 (OCP "fn": bias 7, max 448, no inf), round to nearest
 * even, saturating to +-448 (satfinite); NaN -> 0x7f. */
ORC_EXPORT uint8_t orc_f2e4m3(float f) {
    uint32_t x = f2u(f);
    uint8_t sign = (uint8_t)((x >> 24) & 0x80u);
    uint32_t ax = x & 0x7fffffffu;
    if (ax > 0x7f800000u) return 0x7f;
    float a = u2f(ax);
    if (a > 448.0f) return (uint8_t)(sign | 0x7e);
    int E = (int)(ax >> 23) - 127;
    if (E >= -6) {
        /* normal: 3 mantissa bits */
        uint32_t m = (ax & 0x7fffffu) | 0x800000u; /* 24-bit significand */
        uint32_t q = m >> 20;                       /* 4 bits: 1.xxx */
        uint32_t rem = m & 0xfffffu;
        if (rem > 0x80000u || (rem == 0x80000u && (q & 1u))) q += 1u;
        if (q == 16u) {
            q = 8u;
            E += 1;
        }
        if (E > 8 || (E == 8 && q > 14u)) return (uint8_t)(sign | 0x7e);
        return (uint8_t)(sign | (uint8_t)(((uint32_t)(E + 7) << 3) | (q - 8u)));
    }
    /* subnormal: value = q * 2^-9, q in [0, 8] */
    double v = (double)a * 512.0; /* exact */
    double fl = floor(v);
    double rem = v - fl;
    uint32_t q = (uint32_t)fl;
    if (rem > 0.5 || (rem == 0.5 && (q & 1u))) q += 1u;
    return (uint8_t)(sign | (uint8_t)q); /* q == 8 encodes 2^-6 (e=1,m=0) */
}

ORC_EXPORT float orc_e4m32f(uint8_t b) {
    uint32_t sign = (b & 0x80u) ? 1u : 0u;
    uint32_t e = (b >> 3) & 0xfu;
    uint32_t m = b & 0x7u;
    float v;
    if (e == 15 && m == 7) return u2f(0x7fc00000u);
    if (e == 0)
        v = (float)m * 0x1p-9f;
    else
        v = ldexpf(1.0f + (float)m / 8.0f, (int)e - 7);
    return sign ? -v : v;
}

/* Per-tile power-of-two scale exponent for E4M3: the largest e with
 * amax * 2^e <= 448.  amax == 0 (or non-finite) -> 0. */
ORC_EXPORT int orc_e4m3_scale_exp(float amax) {
    if (!(amax > 0.0f) || !(amax < 3.0e38f)) return 0;
    int ea = (int)((f2u(amax) >> 23) & 0xffu) - 127;
    if (ea < -126) ea = -126; /* subnormal amax: treat as 2^-126 range */
    int e = 8 - ea;
    if (ldexpf(amax, e) > 448.0f) e -= 1;
    if (e > 126) e = 126;
    if (e < -126) e = -126;
    return e;
}

/* ------------------------------------------------------------------------ */
/* Dense kernels of the LU                                                   */
/* ------------------------------------------------------------------------ */

/* Unblocked right-looking no-pivot LU, FP32 (sgetrf_nopiv.cpp:27-61). */
ORC_EXPORT int orc_getrf_nopiv(int m, int n, float *a, int64_t lda) {
    int kend = n < m ? n : m;
    for (int k = 0; k < kend; ++k) {
        float piv = a[k + lda * k];
        if (piv == 0.0f || !isfinite(piv)) return k + 1;
        float inv = 1.0f / piv;
        for (int i = k + 1; i < m; ++i) a[i + lda * k] *= inv;
        for (int j = k + 1; j < n; ++j) {
            float akj = a[k + lda * j];
            float *aj = a + lda * j;
            const float *ak = a + lda * k;
            for (int i = k + 1; i < m; ++i) aj[i] -= ak[i] * akj;
        }
    }
    return 0;
}

/* B <- B * U^{-1}, U upper non-unit (STRSM R/U/N/N, panel_trf.hpp:188-207;
 * getrf_nopiv.hpp:13-16).  BLAS reference order: column j gets the
 * contributions of columns k<j, then is scaled by 1/U(j,j). */
ORC_EXPORT void orc_trsm_runn(int m, int n, const float *u, int64_t ldu, float *b, int64_t ldb) {
#pragma omp parallel for schedule(static)
    for (int i0 = 0; i0 < m; i0 += 256) {
        int i1 = i0 + 256 < m ? i0 + 256 : m;
        for (int j = 0; j < n; ++j) {
            float *bj = b + ldb * j;
            for (int k = 0; k < j; ++k) {
                float ukj = u[k + ldu * j];
                const float *bk = b + ldb * k;
                for (int i = i0; i < i1; ++i) bj[i] -= ukj * bk[i];
            }
            float t = 1.0f / u[j + ldu * j];
            for (int i = i0; i < i1; ++i) bj[i] *= t;
        }
    }
}

/* B <- L^{-1} B, L unit lower (STRSM L/L/N/U, panel_trf.hpp:225-246;
 * getrf_nopiv.hpp:21-24). */
ORC_EXPORT void orc_trsm_llnu(int m, int n, const float *l, int64_t ldl, float *b, int64_t ldb) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) {
        float *bj = b + ldb * j;
        for (int k = 0; k < m; ++k) {
            float bkj = bj[k];
            const float *lk = l + ldl * k;
            for (int i = k + 1; i < m; ++i) bj[i] -= bkj * lk[i];
        }
    }
}

/* C(i,j) -= sum_k Lf(i,k) * Rf(j,k) with FP32 accumulation; Lf/Rf are the
 * dequantised panel values (column-major m x K and n x K here).  Semantics
 * of the FP16 Schur gemm_ex (OP_N, OP_T, alpha=-1, beta=1), panel_trf.hpp:
 * 828-834 / rocm_device_macros.h:267-268, and of shgemm (fp16sim.hpp:232-241):
 * FP16 products are exact in FP32, only the accumulation rounds. */
static void schur_f32(int m, int n, int K, const float *Lf, int64_t ldl, const float *Rf,
                      int64_t ldr, float *C, int64_t ldc) {
    const int MB = 128, NB = 64, KB = 256;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int j0 = 0; j0 < n; j0 += NB) {
        for (int i0 = 0; i0 < m; i0 += MB) {
            int i1 = i0 + MB < m ? i0 + MB : m;
            int j1 = j0 + NB < n ? j0 + NB : n;
            float acc[64][128];
            for (int j = j0; j < j1; ++j)
                for (int i = 0; i < MB; ++i) acc[j - j0][i] = 0.0f;
            for (int k0 = 0; k0 < K; k0 += KB) {
                int k1 = k0 + KB < K ? k0 + KB : K;
                for (int j = j0; j < j1; ++j) {
                    float *aj = acc[j - j0];
                    for (int k = k0; k < k1; ++k) {
                        float r = Rf[j + ldr * k];
                        const float *lk = Lf + ldl * k + i0;
                        for (int i = 0; i < i1 - i0; ++i) aj[i] += lk[i] * r;
                    }
                }
            }
            for (int j = j0; j < j1; ++j) {
                float *cj = C + ldc * j;
                for (int i = i0; i < i1; ++i) cj[i] -= acc[j - j0][i - i0];
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Blocked diagonal-block LU and triangular inverses                         */
/* ------------------------------------------------------------------------ */

/* Right-looking no-pivot LU of an n x n FP32 block in 64-column steps: the
 * 64 x 64 diagonal block by sgetrf_nopiv_naive's order (reciprocal pivot,
 * scale, rank-1 update; sgetrf_nopiv.cpp:27-61), the L strip below it by
 * STRSM(R,U,N,N), the U strip right of it by STRSM(L,L,N,U), then the
 * rank-64 FP32 update of the trailing block.  The reference factors the
 * diagonal block with rocSOLVER sgetrf_npvt (panel_trf.hpp:678-681), whose
 * blocking is not part of the reference tree; this is the same no-pivot LU,
 * blocked the way the product's diagonal kernel is, so both round alike.
 * Returns 0 or 1 + the index of the first zero / non-finite pivot. */
ORC_EXPORT int orc_getrf_nopiv_blocked(int n, float *a, int64_t lda) {
    const int NB = 64;
    for (int j0 = 0; j0 < n; j0 += NB) {
        int nb = n - j0 < NB ? n - j0 : NB;
        float *D = a + j0 + lda * j0;
        int info = orc_getrf_nopiv(nb, nb, D, lda);
        if (info) return j0 + info;
        int m = n - j0 - nb;
        if (m <= 0) break;
        orc_trsm_runn(m, nb, D, lda, D + nb, lda);
        orc_trsm_llnu(nb, m, D, lda, D + lda * nb, lda);
        const float *L = D + nb;
        const float *U = D + lda * nb;
        float *T = D + nb + lda * nb;
#pragma omp parallel for schedule(static)
        for (int j = 0; j < m; ++j) {
            float *tj = T + lda * j;
            const float *uj = U + lda * j;
            for (int k = 0; k < nb; ++k) {
                float ukj = uj[k];
                const float *lk = L + lda * k;
                for (int i = 0; i < m; ++i) tj[i] -= lk[i] * ukj;
            }
        }
    }
    return 0;
}

/* C (m x n) = alpha * A (m x K) B (K x n), FP32, with the k range of every
 * output column limited to [kb(j), ke(j)) or of every row to [kb(i), ke(i))
 * by the triangular operand (tri: 1 A upper, 2 A lower, 3 B upper, 4 B
 * lower; 0 none).  The zeros skipped contribute exact zeros. */
static void gemm_f32_tri(int m, int n, int K, float alpha, const float *A, int64_t lda, const float *B,
                         int64_t ldb, float *C, int64_t ldc, int tri) {
#pragma omp parallel for schedule(dynamic, 8)
    for (int j = 0; j < n; ++j) {
        float *cj = C + ldc * j;
        for (int i = 0; i < m; ++i) cj[i] = 0.0f;
        int kb = 0, ke = K;
        if (tri == 3) ke = j + 1 < K ? j + 1 : K;
        if (tri == 4) kb = j;
        for (int k = kb; k < ke; ++k) {
            float bkj = B[k + ldb * j];
            const float *ak = A + lda * k;
            int ib = 0, ie = m;
            if (tri == 1) ie = k + 1 < m ? k + 1 : m; /* A upper: rows <= k */
            if (tri == 2) ib = k;                     /* A lower: rows >= k */
            for (int i = ib; i < ie; ++i) cj[i] += ak[i] * bkj;
        }
        for (int i = 0; i < m; ++i) cj[i] *= alpha;
    }
}

/* inv(U) -> XU and inv(L) -> XL (L unit lower) of a factored n x n block by
 * recursive doubling.  The reference forms the same inverses for its
 * TRSM-by-inverse path by a triangular solve against the identity
 * (gen_identity_mat + STRSM, panel_trf_gdirect.hpp:86-92,124-129); the
 * product computes them by doubling, and this is that computation:
 *   1. every 64 x 64 diagonal block by substitution: row i of the inverse
 *      solves x T = e_i (x_j = (delta_ij - sum_{q<j} x_q U(q,j)) / U(j,j)
 *      for U; x_j = delta_ij - sum_{q>j} x_q L(q,j) for L);
 *   2. for S = 64, 128, ... while S < s_stop (or S < n when s_stop <= 0):
 *      adjacent S-blocks (the last pair may be ragged, second block c < S)
 *      give the off-diagonal blocks X12 = -inv(U11) (U12 inv(U22)) and
 *      X21 = -inv(L22) (L21 inv(L11)), FP32 products.
 * Levels from s_stop on are left to the caller (they run as low-precision
 * tensor-core products in the product path).  Everything outside the
 * block triangles written is set to zero. */
ORC_EXPORT void orc_tri_inverses(int n, const float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                                 int s_stop) {
    const int NB = 64;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            XU[i + ldx * j] = 0.0f;
            XL[i + ldx * j] = 0.0f;
        }
    int nblk = (n + NB - 1) / NB;
#pragma omp parallel for schedule(dynamic, 1)
    for (int it = 0; it < 2 * nblk; ++it) {
        int upper = it < nblk;
        int r0 = (it % nblk) * NB;
        int nb = n - r0 < NB ? n - r0 : NB;
        float *X = upper ? XU : XL;
        float x[64];
        for (int i = 0; i < nb; ++i) {
            if (upper) {
                for (int jj = 0; jj < nb; ++jj) {
                    float v = (jj == i) ? 1.0f : 0.0f;
                    for (int q = 0; q < jj; ++q) v = fmaf(-x[q], A[r0 + q + lda * (r0 + jj)], v);
                    x[jj] = jj >= i ? v / A[r0 + jj + lda * (r0 + jj)] : 0.0f;
                }
            } else {
                for (int jj = nb - 1; jj >= 0; --jj) {
                    float v = (jj == i) ? 1.0f : 0.0f;
                    for (int q = jj + 1; q < nb; ++q) v = fmaf(-x[q], A[r0 + q + lda * (r0 + jj)], v);
                    x[jj] = jj <= i ? v : 0.0f;
                }
            }
            for (int jj = 0; jj < nb; ++jj) X[r0 + i + ldx * (r0 + jj)] = x[jj];
        }
    }
    float *T = (float *)malloc(sizeof(float) * (size_t)n * n);
    for (int S = NB; S < n && (s_stop <= 0 || S < s_stop); S *= 2) {
        int np = n / (2 * S);
        int c = n - np * 2 * S - S;
        for (int p = 0; p <= np; ++p) {
            int s2 = p < np ? S : c;
            if (s2 <= 0) break;
            int64_t r0 = (int64_t)p * 2 * S, r1 = r0 + S;
            /* U: T = U12 inv(U22) (S x s2), X12 = -inv(U11) T */
            gemm_f32_tri(S, s2, s2, 1.0f, A + r0 + lda * r1, lda, XU + r1 + ldx * r1, ldx, T, S, 3);
            gemm_f32_tri(S, s2, S, -1.0f, XU + r0 + ldx * r0, ldx, T, S, XU + r0 + ldx * r1, ldx, 1);
            /* L: T = L21 inv(L11) (s2 x S), X21 = -inv(L22) T */
            gemm_f32_tri(s2, S, S, 1.0f, A + r1 + lda * r0, lda, XL + r0 + ldx * r0, ldx, T, s2, 4);
            gemm_f32_tri(s2, S, s2, -1.0f, XL + r1 + ldx * r1, ldx, T, s2, XL + r1 + ldx * r0, ldx, 2);
        }
    }
    free(T);
}

/* Precision forms of the Schur update. */
enum { ORC_FORM_FP16 = 0, ORC_FORM_BF16X2 = 1, ORC_FORM_FP8 = 2, ORC_FORM_FP32 = 3, ORC_FORM_BF16 = 4 };

/* Quantise an m x K FP32 block (column-major, ld) to the dequantised FP32
 * values the tensor cores see.  out is m x Kout column-major (ld = m).
 * FP16: RN cast (fp16_gpu_kernels.cpp:11-36).  BF16X2: hi,lo split laid out
 * as three K segments (hi|hi|lo for the left panel, hi|lo|hi for the right),
 * so one K'=3K product gives hi*hi + hi*lo + lo*hi.  FP8: E4M3 with a
 * power-of-two scale per 128 x 128 tile. */
static void quantise_panel(int form, int is_right, int m, int K, const float *src, int64_t ld,
                           float *out);

/* Exported quantiser: the dequantised tensor-core operand of an m x K panel
 * (rows = output rows, columns = K; element (i, k) at src[i + ld k], or at
 * src[k + ld i] when src_rowmajor) into out, m x K*kmul column-major with
 * ld = m (BF16X2: hi|hi|lo segments, or hi|lo|hi when is_right). */
ORC_EXPORT void orc_quantise(int form, int is_right, int m, int K, const float *src, int64_t ld, int src_rowmajor,
                             float *out) {
    if (!src_rowmajor) {
        quantise_panel(form, is_right, m, K, src, ld, out);
        return;
    }
    float *t = (float *)malloc(sizeof(float) * (size_t)m * K);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < K; ++k)
        for (int i = 0; i < m; ++i) t[(int64_t)k * m + i] = src[k + ld * (int64_t)i];
    quantise_panel(form, is_right, m, K, t, m, out);
    free(t);
}

static void quantise_panel(int form, int is_right, int m, int K, const float *src, int64_t ld,
                           float *out) {
    if (form == ORC_FORM_FP32) {
        for (int k = 0; k < K; ++k)
            for (int i = 0; i < m; ++i) out[(int64_t)k * m + i] = src[i + ld * k];
    } else if (form == ORC_FORM_FP16) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < K; ++k)
            for (int i = 0; i < m; ++i) out[(int64_t)k * m + i] = orc_h2f(orc_f2h(src[i + ld * k]));
    } else if (form == ORC_FORM_BF16) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < K; ++k)
            for (int i = 0; i < m; ++i) out[(int64_t)k * m + i] = orc_bf2f(orc_f2bf(src[i + ld * k]));
    } else if (form == ORC_FORM_BF16X2) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < K; ++k)
            for (int i = 0; i < m; ++i) {
                float x = src[i + ld * k];
                float hi = orc_bf2f(orc_f2bf(x));
                float lo = orc_bf2f(orc_f2bf(x - hi));
                out[(int64_t)k * m + i] = hi;
                out[(int64_t)(K + k) * m + i] = is_right ? lo : hi;
                out[(int64_t)(2 * K + k) * m + i] = is_right ? hi : lo;
            }
    } else { /* FP8 */
        int mt = (m + 127) / 128, kt = (K + 127) / 128;
#pragma omp parallel for collapse(2) schedule(static)
        for (int ti = 0; ti < mt; ++ti)
            for (int tk = 0; tk < kt; ++tk) {
                int i0 = ti * 128, i1 = i0 + 128 < m ? i0 + 128 : m;
                int k0 = tk * 128, k1 = k0 + 128 < K ? k0 + 128 : K;
                float amax = 0.0f;
                for (int k = k0; k < k1; ++k)
                    for (int i = i0; i < i1; ++i) {
                        float a = fabsf(src[i + ld * k]);
                        if (a > amax) amax = a;
                    }
                int e = orc_e4m3_scale_exp(amax);
                float up = ldexpf(1.0f, e), down = ldexpf(1.0f, -e);
                for (int k = k0; k < k1; ++k)
                    for (int i = i0; i < i1; ++i)
                        out[(int64_t)k * m + i] = orc_e4m32f(orc_f2e4m3(src[i + ld * k] * up)) * down;
            }
    }
}

static int form_kmul(int form) { return form == ORC_FORM_BF16X2 ? 3 : 1; }


/* Exported single Schur update on FP32 sources (quantise both panels then
 * C -= L * R^T): L is m x K (column-major, ldl), U is K x n (the U row
 * panel, column-major, ldu), C is m x n.  This is the oracle of
 * mxp_panel_cast_{l,r} + mxp_schur_update for one step. */
ORC_EXPORT void orc_schur_update(int form, int m, int n, int K, const float *L, int64_t ldl,
                                 const float *U, int64_t ldu, float *C, int64_t ldc) {
    int Kq = K * form_kmul(form);
    float *Lf = (float *)malloc(sizeof(float) * (size_t)m * Kq);
    float *Rf = (float *)malloc(sizeof(float) * (size_t)n * Kq);
    float *Ut = (float *)malloc(sizeof(float) * (size_t)n * K);
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < K; ++k) Ut[(int64_t)k * n + j] = U[k + ldu * j];
    quantise_panel(form, 0, m, K, L, ldl, Lf);
    quantise_panel(form, 1, n, K, Ut, n, Rf);
    schur_f32(m, n, Kq, Lf, m, Rf, n, C, ldc);
    free(Lf);
    free(Rf);
    free(Ut);
}

/* Blocked right-looking no-pivot LU (panel_lu_async_wGPU, panel_trf.hpp:
 * 470-867, at a 1x1 grid).  The reference's look-ahead applies step k-1's
 * update to panel k before the rest of the trailing matrix; every element
 * still receives its updates in k order, which is what this loop does.
 * Per step: getrf of the diagonal block (panel_trf.hpp:678-681), STRSM of
 * the L column (:723, body :188-207) and the U row (:747, body :225-246),
 * casts (:724,:748), Schur update (:825-837).  Returns 0, or 1 + the global
 * index of the first zero / non-finite pivot. */
/* Factor of a diagonal block (returns 0 or 1 + the first bad pivot) and the
 * residual GEMV y = beta y + alpha A x: the oracle's own by default; the
 * CPU baseline passes the reference's compiled CPU kernels instead
 * (oracle/ref_wrap.cpp). */
typedef int (*orc_getrf_fn)(int n, float *a, int64_t lda);
typedef void (*orc_gemv_fn)(int n, int b, uint64_t seed, const double *d, double alpha, const double *x,
                            double beta, double *y);

static int getrf_default(int n, float *a, int64_t lda) { return orc_getrf_nopiv(n, n, a, lda); }

static int panel_lu_impl(int n, int b, float *A, int64_t lda, int form, orc_getrf_fn getrf);

ORC_EXPORT int orc_panel_lu(int n, int b, float *A, int64_t lda, int form) {
    return panel_lu_impl(n, b, A, lda, form, getrf_default);
}

static int panel_lu_impl(int n, int b, float *A, int64_t lda, int form, orc_getrf_fn getrf) {
    int nb = n / b;
    int kmul = form_kmul(form);
    float *Lf = NULL, *Rf = NULL, *Ut = NULL;
    for (int k = 0; k < nb; ++k) {
        int64_t kk = (int64_t)k * b;
        float *Akk = A + kk + lda * kk;
        int info = getrf(b, Akk, lda);
        if (info) {
            free(Lf);
            free(Rf);
            free(Ut);
            return (int)kk + info;
        }
        int m = n - (int)kk - b;
        if (m <= 0) break;
        float *Lcol = A + (kk + b) + lda * kk;
        float *Urow = A + kk + lda * (kk + b);
        orc_trsm_runn(m, b, Akk, lda, Lcol, lda);
        orc_trsm_llnu(b, m, Akk, lda, Urow, lda);
        if (!Lf) {
            Lf = (float *)malloc(sizeof(float) * (size_t)(n - b) * b * kmul);
            Rf = (float *)malloc(sizeof(float) * (size_t)(n - b) * b * kmul);
            Ut = (float *)malloc(sizeof(float) * (size_t)(n - b) * b);
        }
        /* U row panel transposed to m x b (the reference's R panel is U^T,
         * fp16_gpu_kernels.cpp:158-176). */
#pragma omp parallel for schedule(static)
        for (int j = 0; j < m; ++j)
            for (int q = 0; q < b; ++q) Ut[(int64_t)q * m + j] = Urow[q + lda * j];
        quantise_panel(form, 0, m, b, Lcol, lda, Lf);
        quantise_panel(form, 1, m, b, Ut, m, Rf);
        schur_f32(m, m, b * kmul, Lf, m, Rf, m, A + (kk + b) + lda * (kk + b), lda);
    }
    free(Lf);
    free(Rf);
    free(Ut);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FP64 pieces of the refinement                                             */
/* ------------------------------------------------------------------------ */

/* y = beta*y + alpha*A*x with A regenerated from the LCG in FP64 and the
 * diagonal taken from d (otf_gemv_diag_d / otf_gemv_d, panel_gemv.hpp:
 * 13-117; CPU otf_gemv, panel_gemv.hpp:310-338).  A is never read. */
ORC_EXPORT void orc_otf_gemv(int n, uint64_t seed, const double *d, double alpha, const double *x,
                             double beta, double *y) {
    uint64_t s00 = stat00(seed);
    orc_aff jn = aff_pow(ORC_INC1, (uint64_t)n);
#pragma omp parallel for schedule(static, 64)
    for (int64_t i = 0; i < n; ++i) {
        uint64_t s = aff_apply(aff_pow(ORC_INC1, (uint64_t)i), s00);
        double t = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double a = (j == i) ? d[i] : state_to_double(s);
            t += a * x[j];
            s = aff_apply(jn, s);
        }
        y[i] = beta * y[i] + alpha * t;
    }
}

/* x <- U^{-1} L^{-1} x with the FP32 factors upcast to FP64, exact
 * substitution (the column-oriented tttrsvL / tttrsvU loops of
 * panel_trsv.hpp:710-747 applied to the whole matrix; a block substitution
 * with FP64 diagonal solves as in trsvL_h / trsvU_h, panel_trsv.hpp:308-597,
 * computes the same quantity). */
ORC_EXPORT void orc_lu_solve(int n, const float *LU, int64_t lda, double *x) {
    for (int64_t j = 0; j + 1 < n; ++j) {
        double xj = x[j];
        const float *c = LU + lda * j;
        for (int64_t i = j + 1; i < n; ++i) x[i] -= xj * (double)c[i];
    }
    for (int64_t j = n - 1; j >= 0; --j) {
        const float *c = LU + lda * j;
        x[j] /= (double)c[j];
        double xj = x[j];
        for (int64_t i = 0; i < j; ++i) x[i] -= xj * (double)c[i];
    }
}

/* The reference's 1 x 1 block substitution as written (trsvL_h / trsvU_h,
 * panel_trsv.hpp:308-597 with grid.ncol == 1): the running partial sums are
 * sent to MPI_PROC_NULL and the wr/ws buffers swap every block column, so
 * row block r only receives the contributions of block columns c with
 * c == r (mod 2).  Kept to measure the effect of that behaviour; the product
 * path uses the exact substitution above. */
ORC_EXPORT void orc_lu_solve_ref1x1(int n, int b, const float *LU, int64_t lda, double *x) {
    int nb = n / b;
    double *w[2];
    w[0] = (double *)calloc((size_t)n, sizeof(double));
    w[1] = (double *)calloc((size_t)n, sizeof(double));
    for (int pj = 0; pj < nb; ++pj) {
        double *wr = w[pj & 1];
        int64_t o = (int64_t)pj * b;
        for (int q = 0; q < b; ++q) x[o + q] -= wr[o + q];
        for (int q = 0; q < b; ++q) { /* unit lower solve of the block */
            double xq = x[o + q];
            const float *c = LU + lda * (o + q);
            for (int i = q + 1; i < b; ++i) x[o + i] -= xq * (double)c[o + i];
        }
        for (int q = 0; q < b; ++q) {
            double xq = x[o + q];
            const float *c = LU + lda * (o + q);
            for (int64_t i = o + b; i < n; ++i) wr[i] += (double)c[i] * xq;
        }
    }
    memset(w[0], 0, sizeof(double) * (size_t)n);
    memset(w[1], 0, sizeof(double) * (size_t)n);
    for (int pj = nb - 1, it = 0; pj >= 0; --pj, ++it) {
        double *wr = w[it & 1];
        int64_t o = (int64_t)pj * b;
        for (int q = 0; q < b; ++q) x[o + q] -= wr[o + q];
        for (int q = b - 1; q >= 0; --q) {
            const float *c = LU + lda * (o + q);
            x[o + q] /= (double)c[o + q];
            double xq = x[o + q];
            for (int i = 0; i < q; ++i) x[o + i] -= xq * (double)c[o + i];
        }
        for (int q = 0; q < b; ++q) {
            double xq = x[o + q];
            const float *c = LU + lda * (o + q);
            for (int64_t i = 0; i < o; ++i) wr[i] += (double)c[i] * xq;
        }
    }
    free(w[0]);
    free(w[1]);
}

ORC_EXPORT double orc_infnorm(int n, const double *x) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) {
        double a = fabs(x[i]);
        m = m >= a ? m : a;
    }
    return m;
}

/* Classic iterative refinement, GPU branch of iterative_refinement2
 * (iterative_refinement.hpp:141-171):
 *   x0 = b ./ d; repeat: r = b - A x (A regenerated in FP64);
 *   hpl = |r|inf / (|A|inf |x|inf + |b|inf) / (n eps/2); stop when < 16;
 *   x += U^{-1} L^{-1} r.
 * norma: 2*max(d) for the row-sum rule (hpl_infnorm, panel_norm.hpp:129-135),
 * max(rowsum + d) otherwise.  Returns the number of corrections applied
 * before the residual test passed (the reference's "step"), or -1 when maxit
 * evaluations did not converge (iterative_refinement.hpp:173).  hist (may be
 * NULL) receives the scaled residual of every evaluation. */
static void gemv_default(int n, int b, uint64_t seed, const double *d, double alpha, const double *x,
                         double beta, double *y) {
    (void)b;
    orc_otf_gemv(n, seed, d, alpha, x, beta, y);
}

static int ir_classic_impl(int n, int b, uint64_t seed, const float *LU, int64_t lda, const double *d,
                           const double *rowsum, const double *rhs, double *x, int maxit, int ref1x1,
                           double *out_resid, double *out_hpl, double *hist, orc_gemv_fn gemv);

ORC_EXPORT int orc_ir_classic(int n, int b, uint64_t seed, const float *LU, int64_t lda,
                              const double *d, const double *rowsum, const double *rhs,
                              double *x, int maxit, int ref1x1, double *out_resid,
                              double *out_hpl, double *hist) {
    return ir_classic_impl(n, b, seed, LU, lda, d, rowsum, rhs, x, maxit, ref1x1, out_resid, out_hpl, hist,
                           gemv_default);
}

static int ir_classic_impl(int n, int b, uint64_t seed, const float *LU, int64_t lda, const double *d,
                           const double *rowsum, const double *rhs, double *x, int maxit, int ref1x1,
                           double *out_resid, double *out_hpl, double *hist, orc_gemv_fn gemv) {
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double norma = 0.0;
    for (int i = 0; i < n; ++i) {
        double v = rowsum ? rowsum[i] + d[i] : 2.0 * d[i];
        norma = norma >= v ? norma : v;
    }
    double normb = orc_infnorm(n, rhs);
    for (int i = 0; i < n; ++i) x[i] = rhs[i] / d[i];
    const double eps = 0x1p-53; /* DBL_EPSILON / 2 */
    int ret = -1;
    for (int it = 0; it < maxit; ++it) {
        memcpy(r, rhs, sizeof(double) * (size_t)n);
        double normx = orc_infnorm(n, x);
        gemv(n, b, seed, d, -1.0, x, 1.0, r);
        double normr = orc_infnorm(n, r);
        double hpl = normr / (norma * normx + normb) * 1.0 / ((double)n * eps);
        if (hist) hist[it] = hpl;
        if (out_resid) *out_resid = normr;
        if (out_hpl) *out_hpl = hpl;
        if (hpl < 16.0) {
            ret = it;
            break;
        }
        if (ref1x1)
            orc_lu_solve_ref1x1(n, b, LU, lda, r);
        else
            orc_lu_solve(n, LU, lda, r);
        for (int i = 0; i < n; ++i) x[i] += r[i];
    }
    free(r);
    return ret;
}

/* Whole solve (generation excluded from the timing as in main.cpp:617-657):
 * matgen, LU, classic IR.  t_lu / t_ir are wall seconds.  Used as the CPU
 * baseline and by the tests.  Returns the IR step count (>= 0), -1 when IR
 * did not converge, -2 on a zero pivot. */
static double wall(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

ORC_EXPORT int orc_solve_ex(int n, int b, uint64_t seed, int diag_rule, int form, int maxit, double *x,
                            double *out_stats, orc_getrf_fn getrf, orc_gemv_fn gemv);

ORC_EXPORT int orc_solve(int n, int b, uint64_t seed, int diag_rule, int form, int maxit,
                         double *x, double *out_stats /* [t_lu, t_ir, resid, hpl, iters] */) {
    return orc_solve_ex(n, b, seed, diag_rule, form, maxit, x, out_stats, NULL, NULL);
}

/* orc_solve with the diagonal-block factor and the residual GEMV supplied by
 * the caller (NULL: the oracle's own). */
ORC_EXPORT int orc_solve_ex(int n, int b, uint64_t seed, int diag_rule, int form, int maxit, double *x,
                            double *out_stats, orc_getrf_fn getrf, orc_gemv_fn gemv) {
    if (!getrf) getrf = getrf_default;
    if (!gemv) gemv = gemv_default;
    float *A = (float *)malloc(sizeof(float) * (size_t)n * n);
    double *d = (double *)malloc(sizeof(double) * (size_t)n);
    double *rs = (double *)malloc(sizeof(double) * (size_t)n);
    double *rhs = (double *)malloc(sizeof(double) * (size_t)n);
    orc_matgen(n, seed, diag_rule, A, n, d, rs, rhs);
    double t0 = wall();
    int info = panel_lu_impl(n, b, A, n, form, getrf);
    double t1 = wall();
    int ret = -1;
    double resid = -1.0, hpl = -1.0;
    if (info == 0)
        ret = ir_classic_impl(n, b, seed, A, n, d, diag_rule ? rs : NULL, rhs, x, maxit, 0, &resid, &hpl, NULL,
                              gemv);
    double t2 = wall();
    if (out_stats) {
        out_stats[0] = t1 - t0;
        out_stats[1] = t2 - t1;
        out_stats[2] = resid;
        out_stats[3] = hpl;
        out_stats[4] = (double)ret;
    }
    free(A);
    free(d);
    free(rs);
    free(rhs);
    return info ? -2 : ret;
}

/* ------------------------------------------------------------------------ */
/* Higham's HPL-AI matrix A = L U                                            */
/* ------------------------------------------------------------------------ */
/* L is unit lower triangular with every strictly lower entry alpha, U unit
 * upper triangular with every strictly upper entry beta (highammgen.hpp:4-30),
 * so a_ij = beta + alpha*beta*i (i < j), 1 + alpha*beta*i (i = j),
 * alpha + alpha*beta*j (i > j) (pmatgen, matgen.hpp:157-208); the diagonal
 * vector is d_i = 1 + alpha*beta*i (pdiaggen, matgen.hpp:399-417).  beta
 * comes from the wanted infinity-norm condition number and rho = alpha/beta
 * by bisection on Fasi and Higham's closed-form estimate of cond(A, inf)
 * (higham_mat_impl.cpp:36-149, from the hpl-ai-matrix project). */

/* The estimate of cond(A, inf) for the matrix with parameters (a, b): the
 * largest of three candidate row sums of A times the largest of two
 * candidate row sums of inv(A) (higham_mat_impl.cpp:36-64).  The integer
 * terms are formed in 64 bits: the reference forms them in int, which
 * overflows once n exceeds about 37800 (3 i'(i'-1)/2 with i' = n); below
 * that the two agree bit for bit. */
static double hg_cond_estimate(int n_, double a, double b) {
    if (isnan(a)) a = b / 2;
    const int64_t n = n_;
    const int64_t ip = floor(1. / a) < (double)n ? (int64_t)floor(1. / a) : n;
    const int64_t k = floor((1 + b) / b) < (double)(n - 1) ? (int64_t)floor((1 + b) / b) : n - 1;
    const double row_1 = 1 + (n - 1) * b;
    const double row_ip = 1 + (2 * k - ip + 1) * a + (n - ip) * b +
                          (-k * k + k + 3 * ip * (ip - 1) / 2 - n * ip + n) * a * b;
    const double row_n = 1 + (2 * k - n + 1) * a + (-k * k + k + n * (n - 1) / 2) * a * b;
    double norm_a = row_1 > row_ip ? row_1 : row_ip;
    norm_a = norm_a > row_n ? norm_a : row_n;
    const double r = (1 + a) * (1 + b);
    const double inv_1 = (1 + a) * (1. / (1 + a) + (r == 0. ? 0. : b * (1 - pow(r, n - 1)) / (1 - r)));
    const double inv_n = pow(1 + a, n) * (1. / (1 + a));
    const double norm_inv = inv_1 > inv_n ? inv_1 : inv_n;
    const double c = norm_a * norm_inv;
    return isinf(c) ? DBL_MAX : c;
}

/* Bisection for the root of f(x) = cond(rho x, x) - kappa between lo (f < 0)
 * and hi (f > 0), to a relative width of about one ulp
 * (higham_mat_impl.cpp:66-96). */
static double hg_bisect(int n, double kappa, double rho, double lo, double hi) {
    const double flo = hg_cond_estimate(n, rho * lo, lo) - kappa;
    const double fhi = hg_cond_estimate(n, rho * hi, hi) - kappa;
    if (flo > 0. || fhi < 0.) return NAN;
    for (;;) {
        if (hi - lo < (2. * fabs(hi) + 0.5) * DBL_EPSILON) break;
        const double mid = (lo + hi) / 2;
        if (mid == lo || mid == hi) break;
        const double fm = hg_cond_estimate(n, rho * mid, mid) - kappa;
        if (fm == 0.) return mid;
        if (fm < 0.)
            lo = mid;
        else
            hi = mid;
    }
    return hi;
}

/* beta for cond(A, inf) = kappa and alpha = rho beta (higham_mat_comp_beta,
 * higham_mat_impl.cpp:98-130): the upper end starts at 1/rho and halves until
 * the estimate exceeds kappa; if the root gives alpha > 1 the upper end is
 * quartered and the search repeated. */
ORC_EXPORT double orc_higham_beta(int n, double kappa, double rho) {
    const double lo = DBL_EPSILON;
    double hi = 1. / rho;
    for (int k = 1; k < 100; ++k) {
        const double f = hg_cond_estimate(n, rho * hi, hi) - kappa;
        if (isfinite(f) && f > 0.) break;
        hi *= 0.5;
    }
    double beta = hg_bisect(n, kappa, rho, lo, hi);
    while (rho * beta > 1.) {
        hi *= 0.25;
        beta = hg_bisect(n, kappa, rho, lo, hi);
    }
    return beta;
}

/* FP32 matrix and FP64 diagonal vector.  The FP32 entries are formed in
 * FP32 from the FP32-rounded parameters, one fused multiply-add each (the
 * pmatgen<float> arithmetic, matgen.hpp:169-201, with the multiply-add
 * fused). */
ORC_EXPORT void orc_higham_matgen_cols(int n, double alpha, double beta, int64_t j0, int64_t ncols, float *A,
                                       int64_t lda) {
    const float fa = (float)alpha, fb = (float)beta, fab = fa * fb;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < ncols; ++c) {
        const int64_t j = j0 + c;
        float *col = A + lda * c;
        const float low = fmaf(fab, (float)j, fa);
        for (int64_t i = 0; i < n; ++i)
            col[i] = i < j ? fmaf(fab, (float)i, fb) : (i == j ? fmaf(fab, (float)j, 1.0f) : low);
    }
}

ORC_EXPORT void orc_higham_matgen(int n, double alpha, double beta, float *A, int64_t lda, double *d) {
    const float fa = (float)alpha, fb = (float)beta, fab = fa * fb;
    const double ab = alpha * beta;
    if (A) {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < n; ++j) {
            float *col = A + lda * j;
            const float low = fmaf(fab, (float)j, fa);
            for (int64_t i = 0; i < n; ++i)
                col[i] = i < j ? fmaf(fab, (float)i, fb) : (i == j ? fmaf(fab, (float)j, 1.0f) : low);
        }
    }
    if (d)
        for (int64_t i = 0; i < n; ++i) d[i] = fma(ab, (double)i, 1.0);
}

/* FP64 entry (i, j) of the matrix the residual uses (the hmg_gemv_* values,
 * otf_gemv.cpp:135-316, with alpha and beta in the places pmatgen gives
 * them). */
static inline double hg_elem(double alpha, double beta, double ab, int64_t i, int64_t j) {
    if (i < j) return fma(ab, (double)i, beta);
    if (i > j) return fma(ab, (double)j, alpha);
    return fma(ab, (double)i, 1.0);
}

/* The FP64 matrix the residual uses, column-major (for FP64 references). */
ORC_EXPORT void orc_higham_matgen_f64(int n, double alpha, double beta, double *A, int64_t lda) {
    const double ab = alpha * beta;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < n; ++i) A[i + lda * j] = hg_elem(alpha, beta, ab, i, j);
}

/* y = b y + a A x with A regenerated in FP64, each row summed in column
 * order with fused multiply-adds (otf_gemv for HMGen, panel_gemv.hpp:362-388). */
ORC_EXPORT void orc_higham_gemv(int n, double alpha, double beta, double a, const double *x, double b,
                                double *y) {
    const double ab = alpha * beta;
#pragma omp parallel for schedule(static, 64)
    for (int64_t i = 0; i < n; ++i) {
        double t = 0.0;
        for (int64_t j = 0; j < n; ++j) t = fma(hg_elem(alpha, beta, ab, i, j), x[j], t);
        y[i] = b == 0.0 ? a * t : fma(b, y[i], a * t);
    }
}

/* ||A||_inf: every entry is positive, so the largest row sum of the entries
 * (higham_infnorm, panel_norm.hpp:136-175), each row summed in column order. */
ORC_EXPORT double orc_higham_infnorm(int n, double alpha, double beta) {
    const double ab = alpha * beta;
    double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static, 64)
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) s += hg_elem(alpha, beta, ab, i, j);
        m = m > s ? m : s;
    }
    return m;
}

ORC_EXPORT int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
