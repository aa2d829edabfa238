/*
 * mxp.h -- C ABI of the B200-native HPL-MxP single-GPU solve path.
 *
 * One GPU, 1x1 process grid: LCG matrix generation, blocked no-pivot LU with
 * a low-precision Schur update on tcgen05 tensor cores, FP64 iterative
 * refinement whose residual regenerates A on the fly.  Every entry point is
 * extern "C" with plain pointers and sizes, takes the CUDA stream it runs on
 * (as void*, 0 = legacy default stream), is asynchronous unless it says
 * otherwise, and returns an mxp_status.  Matrices are column-major with an
 * explicit leading dimension, as in the reference (panel.hpp:189-302).
 * Pointers named d_* are device pointers; h_* are host pointers.
 *
 * The comment above each function names the reference interface it replaces
 * (file:line in the OpenMxP source tree).
 */
#ifndef MXP_H
#define MXP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MXP_OK = 0,
    MXP_INVALID_ARG = 1,   /* bad size, alignment or pointer */
    MXP_ZERO_PIVOT = 2,    /* zero / non-finite pivot in the no-pivot LU */
    MXP_NONFINITE = 3,     /* NaN/Inf met in a vector or panel */
    MXP_NOT_CONVERGED = 4, /* refinement hit maxit (iterative_refinement.hpp:173) */
    MXP_TIMEOUT = 5,       /* a bounded device-side wait gave up */
    MXP_CUDA_ERROR = 6,    /* a CUDA runtime / driver call failed */
    MXP_UNSUPPORTED = 7,   /* form / size combination not built */
    MXP_NO_MEMORY = 8
} mxp_status;

/* Precision form of the Schur update (FLOW in main.cpp:46-48). */
typedef enum {
    MXP_FORM_FP16 = 0,   /* plain: FP16 x FP16 -> FP32, as the reference */
    MXP_FORM_BF16X2 = 1, /* split hi+lo BF16, three products, FP32 accumulate */
    MXP_FORM_FP8 = 2     /* FP8 E4M3, power-of-two scale per 128x128 tile */
} mxp_form;

/* Diagonal of the generated matrix. */
typedef enum {
    MXP_DIAG_ROWSUM = 0,     /* reference: d_i = sum_{j!=i} |a_ij| (matgen.hpp:26-62) */
    MXP_DIAG_055_PLUS1 = 1   /* stress form: d_i = 0.55 * rowsum_i + 1 */
} mxp_diag_rule;

typedef enum {
    MXP_IR_CLASSIC = 0,      /* iterative_refinement2 (iterative_refinement.hpp:97-174) */
    MXP_IR_GMRES = 1         /* GMRES-IR preconditioned by the low-precision LU */
} mxp_ir_method;

/* Per-phase device times of one LU, milliseconds (timer.hpp:58-85 items). */
typedef struct {
    double ms_total;
    double ms_diag_lu;   /* DIAG_LU */
    double ms_trsm;      /* TRSM_L + TRSM_R */
    double ms_cast;      /* CONV_L + CONV_R, and the split-BF16 operand casts of the TRSM */
    double ms_schur;     /* GEMM_UPDATE */
    int info;            /* 0, or 1 + global index of the first bad pivot */
    int schur_launches;  /* tcgen05 Schur kernel launches */
    double ms_trsm_inv;  /* part of ms_trsm: FP32 triangular inverses */
    double ms_trsm_gemm; /* part of ms_trsm: tensor-core products against the inverses */
    int overlapped_diag; /* diagonal factorisations run beside a trailing pass (not in ms_diag_lu;
                            their time is inside ms_schur) */
    int pad;
} mxp_lu_stats;

typedef struct {
    int iterations;      /* corrections applied before the residual test passed */
    int converged;       /* 1 when scaled residual < threshold */
    double residual;     /* ||b - A x||_inf (IRErrors.residual) */
    double hpl_harness;  /* scaled residual (IRErrors.hpl_harness) */
    double norma, normb, normx;
    double ms_total, ms_gemv, ms_trsv;
    int gemv_calls, trsv_calls;
    int inner_iterations; /* GMRES Arnoldi steps over all corrections (0 for classic) */
    double history[64];  /* scaled residual of every evaluation */
    double history_residual[64];  /* ||b - A x||_inf of every evaluation */
} mxp_ir_stats;

typedef struct mxp_workspace mxp_workspace;

/* Library version string and the last error message of the calling thread. */
const char *mxp_version(void);
const char *mxp_last_error_string(void);

/* Workspace for the LU and refinement: panel buffers (two L and two R, as
 * LRPanels lr[4] of build_panels_wGPU, panel.hpp:361-454), FP8 scale
 * tables, the diagonal-LU and TRSV scratch, IR vectors and a device status
 * word.  All device memory the hot calls use is allocated here, once.
 * device: CUDA ordinal the workspace lives on. */
mxp_status mxp_workspace_create(int n, int b, int form, int device, mxp_workspace **out);

/* Workspace options (no reference counterpart: execution choices of this
 * implementation).  MXP_OPT_TRSM_TENSOR: 1 (default) solves the two panel
 * TRSMs of each LU step as split-BF16 tensor-core products against FP32
 * triangular inverses; 0 uses the FP32 SIMT blocked substitution. */
typedef enum {
    MXP_OPT_TRSM_TENSOR = 1,
    MXP_OPT_GMRES_RESTART = 2,  /* Arnoldi steps per GMRES correction, 1..30 (default 30) */
    MXP_OPT_GMRES_TOL_EXP = 3,  /* inner tolerance 10^-value on the preconditioned residual (default 10) */
    MXP_OPT_MERGE_PANELS = 4,   /* 1 (default): merged look-ahead, MXP_OPT_MERGE_DEPTH panels per
                                   trailing pass (4); 0: one panel per step, as the reference */
    MXP_OPT_SCHUR_PAIR = 5,     /* 1: tensor-core products on pairs of SMs (2-SM MMA, 256 x 256
                                   tiles); 0 (default): one SM per 128 x 256 tile */
    MXP_OPT_DIAG_COOP = 6,      /* 1 (default): diagonal-block LU (and the triangular inverses of
                                   the tensor-core TRSM) in one cooperative launch with grid
                                   barriers; 0: one launch per 64-column step */
    MXP_OPT_TRSM_PAIR = 7,      /* 1: TRSM-by-inverse products on the 2-SM kernel; 0 (default): 1-SM */
    MXP_OPT_TEST_WITHHOLD_FLAG = 8, /* test of the bounded device waits: the next mxp_lu_solve never
                                       publishes the completion flag of this 64-row block of the
                                       forward solve, so the blocks waiting for it give up after
                                       the 2 s bound and the call returns MXP_TIMEOUT (-1: off) */
    MXP_OPT_OVERLAP_DIAG = 9,   /* merged schedule: > 0 factors the diagonal block of the next pair
                                   on this many SMs on a second stream while the trailing pass
                                   runs on the others (which take over its share of tiles when
                                   it ends); 0 (default): in sequence */
    MXP_OPT_OVERLAP_MIN = 10,   /* overlap only while the trailing matrix of the pair has at least
                                   this many blocks of rows (default 6) */
    MXP_OPT_TRSM_SINGLE = 11,   /* tensor-core TRSM by inverse: 0 (default) three split-BF16 products
                                   (hi*hi + hi*lo + lo*hi, near FP32); 1: one BF16 product, K = b
                                   (relative error ~2^-9, the reference's Alt-TRSM idea with BF16's
                                   range in place of FP16's) */
    MXP_OPT_MERGE_DEPTH = 12,   /* panels per trailing pass, 1..4 (default 4): each panel of a group
                                   updates the column and row blocks of the group's later panels,
                                   then one pass with K = depth * b applies the whole group
                                   (MXP_OPT_MERGE_PANELS 0 / 1 = depth 1 / 4) */
    MXP_OPT_INV_TC = 13,        /* triangular inverses of the diagonal block: doubling levels that
                                   join blocks of this size and larger run as tensor-core products
                                   in the TRSM's precision (default 1024; 0: all in the cooperative
                                   kernel, SIMT FP32) */
    MXP_OPT_TRSV_INV = 14,      /* 1 (default): mxp_panel_lu keeps the FP32 inverses of every
                                   diagonal block (2 * n * b floats of the workspace) and the
                                   refinement's triangular solves of that factor run as nb steps
                                   of bandwidth-bound products with them (each diagonal block:
                                   product with its inverse, then one refinement step against
                                   the factor block, in FP64); 0: the chain of 64-row blocks,
                                   each inverting its diagonal block in FP64.  Setting the
                                   option forgets the stored inverses. */
    MXP_OPT_FP8_FUSED_CAST = 15, /* FP8 form, tensor-core TRSM, b % 256 == 0: 1 (default) the
                                   TRSM products that form the L and U panels also write their
                                   E4M3 copies and per-tile scales (the same bytes as the FP8 panel
                                   casts of the stored FP32 panels, without reading them back);
                                   0: separate cast launches */
    MXP_OPT_TRSM_COUNTER = 16,  /* 1-SM TRSM-by-inverse products: 1 (default) CTAs claim output
                                   tiles from a device counter (the triangular K-skip makes tile
                                   work uneven); 0: static round robin.  Each tile is computed the
                                   same way either way, so the factors are bit-identical. */
} mxp_option;
mxp_status mxp_workspace_set_option(mxp_workspace *ws, int key, int value);
mxp_status mxp_workspace_destroy(mxp_workspace *ws);
size_t mxp_workspace_bytes(int n, int b, int form);

/* Where the workspace keeps the low-precision L or R panels the Schur update
 * reads (the device side of LRPanels::operator()(i, 'd') / get_lda(),
 * panel.hpp:321-359).  The buffer holds MXP_OPT_MERGE_DEPTH panel slots
 * side by side along K; after mxp_panel_lu the slots hold the last group's
 * panels: slot s holds panel k0 + s (k0 = first panel of the last group),
 * its row t (a row of L, or a column of U for R) at buffer row s * b + t,
 * K-major: element (row r, k) of slot s at
 *   data + (r * ld + s * slot_k + k) * esize
 * (BF16X2: three K segments, hi|hi|lo for L and hi|lo|hi for R).  FP8: the
 * UE8M0 scale of row tile r / 128 and K tile k / 128 of slot s is
 *   scales[(r / 128) * sc_ld + s * sc_slot + k / 128]
 * (the scale is 2^-(127 - byte)); other forms: scales == NULL.  Read-only
 * for callers; valid until the workspace is destroyed. */
typedef struct {
    void *data;
    int64_t ld;       /* row stride, elements */
    int64_t slot_k;   /* K offset of one slot, elements */
    int esize;        /* bytes per element: 2 (FP16, BF16X2) or 1 (FP8) */
    int slots;        /* slots in the buffer */
    int64_t rows;     /* rows in the buffer */
    uint8_t *scales;
    int sc_ld, sc_slot;
} mxp_panel_view;
mxp_status mxp_workspace_panel_view(const mxp_workspace *ws, int side /* 0: L, 1: R */,
                                    mxp_panel_view *out);

/* ---- generation ------------------------------------------------------- */

/* panel_matgen_dev + panel_colvgen (matgen.hpp:84-117, 419-436):
 * A(i,j) = float(LCG(i + n*j)), d_i = row sum of |a_ij| over j != i in the
 * reference's GPU reduction order (or the stress rule), A(i,i) = float(d_i),
 * rhs_i = LCG(i + n*n).  Bit-exact with the reference generator.  Any of
 * d_A, d_d, d_rowsum, d_rhs may be NULL to skip that output. */
mxp_status mxp_matgen(int n, uint64_t seed, int diag_rule, float *d_A, int64_t lda, double *d_d,
                      double *d_rowsum, double *d_rhs, void *stream);

/* The FP64 system that refinement solves: off-diagonals regenerated in FP64
 * (the values otf_gemv uses, otf_gemv.cpp:5-133) and the diagonal d of
 * mxp_matgen (FP64, not rounded to FP32).  n x n column-major, lda >= n.
 * Used to build FP64 forward-error references. */
mxp_status mxp_matgen_f64(int n, uint64_t seed, int diag_rule, double *d_A, int64_t lda,
                          void *stream);

/* ---- granular LU pieces ----------------------------------------------- */

/* GPUSOLVER_SGETRF(h, b, b, A, lda, work, NULL, info) (panel_trf.hpp:
 * 547-551, 678-681): in-place FP32 no-pivot LU of an n x n block.  A zero
 * or non-finite pivot is reported through the workspace status. */
mxp_status mxp_getrf_nopiv(int n, float *d_A, int64_t lda, mxp_workspace *ws, void *stream);

/* GETRF followed by the inverses of both triangles, the operands of the
 * tensor-core TRSM-by-inverse (the reference's -alt path builds the same
 * inverses with STRSM on an identity, panel_trf_gdirect.hpp:73-92):
 * A (n x n) is factored in place, inv(U) -> d_XU and inv(L) (unit lower)
 * -> d_XL, both n x n with leading dimension ldx.  n <= the workspace's b. */
mxp_status mxp_getrf_nopiv_inv(int n, float *d_A, int64_t lda, float *d_XU, float *d_XL, int64_t ldx,
                               mxp_workspace *ws, void *stream);

/* update_left_panels_wGPU (panel_trf.hpp:188-207):
 * STRSM(Right, Upper, NoTrans, NonUnit): B(m x n) <- B * U^{-1}. */
mxp_status mxp_trsm_right_upper(int m, int n, const float *d_U, int64_t ldu, float *d_B,
                                int64_t ldb, void *stream);

/* update_right_panels_wGPU (panel_trf.hpp:225-246):
 * STRSM(Left, Lower, NoTrans, Unit): B(m x n) <- L^{-1} * B. */
mxp_status mxp_trsm_left_lower_unit(int m, int n, const float *d_L, int64_t ldl, float *d_B,
                                    int64_t ldb, void *stream);

/* update_left_panels_wGPU_alt / update_right_panels_wGPU_alt
 * (panel_trf_gdirect.hpp:73-142), the reference's Alt-TRSM: the panel solve
 * as a product with the triangle's inverse (from mxp_getrf_nopiv_inv) on the
 * tensor cores, in place.  right_upper: B (m x b) <- B * X_U; left_lower:
 * B (b x m) <- X_L * B.  single != 0: both operands rounded to BF16 once (the
 * reference rounds them to FP16); 0: three split-BF16 products (hi*hi + hi*lo
 * + lo*hi, near FP32).  FP32 accumulation; zero blocks of the triangular
 * inverse are skipped.  b <= the workspace's b and m <= its n - b.  Async. */
mxp_status mxp_trsm_inv_right_upper(int m, int b, const float *d_XU, int64_t ldx, float *d_B, int64_t ldb,
                                    int single, mxp_workspace *ws, void *stream);
mxp_status mxp_trsm_inv_left_lower(int b, int m, const float *d_XL, int64_t ldx, float *d_B, int64_t ldb,
                                   int single, mxp_workspace *ws, void *stream);

/* half_conversion_left (fp16_gpu_kernels.h:26-27, .cpp:180-192): FP32 m x b
 * block (column-major, plda) -> FP16 column-major (lplda), round to nearest.
 * Reference layout; bit-exact with copyCoalesced. */
mxp_status mxp_half_conversion_left(const float *d_C, int m, int b, int64_t plda, uint16_t *d_lp,
                                    int64_t lplda, void *stream);

/* half_conversion_right_trans (fp16_gpu_kernels.h:28-29, .cpp:196-211):
 * FP32 b x m block (plda) -> FP16 transposed, rp[k*rplda + j] = C(k, j).
 * Reference layout; bit-exact with transposeCoalesced. */
mxp_status mxp_half_conversion_right_trans(const float *d_C, int b, int m, int64_t plda,
                                           uint16_t *d_rp, int64_t rplda, void *stream);

/* Panel casts in the layout the tcgen05 Schur kernel reads: K-major rows
 * (row i holds its K values contiguously, ld = ldk elements).
 *  left : L column panel, FP32 m x b column-major (lda)   -> m rows
 *  right: U row panel,    FP32 b x m column-major (lda)   -> m rows (= U^T)
 * form FP16: K = b, 2-byte elements.  BF16X2: K = 3b (hi|hi|lo for left,
 * hi|lo|hi for right).  FP8: K = b, 1-byte elements, plus one UE8M0 scale
 * byte per 128 x 128 tile in d_scales (row-tile major, ceil(m/128) x
 * ceil(b/128)).  Replaces convert_left/right_panels_wGPU (panel_trf.hpp:
 * 258-277, 305-325). */
mxp_status mxp_panel_cast_left(int form, int m, int b, const float *d_A, int64_t lda, void *d_out,
                               int64_t ldk, uint8_t *d_scales, void *stream);
mxp_status mxp_panel_cast_right(int form, int m, int b, const float *d_A, int64_t lda, void *d_out,
                                int64_t ldk, uint8_t *d_scales, void *stream);

/* GPUBLAS_SGEMM_EX(OP_N, OP_T, m, n, k, -1, L, lda, R, ldb, 1, C, ldc)
 * (panel_trf.hpp:828-834, rocm_device_macros.h:267-268): C(m x n, FP32,
 * column-major) -= L * R^T on tcgen05 tensor cores, FP32 accumulation.
 * L and R are K-major panels from mxp_panel_cast_*; k is the panel width b
 * (the kernel multiplies it by 3 for BF16X2).  Scales only for FP8. */
mxp_status mxp_schur_update(int form, int m, int n, int k, const void *d_L, int64_t ldl,
                            const uint8_t *d_lscales, const void *d_R, int64_t ldr,
                            const uint8_t *d_rscales, float *d_C, int64_t ldc,
                            mxp_workspace *ws, void *stream);

/* ---- whole LU ------------------------------------------------------------ */

/* panel_lu_async_wGPU (panel_trf.hpp:470-867) at a 1x1 grid: in-place
 * blocked no-pivot LU of the n x n FP32 matrix with block size b (n % b ==
 * 0), Schur update in the workspace's form.  Synchronises the stream at the
 * end to read the pivot status; fills stats when non-NULL. */
mxp_status mxp_panel_lu(int n, int b, float *d_A, int64_t lda, mxp_workspace *ws, void *stream,
                        mxp_lu_stats *stats);

/* ---- refinement ------------------------------------------------------------ */

/* otf_gemv_h / panel_gemv_h (panel_gemv.hpp:83-179): y = beta*y +
 * alpha*A*x with a_ij regenerated from the LCG in FP64 (never read from
 * memory) and the diagonal taken from d.  Deterministic. */
mxp_status mxp_otf_gemv(int n, uint64_t seed, const double *d_d, double alpha, const double *d_x,
                        double beta, double *d_y, mxp_workspace *ws, void *stream);

/* No counterpart in the reference.  mxp_otf_gemv for callers that cannot
 * allocate device memory or own a workspace (code placed inside an existing
 * refinement loop that only holds raw vector pointers, or applications that
 * forbid device allocation after start-up because cudaMalloc / cudaFree can
 * synchronise the whole device).  Same result as mxp_otf_gemv within FP64
 * rounding; the split partial sums live in a fixed 4 MiB device array inside
 * the library, reserved on every GPU that loads it until the process exits.
 * Limit: n <= 262144, larger n returns MXP_INVALID_ARG.  The first call on a
 * device resolves the array's address (make it before any stream capture).
 * The stream must belong to the current device (another device's stream
 * returns MXP_INVALID_ARG).  All calls share the array: calls that overlap
 * on the GPU race. */
mxp_status mxp_otf_gemv_noalloc(int n, uint64_t seed, const double *d_d, double alpha,
                                const double *d_x, double beta, double *d_y, void *stream);

/* ---- Higham's HPL-AI matrix --------------------------------------------- */

/* higham_mat_comp_beta (higham_mat_impl.cpp:98-130) and HMGen's alpha =
 * rho * beta (highammgen.hpp:15-20): the parameters of Higham's matrix
 * A = L U (L unit lower with strictly lower entries alpha, U unit upper with
 * strictly upper entries beta) whose estimated cond(A, inf) is `cond`, by
 * bisection on Fasi and Higham's closed-form estimate.  Host only. */
mxp_status mxp_higham_params(int n, double cond, double rho, double *alpha, double *beta);

/* pmatgen(HMGen) + pdiaggen (matgen.hpp:157-208, 399-417): A(i,j) = beta +
 * ab*i above the diagonal, 1 + ab*i on it, alpha + ab*j below it (ab =
 * alpha*beta; FP32, formed from the FP32-rounded parameters by one fused
 * multiply-add each), d_i = 1 + ab*i (FP64), and the right-hand side from the
 * LCG stream of `seed` (column n, as panel_colvgen, matgen.hpp:419-436).
 * Any of d_A, d_d, d_rhs may be NULL. */
mxp_status mxp_matgen_higham(int n, double alpha, double beta, uint64_t seed, float *d_A, int64_t lda,
                             double *d_d, double *d_rhs, void *stream);

/* otf_gemv for HMGen (panel_gemv.hpp:362-388; hmg_gemv_up / hmg_gemv_low /
 * hmg_gemv_diag, otf_gemv.cpp:135-316): y = b*y + a*A*x with the entries of
 * Higham's matrix regenerated in FP64 (never read), every row summed in
 * column order with fused multiply-adds.  The diagonal blocks use the
 * generator's entries (the reference's hmg_gemv_diag swaps alpha and beta
 * there).  Deterministic. */
mxp_status mxp_higham_gemv(int n, double alpha, double beta, double a, const double *d_x, double b,
                           double *d_y, void *stream);

/* higham_infnorm (panel_norm.hpp:136-175): ||A||_inf of Higham's matrix (all
 * entries are positive: the largest row sum).  Host only. */
mxp_status mxp_higham_infnorm(int n, double alpha, double beta, double *h_out);

/* The refinement of this workspace (mxp_iterative_refinement, mxp_solve,
 * mxp_solve_host) regenerates Higham's matrix with these parameters instead
 * of the LCG matrix of the seed, and takes ||A||_inf from
 * mxp_higham_infnorm when its norma argument is <= 0.  alpha = beta = 0
 * goes back to the LCG matrix.  (The reference's HMGen overloads of
 * otf_gemv / higham_infnorm, templated on the generator type.) */
mxp_status mxp_workspace_set_matrix_higham(mxp_workspace *ws, double alpha, double beta);

/* trsvL_h + trsvU_h (panel_trsv.hpp:308-597): x <- U^{-1} L^{-1} x with
 * the FP32 factors of mxp_panel_lu, vectors in FP64, block substitution.
 * When d_LU, n and lda are those of the last successful mxp_panel_lu on this
 * workspace (and MXP_OPT_TRSV_INV is on), the diagonal blocks are solved
 * with the inverses that LU kept (a product, then one refinement step against
 * the factor block); a factor written into that buffer by other means must be
 * solved after MXP_OPT_TRSV_INV is set again (setting it, to either value,
 * forgets the stored inverses) or from another buffer.  Otherwise 64-row
 * blocks substitute exactly in FP64 along a chain.  Blocking: reads the
 * workspace status word (MXP_TIMEOUT when a bounded wait between row blocks
 * gave up). */
mxp_status mxp_lu_solve(int n, const float *d_LU, int64_t lda, double *d_x, mxp_workspace *ws,
                        void *stream);

/* iterative_refinement2, GPU branch (iterative_refinement.hpp:141-171):
 * x0 = rhs ./ d, then refine until the scaled residual
 * ||r||inf / (norma ||x||inf + normb) / (n eps/2) < 16 or maxit.
 * norma <= 0 selects 2*max(d) (hpl_infnorm, panel_norm.hpp:129-135) or,
 * with d_rowsum != NULL, max(rowsum + d).  method MXP_IR_CLASSIC corrects
 * with x += U^{-1} L^{-1} r; MXP_IR_GMRES solves the correction equation
 * with GMRES preconditioned by the LU (FP64 Arnoldi, CGS2, Givens on the GPU).
 * Blocking: returns when done. */
mxp_status mxp_iterative_refinement(int n, uint64_t seed, const float *d_LU, int64_t lda,
                                    const double *d_d, const double *d_rowsum,
                                    const double *d_rhs, double *d_x, double norma, int maxit,
                                    int method, mxp_workspace *ws, void *stream,
                                    mxp_ir_stats *stats);

/* The timed region of main.cpp:617-657 in one call: LU then refinement on
 * a matrix produced by mxp_matgen.  d_A is overwritten by the factors. */
mxp_status mxp_solve(int n, int b, uint64_t seed, float *d_A, int64_t lda, const double *d_d,
                     const double *d_rowsum, const double *d_rhs, double *d_x, int maxit,
                     int method, mxp_workspace *ws, void *stream, mxp_lu_stats *lu_stats,
                     mxp_ir_stats *ir_stats);

/* Host-buffer variant (the end-to-end call): rhs is read from host memory
 * and x written to host memory, both copies on the stream inside the call
 * and staged in the workspace (no allocation).  A, d (and rowsum for the
 * stress rule) are device-resident, produced by mxp_matgen as in the
 * reference's default -init 1 path (main.cpp:536-538).  Blocking. */
mxp_status mxp_solve_host(int n, int b, uint64_t seed, float *d_A, int64_t lda, const double *d_d,
                          const double *d_rowsum, const double *h_rhs, double *h_x, int maxit,
                          int method, mxp_workspace *ws, void *stream, mxp_lu_stats *lu_stats,
                          mxp_ir_stats *ir_stats);

/* ---- small utilities ------------------------------------------------------ */

/* ||x||_inf of a device FP64 vector (colv_infnorm_h, panel_norm.hpp:35-58).
 * Blocking. */
mxp_status mxp_infnorm(int n, const double *d_x, double *h_out, mxp_workspace *ws, void *stream);

/* Self-check of the branch-free FP32 reciprocal the 64 x 64 diagonal LU uses
 * for its pivots (no reference counterpart; the reference's sgetrf_nopiv_naive
 * divides by the pivot, sgetrf_nopiv.cpp:27-61, which is the same correctly
 * rounded value): compares it bit for bit with the CUDA runtime's IEEE
 * round-to-nearest reciprocal on 2 x 254 x 65536 normal inputs (every sign and
 * exponent, mantissas spread over the range plus the extremes).  h_mismatches
 * and h_checked receive the counts.  Blocking. */
mxp_status mxp_check_reciprocal(uint64_t *h_mismatches, uint64_t *h_checked);

/* Number of tcgen05 / other kernels this library launched on the calling
 * thread since the last reset (for launch accounting in benchmarks). */
int64_t mxp_kernel_launches(void);
void mxp_reset_kernel_launches(void);

/* ---- 2D block-cyclic process grid -----------------------------------------
 * Device pieces of the multi-GPU driver (openmxp_b200/grid.py; the
 * reference's panel_trf / iterative_refinement over a P x Q Grid, grid.hpp:
 * 25-80): global b x b block (I, J) lives on process (I mod P, J mod Q), kept
 * in one column-major local matrix at local block (I div P, J div Q).  The
 * LU steps use the granular entry points above on local views. */

/* Rows (or columns) of the local matrix of process coordinate me among nproc:
 * b times the number of block indices I < n/b with I mod nproc == me. */
mxp_status mxp_local_extent(int n, int b, int nproc, int me, int64_t *h_extent);

/* panel_matgen_dev for one process of a P x Q grid (matgen.hpp:84-117): its
 * local blocks of the generator matrix, bit-exact with mxp_matgen's, the
 * diagonal A(i,i) = float(d_i) taken from d_d (all n entries, as mxp_matgen
 * computes them).  lda >= the local row count. */
mxp_status mxp_matgen_local(int n, int b, uint64_t seed, int nprow, int npcol, int myrow, int mycol,
                            const double *d_d, float *d_A, int64_t lda, void *stream);

/* The per-process part of panel_gemv_h (panel_gemv.hpp:119-176), before the
 * sum across the process row (:177): for this process's rows i,
 * y_i += alpha * sum over its columns j of a_ij x_j, a_ij regenerated in FP64
 * (a_ii = d_i).  x, y and d are whole-length (n) device vectors; entries of y
 * outside this process's rows are left alone.  b <= 6144. */
mxp_status mxp_otf_gemv_local(int n, int b, uint64_t seed, int nprow, int npcol, int myrow, int mycol,
                              const double *d_d, double alpha, const double *d_x, double *d_y, void *stream);

/* HPLMXP_gemv (panel_trsv.hpp:13-225): y = beta y + alpha A x with A FP32
 * (m x n, column-major, lda) and x, y FP64; deterministic summation order. */
mxp_status mxp_block_gemv(int m, int n, double alpha, const float *d_A, int64_t lda, const double *d_x,
                          double beta, double *d_y, void *stream);

/* ---- batched form ----------------------------------------------------------
 * Many independent systems of uneven orders (each n a multiple of 128, at most
 * 8192), every one generated, factored and refined exactly as the single-system
 * path does (diagonal rule: row sum), all in ONE persistent kernel launch that
 * is captured once in a CUDA graph and replayed.  The reference has no batched
 * entry point: it solves one system per job (main.cpp:617-657); this is that
 * solve repeated over a batch.  Storage is packed: system i's column-major
 * matrix starts at float offset a_off[i] of A (lda = n[i]) and its vectors at
 * double offset v_off[i] of d, rhs and x (mxp_batch_layout gives both). */
typedef struct mxp_batch mxp_batch;

typedef struct {
    int iterations;      /* refinement corrections applied */
    int converged;       /* 1 when the scaled residual went below 16 */
    int info;            /* first zero pivot (1-based) or 0 */
    int pad;
    double hpl_harness;  /* final scaled residual */
    double residual;     /* final ||b - A x||_inf */
} mxp_batch_result;

typedef struct {
    double ms_total;     /* device time of the launch */
    int b, tile_n, stages;
    int autotuned;
    int grid;
} mxp_batch_stats;

/* Orders of a batch drawn from the generator stream of size_seed: value i,
 * v in [-0.5, 0.5], gives n = 128 * (2 + floor((v + 0.5) * 31)). */
mxp_status mxp_batch_sizes(int count, uint64_t size_seed, int *h_n);
/* Split a batch over nparts GPUs (no reference counterpart: the reference
 * solves one system per job).  Systems are independent, so each part is
 * solved by its own mxp_batch with no exchange between GPUs; the parts are
 * balanced by the LU work n^3: largest first, each to the part with the least
 * work so far (ties to the lower part).  Deterministic, so every rank computes
 * the same split.  h_part[i] in [0, nparts). */
mxp_status mxp_batch_partition(int count, const int *h_n, int nparts, int *h_part);
mxp_status mxp_batch_create(int count, const int *h_n, const uint64_t *h_seed, int device, mxp_batch **out);
mxp_status mxp_batch_destroy(mxp_batch *bt);
mxp_status mxp_batch_layout(const mxp_batch *bt, int64_t *matrix_floats, int64_t *vector_doubles,
                            int64_t *h_a_off, int64_t *h_v_off);
/* panel_matgen_dev + panel_colvgen for every system (matgen.hpp:84-117, 419-436) */
mxp_status mxp_batch_matgen(mxp_batch *bt, float *d_A, double *d_d, double *d_rhs, void *stream);
/* block size b in {64, 128, 256}, Schur tile width tile_n in {128, 256}, smem
 * pipeline depth stages in 2..4 within 227 KB of shared memory (default 128 / 256 / 3) */
mxp_status mxp_batch_set_config(mxp_batch *bt, int b, int tile_n, int stages);
/* times every admissible configuration on `sample` systems (0: an eighth of
 * the batch, spread over the sizes; those matrices are regenerated and
 * overwritten) and keeps the fastest */
mxp_status mxp_batch_autotune(mxp_batch *bt, float *d_A, double *d_d, double *d_rhs, double *d_x, int sample,
                              void *stream, mxp_batch_stats *stats);
/* LU + classic refinement of every system; A is overwritten by the factors,
 * x receives the solutions.  Blocking (reads the status word). */
mxp_status mxp_batch_solve(mxp_batch *bt, float *d_A, const double *d_d, const double *d_rhs, double *d_x,
                           int maxit, void *stream, mxp_batch_stats *stats);
mxp_status mxp_batch_results(const mxp_batch *bt, mxp_batch_result *h_results);

#ifdef __cplusplus
}
#endif

#endif /* MXP_H */
