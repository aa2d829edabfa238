// Host driver and C ABI of libmxp.
//
// mxp_panel_lu is the single-GPU (1x1 grid) form of panel_lu_async_wGPU
// (panel_trf.hpp:470-867): the reference's broadcasts of the diagonal
// factor and of the FP16 panels (broadcast_pivlu_wGPU, broadcast_left/
// right_panels, :63-170) and its per-step host copies of the panels become
// on-device hand-offs: the cast kernels write the panels straight into the
// buffers the Schur kernel reads.  All calls are stream-ordered; the only
// synchronisation of the LU is the final read of the device status word.
//
// mxp_iterative_refinement follows the GPU branch of iterative_refinement2
// (iterative_refinement.hpp:141-171); its one host synchronisation per step
// is the 16-byte read of ||x|| and ||r|| needed for the stopping test.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <string>
#include <vector>

#include "mxp_internal.cuh"

// ---------------------------------------------------------------------------
// status plumbing
// ---------------------------------------------------------------------------
namespace mxp {

static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }

mxp_status fail(mxp_status st, const std::string &msg) {
    g_last_error = msg;
    return st;
}

mxp_status cuda_fail(cudaError_t e, const char *where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return MXP_CUDA_ERROR;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int num_sms() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

}  // namespace mxp

using namespace mxp;

namespace mxp {
mxp_status launch_higham_gemv(int n, double alpha, double beta, double a, const double *x, double b, double *y,
                              cudaStream_t st);
double higham_infnorm(int n, double alpha, double beta);
int gmres_dot_blocks(int n);
mxp_status launch_mdot(int n, int nv, const double *V, int64_t ldv, const double *w,
                       double *partial, double *out, int accumulate, cudaStream_t st);
mxp_status launch_vsub(int n, int nv, const double *V, int64_t ldv, const double *h, double *w,
                       cudaStream_t st);
mxp_status launch_vadd(int n, int nv, const double *V, int64_t ldv, const double *c, double *y,
                       cudaStream_t st);
mxp_status launch_vdiv(int n, const double *src, const double *den, double *dst, cudaStream_t st);
mxp_status launch_givens(int j, double *H, int ldh, const double *hcol, const double *hnext,
                         double *cs, double *sn, double *g, double *resid_out, cudaStream_t st);
mxp_status launch_backsolve(int k, const double *H, int ldh, const double *g, double *y,
                            cudaStream_t st);
mxp_status launch_set_g0(int m, double *g, const double *beta, cudaStream_t st);
mxp_status launch_sqrt(const double *in, double *out, cudaStream_t st);
}  // namespace mxp

// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------
// Panel slots of the workspace buffers: at most this many panels per trailing
// pass (K = kMaxMerge * b).
constexpr int kMaxMerge = 4;

struct mxp_workspace {
    int n = 0, b = 0, form = 0, device = 0;
    int64_t ldk = 0;         // K-major panel row stride (elements): kMaxMerge panel slots side by side
    int64_t kp = 0;          // K extent of one panel (b, or 3b for BF16X2)
    int sc_ld = 0;           // FP8 scale-table row stride (tiles): kMaxMerge panel slots side by side
    int merge = kMaxMerge;   // panels per trailing pass (merged look-ahead), 1..kMaxMerge
    int pair = 0;            // trailing Schur products on the 2-SM (cta_group::2) kernel
    int trsm_pair = 0;       // TRSM-by-inverse products on the 2-SM kernel
    int withhold = -1;       // test: row block whose TRSV flag the next mxp_lu_solve withholds
    // diagonal factorisation of the next pair overlapped with the trailing pass
    int overlap = 0;         // SMs given to it (0: off)
    int overlap_min = 6;     // minimum trailing size, in blocks
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_inv[2] = {nullptr, nullptr};  // fork / join of the two inverse chains
    int *tile_ctr = nullptr;  // shared tile counter of the split trailing pass
    int *trsm_ctr = nullptr;  // tile counter of the TRSM-by-inverse products (claimed dynamically)
    int trsm_counter = 1;     // TRSM products take tiles from trsm_ctr (0: static round robin)
    // matrix the refinement's residual regenerates: the LCG matrix of the
    // seed (default) or Higham's matrix with parameters (h_alpha, h_beta)
    int higham = 0;
    double h_alpha = 0.0, h_beta = 0.0;
    size_t esize = 2;        // panel element size
    void *lpanel[2] = {nullptr, nullptr};
    void *rpanel[2] = {nullptr, nullptr};
    uint8_t *lscale[2] = {nullptr, nullptr};
    uint8_t *rscale[2] = {nullptr, nullptr};
    DevStatus *status = nullptr;
    double *vec = nullptr;   // IR vectors: r, w, x, rhs | gemv partials | scalars
    double *r = nullptr, *w = nullptr, *xv = nullptr, *rhsv = nullptr;
    double *partials = nullptr, *scal = nullptr;
    int max_splits = 16;
    int *flags = nullptr;
    // tensor-core panel TRSM: FP32 triangular inverses and split-BF16 operands
    int trsm_tc = 1;
    int trsm_single = 0;     // one BF16 product instead of three split products
    int fp8_fused = 1;       // FP8 form: the L panel's E4M3 copy written by the TRSM product's epilogue
    int inv_tc = 1024;       // inverse doubling levels from this block size on the tensor cores (0: none)
    int64_t ldk3 = 0;
    float *tinv_u = nullptr, *tinv_l = nullptr, *tinv_tmp = nullptr;
    // inverses of every diagonal block kept for the refinement's triangular
    // solves: block k's inv(U_kk) at inv_store + 2k*b*b, inv(L_kk) after it
    int trsv_inv = 1;
    int inv_blocks = 0;
    float *inv_store = nullptr;
    double *trsv_t = nullptr;             // 4 b doubles
    cudaEvent_t ev_trsv[4] = {nullptr, nullptr, nullptr, nullptr};  // two-stream refinement solves
    const float *inv_lu = nullptr;        // factor the stored inverses belong to (nullptr: none)
    int inv_n = 0;
    int64_t inv_lda = 0;
    // cooperative diagonal-block factorisation (LU + inverses in one launch)
    int coop = 1;
    float *coop_tmp = nullptr;          // 2 x diag_factor_tmp_floats(b)
    unsigned int *coop_sync = nullptr;  // grid-barrier counter + abort word
    void *split_big = nullptr, *split_u = nullptr, *split_l = nullptr;
    // GMRES-IR: basis V ((m+1) x n), Hessenberg H ((m+1) x m), rotations, scalars
    int gm_m = 30;
    double gm_tol = 1e-10;
    double *gV = nullptr, *gH = nullptr, *gsmall = nullptr, *gpart = nullptr;
    double *h_scal = nullptr;  // pinned host scalars
    // timing events, created once: the refinement's six, and a pool the LU
    // phase marks and the GMRES regions draw from (grown on first use only)
    cudaEvent_t ev_ir[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> ev_pool;
    std::vector<void *> allocs;
};

// Event i of the workspace's pool (created the first time it is asked for).
static cudaEvent_t pool_event(mxp_workspace *ws, size_t i) {
    while (ws->ev_pool.size() <= i) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ws->ev_pool.push_back(e);
    }
    return ws->ev_pool[i];
}

static int64_t panel_ldk(int b, int form) {
    const int64_t K = form == MXP_FORM_BF16X2 ? 3 * (int64_t)b : b;
    const int64_t esize = form == MXP_FORM_FP8 ? 1 : 2;
    const int64_t align = 16 / esize;
    return (K + align - 1) / align * align;
}

static size_t trsm_bytes(int n, int b) {
    const int64_t ldk3 = panel_ldk(b, MXP_FORM_BF16X2);
    const int64_t rows = n > b ? n - b : 1;
    return 2 * (size_t)b * b * 4 + ((size_t)b * b / 4 + 64 * (size_t)b) * 4 +
           (size_t)(rows + 2 * (int64_t)b) * ldk3 * 2 + 4096 + 2 * diag_factor_tmp_floats(b) * 4 + 256;
}

// Stored inverses of the diagonal blocks: 2 x (n / b) blocks of b x b floats.
static size_t inv_store_bytes(int n, int b) { return 2 * (size_t)(n / b) * b * b * 4 + 256; }

static size_t ws_layout(int n, int b, int form, size_t *panel_bytes, size_t *scale_bytes,
                        size_t *vec_doubles, size_t *flag_ints) {
    const int64_t ldk = panel_ldk(b, form);
    const int64_t esize = form == MXP_FORM_FP8 ? 1 : 2;
    const int64_t rows = n > b ? n - b : 1;
    *panel_bytes = (size_t)(rows * kMaxMerge * ldk * esize + 1024) / 256 * 256 + 256;
    *scale_bytes = (size_t)(cdiv(rows, 128) * kMaxMerge * cdiv(b, 128) + 256) / 256 * 256 + 256;
    *vec_doubles = (size_t)n * (4 + 16) + 64;
    *flag_ints = lu_solve_flag_ints(n) + 64;
    *vec_doubles += (size_t)31 * n + 64 * 32 + 2 * 31 * 64 + 31 * (size_t)(2 * 148 + 2) + 1024;
    return 2 * *panel_bytes + 2 * *scale_bytes + *vec_doubles * 8 + *flag_ints * 4 + 256 +
           trsm_bytes(n, b) + inv_store_bytes(n, b) + (size_t)4 * b * 8 + 256;
}

extern "C" size_t mxp_workspace_bytes(int n, int b, int form) {
    size_t pb, sb, vd, fi;
    if (n <= 0 || b <= 0) return 0;
    return ws_layout(n, b, form, &pb, &sb, &vd, &fi);
}

extern "C" mxp_status mxp_workspace_destroy(mxp_workspace *ws) {
    if (!ws) return MXP_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(ws->device);
    if (ws->side) cudaStreamSynchronize(ws->side);
    for (void *p : ws->allocs) cudaFree(p);
    if (ws->h_scal) cudaFreeHost(ws->h_scal);
    if (ws->ev_fork) cudaEventDestroy(ws->ev_fork);
    if (ws->ev_join) cudaEventDestroy(ws->ev_join);
    for (cudaEvent_t e : ws->ev_trsv)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ws->ev_inv)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ws->ev_ir)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ws->ev_pool)
        if (e) cudaEventDestroy(e);
    if (ws->side) cudaStreamDestroy(ws->side);
    cudaSetDevice(cur);
    delete ws;
    return MXP_OK;
}

extern "C" mxp_status mxp_workspace_create(int n, int b, int form, int device, mxp_workspace **out) {
    if (!out) return fail(MXP_INVALID_ARG, "workspace_create: out is NULL");
    *out = nullptr;
    if (n <= 0 || b <= 0 || b > n) return fail(MXP_INVALID_ARG, "workspace_create: bad n/b");
    if (form != MXP_FORM_FP16 && form != MXP_FORM_BF16X2 && form != MXP_FORM_FP8)
        return fail(MXP_INVALID_ARG, "workspace_create: unknown form");
    int cur = 0;
    MXP_CUDA(cudaGetDevice(&cur));
    MXP_CUDA(cudaSetDevice(device));
    mxp_workspace *ws = new mxp_workspace();
    ws->n = n;
    ws->b = b;
    ws->form = form;
    ws->device = device;
    ws->kp = form == MXP_FORM_BF16X2 ? 3 * (int64_t)b : b;
    ws->ldk = kMaxMerge * panel_ldk(b, form);
    ws->sc_ld = kMaxMerge * (int)cdiv(b, 128);
    ws->esize = form == MXP_FORM_FP8 ? 1 : 2;
    size_t pb, sb, vd, fi;
    ws_layout(n, b, form, &pb, &sb, &vd, &fi);
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        ws->allocs.push_back(p);
        return p;
    };
    bool ok = true;
    ok = (ws->lpanel[0] = alloc(pb)) && (ws->rpanel[0] = alloc(pb)) &&
         (ws->lscale[0] = (uint8_t *)alloc(sb)) && (ws->rscale[0] = (uint8_t *)alloc(sb));
    ok = ok && (ws->status = (DevStatus *)alloc(sizeof(DevStatus) * 4));
    ok = ok && (ws->vec = (double *)alloc(vd * sizeof(double)));
    ok = ok && (ws->flags = (int *)alloc(fi * sizeof(int)));
    ws->ldk3 = panel_ldk(b, MXP_FORM_BF16X2);
    {
        const int64_t rows = n > b ? n - b : 1;
        ok = ok && (ws->tinv_u = (float *)alloc((size_t)b * b * 4));
        ok = ok && (ws->tinv_l = (float *)alloc((size_t)b * b * 4));
        ok = ok && (ws->tinv_tmp = (float *)alloc(((size_t)b * b / 4 + 64 * (size_t)b) * 4));
        ok = ok && (ws->coop_tmp = (float *)alloc(2 * diag_factor_tmp_floats(b) * 4));
        ok = ok && (ws->coop_sync = (unsigned int *)alloc(256));
        if (ok) ws->tile_ctr = reinterpret_cast<int *>(ws->coop_sync + 32);
        if (ok) ws->trsm_ctr = reinterpret_cast<int *>(ws->coop_sync + 33);
        ok = ok && (ws->split_big = alloc((size_t)rows * ws->ldk3 * 2 + 1024));
        ok = ok && (ws->split_u = alloc((size_t)b * ws->ldk3 * 2 + 1024));
        ok = ok && (ws->split_l = alloc((size_t)b * ws->ldk3 * 2 + 1024));
        ws->inv_blocks = n / b;
        ok = ok && (ws->inv_store = (float *)alloc(inv_store_bytes(n, b)));
        ok = ok && (ws->trsv_t = (double *)alloc((size_t)4 * b * 8 + 256));
    }
    if (ok) ok = cudaMallocHost(&ws->h_scal, 64 * sizeof(double)) == cudaSuccess;
    if (ok) {
        int least = 0, greatest = 0;
        ok = cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess &&
             cudaStreamCreateWithPriority(&ws->side, cudaStreamNonBlocking, greatest) == cudaSuccess &&
             cudaEventCreateWithFlags(&ws->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&ws->ev_join, cudaEventDisableTiming) == cudaSuccess;
        for (int e = 0; e < 4 && ok; ++e)
            ok = cudaEventCreateWithFlags(&ws->ev_trsv[e], cudaEventDisableTiming) == cudaSuccess;
        for (int e = 0; e < 2 && ok; ++e)
            ok = cudaEventCreateWithFlags(&ws->ev_inv[e], cudaEventDisableTiming) == cudaSuccess;
        for (int e = 0; e < 6 && ok; ++e) ok = cudaEventCreate(&ws->ev_ir[e]) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        mxp_workspace_destroy(ws);
        cudaSetDevice(cur);
        return fail(MXP_NO_MEMORY, "workspace_create: device allocation failed");
    }
    ws->r = ws->vec;
    ws->w = ws->vec + n;
    ws->xv = ws->vec + 2 * (size_t)n;
    ws->rhsv = ws->vec + 3 * (size_t)n;
    ws->partials = ws->vec + 4 * (size_t)n;
    ws->scal = ws->vec + 20 * (size_t)n;
    ws->gV = ws->vec + 20 * (size_t)n + 64;
    ws->gH = ws->gV + 31 * (size_t)n;             // 31 x 30 (ldh 31), padded to 64*32
    ws->gsmall = ws->gH + 64 * 32;                 // cs, sn, g, y, hcol, hcol2, scalars
    ws->gpart = ws->gsmall + 2 * 31 * 64;          // dot partials
    cudaMemset(ws->status, 0, sizeof(DevStatus) * 4);
    cudaMemset(ws->flags, 0, fi * sizeof(int));
    cudaDeviceSynchronize();
    cudaSetDevice(cur);
    *out = ws;
    return MXP_OK;
}

extern "C" mxp_status mxp_workspace_set_option(mxp_workspace *ws, int key, int value) {
    if (!ws) return fail(MXP_INVALID_ARG, "set_option: workspace is NULL");
    switch (key) {
        case MXP_OPT_TRSM_TENSOR:
            ws->trsm_tc = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_MERGE_PANELS:
            ws->merge = value ? kMaxMerge : 1;
            return MXP_OK;
        case MXP_OPT_MERGE_DEPTH:
            if (value < 1 || value > kMaxMerge) return fail(MXP_INVALID_ARG, "set_option: merge depth must be 1..4");
            ws->merge = value;
            return MXP_OK;
        case MXP_OPT_SCHUR_PAIR:
            ws->pair = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_DIAG_COOP:
            ws->coop = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_TRSM_PAIR:
            ws->trsm_pair = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_TEST_WITHHOLD_FLAG:
            ws->withhold = value;
            return MXP_OK;
        case MXP_OPT_OVERLAP_DIAG:
            if (value < 0 || value > num_sms() / 2)
                return fail(MXP_INVALID_ARG, "set_option: overlap SMs must be 0..half the SM count");
            ws->overlap = value;
            return MXP_OK;
        case MXP_OPT_TRSM_SINGLE:
            ws->trsm_single = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_INV_TC:
            if (value != 0 && (value < 128 || (value & (value - 1)) != 0))
                return fail(MXP_INVALID_ARG, "set_option: inverse level must be 0 or a power of two >= 128");
            ws->inv_tc = value;
            return MXP_OK;
        case MXP_OPT_FP8_FUSED_CAST:
            ws->fp8_fused = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_TRSM_COUNTER:
            ws->trsm_counter = value ? 1 : 0;
            return MXP_OK;
        case MXP_OPT_TRSV_INV:
            ws->trsv_inv = value ? 1 : 0;
            ws->inv_lu = nullptr;  // setting it forgets the stored inverses
            return MXP_OK;
        case MXP_OPT_OVERLAP_MIN:
            if (value < 2) return fail(MXP_INVALID_ARG, "set_option: overlap minimum must be >= 2 blocks");
            ws->overlap_min = value;
            return MXP_OK;
        case MXP_OPT_GMRES_RESTART:
            if (value < 1 || value > 30) return fail(MXP_INVALID_ARG, "set_option: GMRES restart must be 1..30");
            ws->gm_m = value;
            return MXP_OK;
        case MXP_OPT_GMRES_TOL_EXP:
            if (value < 1 || value > 15) return fail(MXP_INVALID_ARG, "set_option: GMRES tolerance exponent must be 1..15");
            ws->gm_tol = std::pow(10.0, -value);
            return MXP_OK;
        default:
            return fail(MXP_INVALID_ARG, "set_option: unknown key");
    }
}

extern "C" mxp_status mxp_workspace_set_matrix_higham(mxp_workspace *ws, double alpha, double beta) {
    if (!ws) return fail(MXP_INVALID_ARG, "set_matrix_higham: workspace is NULL");
    if (alpha == 0.0 && beta == 0.0) {
        ws->higham = 0;
        return MXP_OK;
    }
    if (!(alpha > 0.0) || !(beta > 0.0) || !std::isfinite(alpha) || !std::isfinite(beta))
        return fail(MXP_INVALID_ARG, "set_matrix_higham: alpha and beta must be positive (both 0: back to the LCG)");
    ws->higham = 1;
    ws->h_alpha = alpha;
    ws->h_beta = beta;
    return MXP_OK;
}

extern "C" mxp_status mxp_workspace_panel_view(const mxp_workspace *ws, int side, mxp_panel_view *out) {
    if (!ws || !out) return fail(MXP_INVALID_ARG, "panel_view: NULL argument");
    if (side != 0 && side != 1) return fail(MXP_INVALID_ARG, "panel_view: side must be 0 (L) or 1 (R)");
    const bool fp8 = ws->form == MXP_FORM_FP8;
    out->data = side ? ws->rpanel[0] : ws->lpanel[0];
    out->ld = ws->ldk;
    out->slot_k = ws->kp;
    out->esize = (int)ws->esize;
    out->slots = kMaxMerge;
    out->rows = ws->n > ws->b ? ws->n - ws->b : 1;
    out->scales = fp8 ? (side ? ws->rscale[0] : ws->lscale[0]) : nullptr;
    out->sc_ld = fp8 ? ws->sc_ld : 0;
    out->sc_slot = fp8 ? (int)cdiv(ws->b, 128) : 0;
    return MXP_OK;
}

// Read and clear the device status word; synchronises the stream.
static mxp_status read_status(mxp_workspace *ws, cudaStream_t st, DevStatus *out = nullptr) {
    DevStatus h;
    MXP_CUDA(cudaMemcpyAsync(&h, ws->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
    MXP_CUDA(cudaStreamSynchronize(st));
    if (out) *out = h;
    if (h.code != 0) {
        char buf[160];
        snprintf(buf, sizeof buf, "device status %d (detail %d, %d)", h.code, h.info0, h.info1);
        MXP_CUDA(cudaMemsetAsync(ws->status, 0, sizeof(DevStatus), st));
        return fail((mxp_status)h.code, buf);
    }
    return MXP_OK;
}

// ---------------------------------------------------------------------------
// simple entry points
// ---------------------------------------------------------------------------
extern "C" const char *mxp_version(void) { return "openmxp_b200 0.1 (sm_100a)"; }
extern "C" const char *mxp_last_error_string(void) { return g_last_error.c_str(); }
extern "C" int64_t mxp_kernel_launches(void) { return g_launches.load(); }
extern "C" void mxp_reset_kernel_launches(void) { g_launches.store(0); }

extern "C" mxp_status mxp_matgen(int n, uint64_t seed, int diag_rule, float *d_A, int64_t lda,
                                 double *d_d, double *d_rowsum, double *d_rhs, void *stream) {
    return launch_matgen(n, seed, diag_rule, d_A, lda, d_d, d_rowsum, d_rhs, as_stream(stream));
}

extern "C" mxp_status mxp_matgen_f64(int n, uint64_t seed, int diag_rule, double *d_A, int64_t lda,
                                     void *stream) {
    return launch_matgen_f64(n, seed, diag_rule, d_A, lda, as_stream(stream));
}

// The doubling levels of the triangular inverses from blocks of size s_start
// up, as tensor-core products (the cooperative kernel stops before them): for
// adjacent diagonal blocks of sizes S and s2, the off-diagonal block of
// inv(U) is -inv(U11) (U12 inv(U22)) and that of inv(L) is
// -inv(L22) (L21 inv(L11)), the same recursion as the kernel's SIMT levels.
// form: MXP_FORM_BF16X2 (three split products, near FP32) or kFormBf16 (one
// product).  T: S * s2 floats of scratch; the operands go through the
// workspace's split buffers.
// The doubling levels of one triangle's inverse from s_start up, as
// tensor-core products in `form` (split BF16 or one BF16 product) on stream
// `st`, with the operand casts in P and Q (each b rows x ldk3) and T as the
// level's temporary: for U, T = U12 inv(U22) then X12 = -inv(U11) T; for L,
// T = L21 inv(L11) then X21 = -inv(L22) T.
static mxp_status inverse_chain(bool upper, int n, const float *A, int64_t lda, float *X, int64_t ldx, int s_start,
                                int form, float *T, void *P, void *Q, mxp_workspace *ws, cudaStream_t st) {
    // C (m x nn) = P (m x K) Q (K x nn), or its negative; column-major FP32
    auto gemm = [&](int m, int nn, int K, const float *Pm, int64_t ldp, const float *Qm, int64_t ldq, float *C,
                    int64_t ldc, bool neg) -> mxp_status {
        mxp_status q = launch_cast_left(form, m, K, Pm, ldp, P, ws->ldk3, nullptr, st);
        if (q == MXP_OK) q = launch_cast_right(form, nn, K, Qm, ldq, Q, ws->ldk3, nullptr, st);
        if (q == MXP_OK)
            q = launch_schur(form, m, nn, K, P, ws->ldk3, nullptr, Q, ws->ldk3, nullptr, C, ldc, ws->status, st,
                             neg ? 2 : 1, 0, 0, 0, 0);
        return q;
    };
    mxp_status q = MXP_OK;
    for (int S = s_start; S < n && q == MXP_OK; S *= 2) {
        const int np = n / (2 * S);
        const int c = n - np * 2 * S - S;  // second block of a ragged last pair
        for (int p = 0; p <= np && q == MXP_OK; ++p) {
            const int s2 = p < np ? S : c;
            if (s2 <= 0) break;
            const int64_t r0 = (int64_t)p * 2 * S, r1 = r0 + S;
            if (upper) {
                q = gemm(S, s2, s2, A + r0 + r1 * lda, lda, X + r1 + r1 * ldx, ldx, T, S, false);
                if (q == MXP_OK) q = gemm(S, s2, S, X + r0 + r0 * ldx, ldx, T, S, X + r0 + r1 * ldx, ldx, true);
            } else {
                q = gemm(s2, S, S, A + r1 + r0 * lda, lda, X + r0 + r0 * ldx, ldx, T, s2, false);
                if (q == MXP_OK) q = gemm(s2, S, s2, X + r1 + r1 * ldx, ldx, T, s2, X + r1 + r0 * ldx, ldx, true);
            }
        }
    }
    return q;
}

// Both triangles' tensor-core levels.  The U and L chains share nothing, so
// when the workspace's panel-operand buffer has room for a second pair of
// operand casts (n >= 3b) the L chain runs on the side stream beside the U
// chain on `st` (each level is a few products on at most 32 tiles, far from
// filling the GPU), with its own temporary TL; otherwise one after the other.
// Either way every product is the same, so the inverses are bit-identical.
static mxp_status finish_inverses_tc(int n, const float *A, int64_t lda, float *XU, float *XL, int64_t ldx,
                                     int s_start, int form, float *T, float *TL, mxp_workspace *ws,
                                     cudaStream_t st) {
    const int64_t big_rows = ws->n > ws->b ? ws->n - ws->b : 1;
    const bool two = TL && ws->side && ws->ev_inv[0] && big_rows >= 2 * (int64_t)ws->b;
    if (!two) {
        mxp_status q = inverse_chain(true, n, A, lda, XU, ldx, s_start, form, T, ws->split_l, ws->split_u, ws, st);
        if (q == MXP_OK)
            q = inverse_chain(false, n, A, lda, XL, ldx, s_start, form, T, ws->split_l, ws->split_u, ws, st);
        return q;
    }
    uint8_t *big = (uint8_t *)ws->split_big;
    void *P2 = big, *Q2 = big + (size_t)ws->b * ws->ldk3 * 2;
    MXP_CUDA(cudaEventRecord(ws->ev_inv[0], st));
    MXP_CUDA(cudaStreamWaitEvent(ws->side, ws->ev_inv[0], 0));
    mxp_status qL = inverse_chain(false, n, A, lda, XL, ldx, s_start, form, TL, P2, Q2, ws, ws->side);
    mxp_status qU = inverse_chain(true, n, A, lda, XU, ldx, s_start, form, T, ws->split_l, ws->split_u, ws, st);
    // join even after an error, so nothing is left running on the side stream unseen
    MXP_CUDA(cudaEventRecord(ws->ev_inv[1], ws->side));
    MXP_CUDA(cudaStreamWaitEvent(st, ws->ev_inv[1], 0));
    return qU != MXP_OK ? qU : qL;
}

// Tensor-core inverse levels apply from this block size (0: none), when the
// block is large enough for them to matter and the split buffers hold it.
static int inv_tc_start(const mxp_workspace *ws, int n) {
    if (ws->inv_tc <= 0 || n > ws->b || 2 * ws->inv_tc > n) return 0;
    return ws->inv_tc;
}

extern "C" mxp_status mxp_getrf_nopiv(int n, float *d_A, int64_t lda, mxp_workspace *ws,
                                      void *stream) {
    if (!ws) return fail(MXP_INVALID_ARG, "getrf: workspace is NULL");
    cudaStream_t st = as_stream(stream);
    mxp_status s = ws->coop ? launch_diag_factor(n, d_A, lda, nullptr, nullptr, 0, nullptr, nullptr,
                                                 ws->coop_sync, ws->status, 0, st)
                            : launch_getrf_blocked(n, d_A, lda, ws->status, 0, st);
    if (s != MXP_OK) return s;
    return read_status(ws, st);
}

extern "C" mxp_status mxp_getrf_nopiv_inv(int n, float *d_A, int64_t lda, float *d_XU, float *d_XL,
                                          int64_t ldx, mxp_workspace *ws, void *stream) {
    if (!ws || !d_A || !d_XU || !d_XL) return fail(MXP_INVALID_ARG, "getrf_inv: NULL argument");
    if (n <= 0 || n > ws->b) return fail(MXP_INVALID_ARG, "getrf_inv: n must be in 1..b of the workspace");
    if (lda < n || ldx < n) return fail(MXP_INVALID_ARG, "getrf_inv: bad leading dimension");
    cudaStream_t st = as_stream(stream);
    mxp_status s;
    if (ws->coop) {
        const int tc = inv_tc_start(ws, n);
        s = launch_diag_factor(n, d_A, lda, d_XU, d_XL, ldx, ws->coop_tmp,
                               ws->coop_tmp + diag_factor_tmp_floats(ws->b), ws->coop_sync, ws->status, 0, st, 0,
                               tc);
        if (s == MXP_OK && tc > 0)
            s = finish_inverses_tc(n, d_A, lda, d_XU, d_XL, ldx, tc,
                                   ws->trsm_single ? kFormBf16 : MXP_FORM_BF16X2, ws->coop_tmp,
                                   ws->coop_tmp + diag_factor_tmp_floats(ws->b), ws, st);
    } else {
        s = launch_getrf_blocked(n, d_A, lda, ws->status, 0, st);
        if (s == MXP_OK) s = launch_tri_inv_upper(n, d_A, lda, d_XU, ldx, ws->tinv_tmp, st);
        if (s == MXP_OK) s = launch_tri_inv_lower_unit(n, d_A, lda, d_XL, ldx, ws->tinv_tmp, st);
    }
    if (s != MXP_OK) return s;
    return read_status(ws, st);
}

extern "C" mxp_status mxp_trsm_right_upper(int m, int n, const float *d_U, int64_t ldu, float *d_B,
                                           int64_t ldb, void *stream) {
    return launch_trsm_runn(m, n, d_U, ldu, d_B, ldb, as_stream(stream));
}

extern "C" mxp_status mxp_trsm_left_lower_unit(int m, int n, const float *d_L, int64_t ldl,
                                               float *d_B, int64_t ldb, void *stream) {
    return launch_trsm_llnu(m, n, d_L, ldl, d_B, ldb, as_stream(stream));
}

// TRSM by inverse on the tensor cores, one panel side at a time: the panel and
// the triangular inverse cast to BF16 (one product, single != 0) or split
// BF16 (hi*hi + hi*lo + lo*hi), then one store-mode product with the
// triangular K-skip, the panel overwritten in place (its cast is taken first).
// The same steps mxp_panel_lu runs per panel.
static mxp_status trsm_inv(bool right_upper, int m, int b, const float *X, int64_t ldx, float *B, int64_t ldb,
                           int single, mxp_workspace *ws, cudaStream_t st) {
    if (!ws || !X || !B) return fail(MXP_INVALID_ARG, "trsm_inv: NULL argument");
    if (m < 0 || b <= 0 || b > ws->b) return fail(MXP_INVALID_ARG, "trsm_inv: b must be in 1..b of the workspace");
    const int64_t big_rows = ws->n > ws->b ? ws->n - ws->b : 1;
    if (m > big_rows) return fail(MXP_INVALID_ARG, "trsm_inv: panel longer than the workspace's n - b");
    if (ldx < b || (right_upper ? ldb < m : ldb < b)) return fail(MXP_INVALID_ARG, "trsm_inv: bad leading dimension");
    if (m == 0) return MXP_OK;
    const int bf = single ? kFormBf16 : MXP_FORM_BF16X2;
    SchurSched ts;
    ts.counter = ws->trsm_ctr;
    mxp_status q;
    if (right_upper) {  // B (m x b) <- B * X, X upper
        q = launch_cast_left(bf, m, b, B, ldb, ws->split_big, ws->ldk3, nullptr, st);
        if (q == MXP_OK) q = launch_cast_right(bf, b, b, X, ldx, ws->split_u, ws->ldk3, nullptr, st);
        if (q == MXP_OK) MXP_CUDA(cudaMemsetAsync(ws->trsm_ctr, 0, sizeof(int), st));
        if (q == MXP_OK)
            q = launch_schur(bf, m, b, b, ws->split_big, ws->ldk3, nullptr, ws->split_u, ws->ldk3, nullptr, B, ldb,
                             ws->status, st, /*store=*/1, 0, 0, /*tri=*/1, 0, &ts);
    } else {            // B (b x m) <- X * B, X unit lower
        q = launch_cast_left(bf, b, b, X, ldx, ws->split_l, ws->ldk3, nullptr, st);
        if (q == MXP_OK) q = launch_cast_right(bf, m, b, B, ldb, ws->split_big, ws->ldk3, nullptr, st);
        if (q == MXP_OK) MXP_CUDA(cudaMemsetAsync(ws->trsm_ctr, 0, sizeof(int), st));
        if (q == MXP_OK)
            q = launch_schur(bf, b, m, b, ws->split_l, ws->ldk3, nullptr, ws->split_big, ws->ldk3, nullptr, B, ldb,
                             ws->status, st, /*store=*/1, 0, 0, /*tri=*/2, 0, &ts);
    }
    return q;
}

extern "C" mxp_status mxp_trsm_inv_right_upper(int m, int b, const float *d_XU, int64_t ldx, float *d_B,
                                               int64_t ldb, int single, mxp_workspace *ws, void *stream) {
    return trsm_inv(true, m, b, d_XU, ldx, d_B, ldb, single, ws, as_stream(stream));
}

extern "C" mxp_status mxp_trsm_inv_left_lower(int b, int m, const float *d_XL, int64_t ldx, float *d_B,
                                              int64_t ldb, int single, mxp_workspace *ws, void *stream) {
    return trsm_inv(false, m, b, d_XL, ldx, d_B, ldb, single, ws, as_stream(stream));
}

extern "C" mxp_status mxp_half_conversion_left(const float *d_C, int m, int b, int64_t plda,
                                               uint16_t *d_lp, int64_t lplda, void *stream) {
    return launch_half_left_ref(d_C, m, b, plda, d_lp, lplda, as_stream(stream));
}

extern "C" mxp_status mxp_half_conversion_right_trans(const float *d_C, int b, int m, int64_t plda,
                                                      uint16_t *d_rp, int64_t rplda, void *stream) {
    return launch_half_right_trans_ref(d_C, b, m, plda, d_rp, rplda, as_stream(stream));
}

extern "C" mxp_status mxp_panel_cast_left(int form, int m, int b, const float *d_A, int64_t lda,
                                          void *d_out, int64_t ldk, uint8_t *d_scales, void *stream) {
    return launch_cast_left(form, m, b, d_A, lda, d_out, ldk, d_scales, as_stream(stream));
}

extern "C" mxp_status mxp_panel_cast_right(int form, int m, int b, const float *d_A, int64_t lda,
                                           void *d_out, int64_t ldk, uint8_t *d_scales, void *stream) {
    return launch_cast_right(form, m, b, d_A, lda, d_out, ldk, d_scales, as_stream(stream));
}

extern "C" mxp_status mxp_schur_update(int form, int m, int n, int k, const void *d_L, int64_t ldl,
                                       const uint8_t *d_lscales, const void *d_R, int64_t ldr,
                                       const uint8_t *d_rscales, float *d_C, int64_t ldc,
                                       mxp_workspace *ws, void *stream) {
    if (!ws) return fail(MXP_INVALID_ARG, "schur: workspace is NULL");
    return launch_schur(form, m, n, k, d_L, ldl, d_lscales, d_R, ldr, d_rscales, d_C, ldc,
                        ws->status, as_stream(stream), 0, 0, 0, 0, ws->pair);
}

// ---------------------------------------------------------------------------
// LU
// ---------------------------------------------------------------------------
namespace {
// Phase marks on the solve stream, from the workspace's event pool (no event
// is created once the pool has grown to a solve's number of marks); read
// after the LU's final synchronisation.
struct PhaseTimer {
    bool on = false;
    cudaStream_t st = 0;
    mxp_workspace *ws = nullptr;
    std::vector<std::pair<cudaEvent_t, int>> marks;  // event, phase id after it
    void mark(int phase) {
        if (!on) return;
        cudaEvent_t e = pool_event(ws, marks.size());
        if (!e) return;
        cudaEventRecord(e, st);
        marks.push_back({e, phase});
    }
    // returns ms per phase id
    void collect(double *ms, int nphase) {
        for (int i = 0; i < nphase; ++i) ms[i] = 0.0;
        for (size_t i = 0; i + 1 < marks.size(); ++i) {
            float t = 0.f;
            cudaEventElapsedTime(&t, marks[i].first, marks[i + 1].first);
            const int ph = marks[i].second;
            if (ph >= 0 && ph < nphase) ms[ph] += t;
        }
        marks.clear();
    }
};
enum { PH_DIAG = 0, PH_TRSM = 1, PH_CAST = 2, PH_SCHUR = 3, PH_TINV = 4, PH_TGEMM = 5, PH_END = 6 };
}  // namespace

extern "C" mxp_status mxp_panel_lu(int n, int b, float *d_A, int64_t lda, mxp_workspace *ws,
                                   void *stream, mxp_lu_stats *stats) {
    if (!ws || !d_A) return fail(MXP_INVALID_ARG, "panel_lu: NULL argument");
    if (n <= 0 || b <= 0 || n % b != 0) return fail(MXP_INVALID_ARG, "panel_lu: n must be a positive multiple of b");
    if (lda < n) return fail(MXP_INVALID_ARG, "panel_lu: lda < n");
    if (n > ws->n || b != ws->b) return fail(MXP_INVALID_ARG, "panel_lu: workspace built for another n/b");
    cudaStream_t st = as_stream(stream);
    const int form = ws->form;
    const int nb = n / b;
    MXP_CUDA(cudaMemsetAsync(ws->status, 0, sizeof(DevStatus), st));
    PhaseTimer pt;
    pt.on = stats != nullptr;
    pt.st = st;
    pt.ws = ws;
    int schur_launches = 0;
    mxp_status s = MXP_OK;
    const int64_t ldk = ws->ldk, kp = ws->kp;
    const size_t es = ws->esize;
    uint8_t *Lb = (uint8_t *)ws->lpanel[0], *Rb = (uint8_t *)ws->rpanel[0];
    uint8_t *Ls = ws->lscale[0], *Rs = ws->rscale[0];
    const int scl = ws->sc_ld;
    const bool fp8 = form == MXP_FORM_FP8;
    // panels per trailing pass; merging needs FP8 scale tiles aligned to the block size
    const int depth = (!fp8 || b % 128 == 0) ? ws->merge : 1;
    const int64_t sct = cdiv(b, 128);  // scale tiles per panel slot (FP8)
    // The inverses of every diagonal block (the last one too) are kept for
    // the refinement's triangular solves when the cooperative kernel makes them.
    ws->inv_lu = nullptr;
    const bool keep_inv = ws->trsv_inv && ws->coop && ws->trsm_tc && nb <= ws->inv_blocks;
    auto inv_u = [&](int64_t kk) -> float * {
        return keep_inv ? ws->inv_store + 2 * (kk / b) * (int64_t)b * b : ws->tinv_u;
    };
    auto inv_l = [&](int64_t kk) -> float * {
        return keep_inv ? ws->inv_store + (2 * (kk / b) + 1) * (int64_t)b * b : ws->tinv_l;
    };
    // C -= L R^T over panel slots slot0 .. slot0+kfac-1 (K = kfac * b), L rows
    // from buffer row lrow, R rows from buffer row rrow.
    auto schur = [&](int64_t mrows, int64_t ncols, int kfac, int64_t lrow, int64_t rrow, float *C,
                     int store, const SchurSched *sched = nullptr, cudaStream_t on = nullptr,
                     int slot0 = 0) -> mxp_status {
        ++schur_launches;
        return launch_schur(form, (int)mrows, (int)ncols, b * kfac, Lb + (lrow * ldk + slot0 * kp) * es, ldk,
                            fp8 ? Ls + (lrow / 128) * scl + slot0 * sct : nullptr,
                            Rb + (rrow * ldk + slot0 * kp) * es, ldk,
                            fp8 ? Rs + (rrow / 128) * scl + slot0 * sct : nullptr, C, lda, ws->status,
                            on ? on : st, store, scl, scl, 0, ws->pair, sched);
    };
    // LU of the diagonal block at kk and, for the tensor-core TRSM, the
    // inverses of both triangles: one cooperative launch on `on`, at most
    // max_grid CTAs (0: all SMs).
    auto factor_diag = [&](int64_t kk, cudaStream_t on, int max_grid) -> mxp_status {
        float *Akk = d_A + kk + kk * lda;
        const int m = n - (int)kk - b;
        const bool coop_inv = ws->coop && ws->trsm_tc && (m > 0 || keep_inv);
        float *tmpU = ws->coop_tmp, *tmpL = ws->coop_tmp + diag_factor_tmp_floats(b);
        float *XU = inv_u(kk), *XL = inv_l(kk);
        if (!ws->coop) return launch_getrf_blocked(b, Akk, lda, ws->status, (int)kk, on);
        // the large doubling levels of the inverses on the tensor cores (same
        // stream; not beside a trailing pass, whose SMs they would share)
        const int tc = coop_inv && max_grid == 0 ? inv_tc_start(ws, b) : 0;
        mxp_status q = launch_diag_factor(b, Akk, lda, coop_inv ? XU : nullptr, coop_inv ? XL : nullptr, b,
                                          tmpU, tmpL, ws->coop_sync, ws->status, (int)kk, on, max_grid, tc);
        if (q == MXP_OK && tc > 0)
            q = finish_inverses_tc(b, Akk, lda, XU, XL, b, tc, ws->trsm_single ? kFormBf16 : MXP_FORM_BF16X2,
                                   tmpU, tmpL, ws, on);
        return q;
    };
    // Factor the diagonal block of step kk (unless diag_done: it was factored
    // on the side stream), solve its two panels, and cast them into panel slot
    // `slot` (0 .. kMaxMerge-1) of the buffers at buffer row `row0`.
    auto factor_panel = [&](int64_t kk, int slot, int64_t row0, bool diag_done) -> mxp_status {
        float *Akk = d_A + kk + kk * lda;
        const int m = n - (int)kk - b;
        const bool coop_inv = ws->coop && ws->trsm_tc && m > 0;
        const bool fuse_f8 = fp8 && ws->trsm_tc && ws->fp8_fused && !ws->trsm_pair && b % 256 == 0 && m > 0;
        mxp_status q = MXP_OK;
        if (!diag_done) {
            pt.mark(PH_DIAG);
            q = factor_diag(kk, st, 0);
        }
        if (q != MXP_OK || m <= 0) return q;
        float *Lcol = Akk + b;
        float *Urow = Akk + (int64_t)b * lda;
        pt.mark(PH_TRSM);
        if (ws->trsm_tc) {
            // X_L = A21 * U11^{-1} and X_U = L11^{-1} * A12 as split-BF16 (hi*hi + hi*lo +
            // lo*hi) tensor-core products against FP32 triangular inverses; the same
            // TRSM-by-inverse idea as the reference's -alt path (panel_trf_gdirect.hpp:73-142)
            // at near-FP32 accuracy instead of FP16.
            const int bf = ws->trsm_single ? kFormBf16 : MXP_FORM_BF16X2;
            if (!coop_inv) {
                pt.mark(PH_TINV);
                q = launch_tri_inv_upper(b, Akk, lda, ws->tinv_u, b, ws->tinv_tmp, st);
                if (q == MXP_OK) q = launch_tri_inv_lower_unit(b, Akk, lda, ws->tinv_l, b, ws->tinv_tmp, st);
            }
            pt.mark(PH_CAST);
            if (q == MXP_OK) q = launch_cast_left(bf, m, b, Lcol, lda, ws->split_big, ws->ldk3, nullptr, st);
            if (q == MXP_OK) q = launch_cast_right(bf, b, b, inv_u(kk), b, ws->split_u, ws->ldk3, nullptr, st);
            pt.mark(PH_TGEMM);
            // FP8 form: the product's epilogue also writes the E4M3 L panel and
            // its scales into the panel slot (the separate casts below are skipped)
            F8Out f8{nullptr, 0, nullptr, 0, 0};
            if (fuse_f8)
                f8 = F8Out{Lb + (row0 * ldk + slot * kp) * es, ldk,
                           Ls + (row0 / 128) * scl + slot * (int64_t)cdiv(b, 128), scl, 0};
            // The triangular K-skip makes the tiles' work uneven (1 to b/256 K blocks):
            // CTAs claim tiles from a counter instead of a static round robin.
            SchurSched tsched;
            tsched.counter = ws->trsm_ctr;
            const SchurSched *ts = ws->trsm_pair || !ws->trsm_counter ? nullptr : &tsched;
            if (q == MXP_OK && ts) {
                cudaError_t e = cudaMemsetAsync(ws->trsm_ctr, 0, sizeof(int), st);
                if (e != cudaSuccess) q = cuda_fail(e, "panel_lu: TRSM tile counter");
            }
            if (q == MXP_OK)
                q = launch_schur(bf, m, b, b, ws->split_big, ws->ldk3, nullptr, ws->split_u, ws->ldk3,
                                 nullptr, Lcol, lda, ws->status, st, /*store=*/1, 0, 0, /*tri=*/1, ws->trsm_pair,
                                 ts, fuse_f8 ? &f8 : nullptr);
            pt.mark(PH_CAST);
            if (q == MXP_OK) q = launch_cast_left(bf, b, b, inv_l(kk), b, ws->split_l, ws->ldk3, nullptr, st);
            if (q == MXP_OK) q = launch_cast_right(bf, m, b, Urow, lda, ws->split_big, ws->ldk3, nullptr, st);
            pt.mark(PH_TGEMM);
            // ... and the one that forms U12 the E4M3 R panel (transposed layout)
            F8Out f8u{nullptr, 0, nullptr, 0, 0};
            if (fuse_f8)
                f8u = F8Out{Rb + (row0 * ldk + slot * kp) * es, ldk,
                            Rs + (row0 / 128) * scl + slot * (int64_t)cdiv(b, 128), scl, 1};
            if (q == MXP_OK && ts) {
                cudaError_t e = cudaMemsetAsync(ws->trsm_ctr, 0, sizeof(int), st);
                if (e != cudaSuccess) q = cuda_fail(e, "panel_lu: TRSM tile counter");
            }
            if (q == MXP_OK)
                q = launch_schur(bf, b, m, b, ws->split_l, ws->ldk3, nullptr, ws->split_big, ws->ldk3,
                                 nullptr, Urow, lda, ws->status, st, /*store=*/1, 0, 0, /*tri=*/2, ws->trsm_pair,
                                 ts, fuse_f8 ? &f8u : nullptr);
        } else {
            q = launch_trsm_runn(m, b, Akk, lda, Lcol, lda, st);
            if (q == MXP_OK) q = launch_trsm_llnu(b, m, Akk, lda, Urow, lda, st);
        }
        if (q != MXP_OK) return q;
        pt.mark(PH_CAST);
        const int64_t koff = slot * kp;
        const int64_t soff = slot * (int64_t)cdiv(b, 128);
        if (!fuse_f8)
            q = launch_cast_left(form, m, b, Lcol, lda, Lb + (row0 * ldk + koff) * es, ldk,
                                 fp8 ? Ls + (row0 / 128) * scl + soff : nullptr, st, scl);
        if (q == MXP_OK && !fuse_f8)
            q = launch_cast_right(form, m, b, Urow, lda, Rb + (row0 * ldk + koff) * es, ldk,
                                  fp8 ? Rs + (row0 / 128) * scl + soff : nullptr, st, scl);
        return q;
    };

    // Overlap of the next group's diagonal factorisation with the trailing pass
    // (single-SM Schur kernel, cooperative diagonal kernel, whole tiles).
    const int ovl_sms = ws->overlap > 0 && !ws->pair && ws->coop && b % 256 == 0
                            ? std::min(ws->overlap, num_sms() / 2) : 0;
    int overlapped = 0;
    bool diag_done = false;
    int k = 0;
    // Groups of `depth` panels (the reference's look-ahead generalised):
    // buffer row 0 is global row (k+1)*b; panel k+j goes to slot j from buffer
    // row j*b.  After panel k+j is factored it updates the column and row
    // blocks of the group's later panels (K = b, its slot alone); one trailing
    // pass with K = D*b then applies the whole group.
    while (k < nb && s == MXP_OK) {
        const int D = std::min(depth, nb - k);
        const int64_t base = (int64_t)(k + 1) * b;  // global row of buffer row 0
        for (int j = 0; j < D && s == MXP_OK; ++j) {
            const int64_t kk = (int64_t)(k + j) * b;
            s = factor_panel(kk, j, (int64_t)j * b, j == 0 && diag_done);
            if (s != MXP_OK) break;
            const int rem = D - 1 - j;                // later panels of the group
            const int64_t r0 = kk + b;                // first row below panel k+j
            if (rem == 0 || r0 >= n) continue;
            pt.mark(PH_SCHUR);
            // column blocks of the later panels: rows r0..n, columns r0..r0+rem*b
            s = schur(n - r0, (int64_t)rem * b, 1, (int64_t)j * b, (int64_t)j * b, d_A + r0 + r0 * lda, 0,
                      nullptr, nullptr, j);
            // their row blocks: rows r0..r0+rem*b, columns right of the group
            const int64_t c0 = r0 + (int64_t)rem * b;
            if (s == MXP_OK && c0 < n)
                s = schur((int64_t)rem * b, n - c0, 1, (int64_t)j * b, (int64_t)j * b + (int64_t)rem * b,
                          d_A + r0 + c0 * lda, 0, nullptr, nullptr, j);
        }
        diag_done = false;
        if (s != MXP_OK) break;
        const int64_t t0 = (int64_t)(k + D) * b;     // trailing matrix: rows / columns t0..n
        const int64_t mt = n - t0;
        k += D;
        if (mt <= 0) break;
        pt.mark(PH_SCHUR);
        const int64_t trow = t0 - base;               // its first buffer row
        float *T = d_A + t0 + t0 * lda;
        if (ovl_sms == 0 || D < 2 || mt <= b || mt < (int64_t)ws->overlap_min * b) {
            s = schur(mt, mt, D, trow, trow, T, 0);
            continue;
        }
        // The next diagonal block first (b x b corner of T), then, at the same
        // time: its factorisation on ovl_sms SMs (side stream) and the rest of
        // T on the other SMs; when the factorisation ends, a second launch on
        // those SMs claims the tiles still left from the shared counter.
        s = schur(b, b, D, trow, trow, T, 0);
        if (s != MXP_OK) break;
        SchurSched main_part, late_part;
        main_part.grid = num_sms() - ovl_sms;
        late_part.grid = ovl_sms;
        main_part.counter = late_part.counter = ws->tile_ctr;
        main_part.skip_rows = late_part.skip_rows = b;
        main_part.skip_cols = late_part.skip_cols = b;
        MXP_CUDA(cudaMemsetAsync(ws->tile_ctr, 0, sizeof(int), st));
        MXP_CUDA(cudaEventRecord(ws->ev_fork, st));
        MXP_CUDA(cudaStreamWaitEvent(ws->side, ws->ev_fork, 0));
        s = factor_diag(t0, ws->side, ovl_sms);
        if (s == MXP_OK) s = schur(mt, mt, D, trow, trow, T, 0, &main_part);
        if (s == MXP_OK) s = schur(mt, mt, D, trow, trow, T, 0, &late_part, ws->side);
        MXP_CUDA(cudaEventRecord(ws->ev_join, ws->side));
        MXP_CUDA(cudaStreamWaitEvent(st, ws->ev_join, 0));
        diag_done = true;
        ++overlapped;
    }
    pt.mark(PH_END);
    if (s != MXP_OK) {
        cudaStreamSynchronize(ws->side);
        pt.collect(nullptr, 0);
        return s;
    }
    DevStatus h;
    mxp_status rs = read_status(ws, st, &h);
    if (rs == MXP_OK && keep_inv) {
        ws->inv_lu = d_A;
        ws->inv_n = n;
        ws->inv_lda = lda;
    }
    if (stats) {
        double ms[6];
        pt.collect(ms, 6);
        stats->ms_diag_lu = ms[PH_DIAG];
        stats->ms_trsm = ms[PH_TRSM] + ms[PH_TINV] + ms[PH_TGEMM];
        stats->ms_trsm_inv = ms[PH_TINV];
        stats->ms_trsm_gemm = ms[PH_TGEMM];
        stats->ms_cast = ms[PH_CAST];
        stats->ms_schur = ms[PH_SCHUR];
        stats->ms_total = ms[0] + ms[1] + ms[2] + ms[3] + ms[4] + ms[5];
        stats->info = h.code == MXP_ZERO_PIVOT ? h.info0 : 0;
        stats->schur_launches = schur_launches;
        stats->overlapped_diag = overlapped;
        stats->pad = 0;
    }
    return rs;
}

// ---------------------------------------------------------------------------
// refinement
// ---------------------------------------------------------------------------
// y = b y + a A x for the matrix the workspace refines against: regenerated
// from the LCG of `seed`, or Higham's matrix when the workspace was set to it.
static mxp_status residual_gemv(mxp_workspace *ws, int n, uint64_t seed, const double *dd, double a,
                                const double *x, double b, double *y, cudaStream_t st) {
    if (ws->higham) return launch_higham_gemv(n, ws->h_alpha, ws->h_beta, a, x, b, y, st);
    return launch_otf_gemv(n, seed, dd, a, x, b, y, ws->partials, ws->max_splits, st);
}

// x <- U^{-1} L^{-1} x with the factor LU: by the stored inverses of the
// diagonal blocks when they belong to this factor (the last mxp_panel_lu on
// the workspace), else by the chain of 64-row blocks.
static mxp_status lu_solve_ws(mxp_workspace *ws, int n, const float *LU, int64_t lda, double *x,
                              cudaStream_t st, int withhold = -1) {
    if (withhold < 0 && ws->trsv_inv && ws->inv_lu && LU == ws->inv_lu && n == ws->inv_n &&
        lda == ws->inv_lda && lu_solve_inv_supported(n, ws->b, LU, lda)) {
        const int64_t bb = (int64_t)ws->b * ws->b;
        return launch_lu_solve_inv(n, ws->b, LU, lda, ws->inv_store, ws->inv_store + bb, 2 * bb, x, ws->trsv_t, st,
                                   ws->side, ws->ev_trsv);
    }
    return launch_lu_solve(n, LU, lda, x, ws->flags, ws->status, st, withhold);
}

extern "C" mxp_status mxp_otf_gemv(int n, uint64_t seed, const double *d_d, double alpha,
                                   const double *d_x, double beta, double *d_y, mxp_workspace *ws,
                                   void *stream) {
    if (!ws) return fail(MXP_INVALID_ARG, "otf_gemv: workspace is NULL");
    if (n > ws->n) return fail(MXP_INVALID_ARG, "otf_gemv: n larger than the workspace");
    return launch_otf_gemv(n, seed, d_d, alpha, d_x, beta, d_y, ws->partials, ws->max_splits,
                           as_stream(stream));
}

extern "C" mxp_status mxp_lu_solve(int n, const float *d_LU, int64_t lda, double *d_x,
                                   mxp_workspace *ws, void *stream) {
    if (!ws) return fail(MXP_INVALID_ARG, "lu_solve: workspace is NULL");
    if (n > ws->n) return fail(MXP_INVALID_ARG, "lu_solve: n larger than the workspace");
    cudaStream_t st = as_stream(stream);
    const int withhold = ws->withhold;
    ws->withhold = -1;  // one call only
    mxp_status s = lu_solve_ws(ws, n, d_LU, lda, d_x, st, withhold);
    if (s != MXP_OK) return s;
    return read_status(ws, st);  // bounded-wait timeouts surface here
}

extern "C" mxp_status mxp_infnorm(int n, const double *d_x, double *h_out, mxp_workspace *ws,
                                  void *stream) {
    if (!ws || !h_out) return fail(MXP_INVALID_ARG, "infnorm: NULL argument");
    cudaStream_t st = as_stream(stream);
    mxp_status s = launch_infnorm(n, d_x, ws->scal, st);
    if (s != MXP_OK) return s;
    MXP_CUDA(cudaMemcpyAsync(h_out, ws->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    MXP_CUDA(cudaStreamSynchronize(st));
    return MXP_OK;
}

static double elapsed(cudaEvent_t a, cudaEvent_t b) {
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    return t;
}

// Correction d = (approx) A^{-1} r by GMRES on M^{-1} A d = M^{-1} r, M = LU,
// zero initial guess, at most ws->gm_m Arnoldi steps, stop when the
// preconditioned residual estimate |g_{k}| <= gm_tol * beta.  r is
// overwritten by d.  Host reads one scalar per Arnoldi step.
static mxp_status gmres_correction(int n, uint64_t seed, const float *LU, int64_t lda, const double *dd,
                                   double *r, mxp_workspace *ws, cudaStream_t st, int *inner_iters,
                                   double *ms_gemv, double *ms_trsv) {
    const int m = ws->gm_m;
    const int ldh = 31;
    double *V = ws->gV, *H = ws->gH;
    double *cs = ws->gsmall, *sn = cs + 31, *g = sn + 31, *y = g + 32, *hcol = y + 31, *hcol2 = hcol + 31;
    double *sc = hcol2 + 31;  // [0] dot scratch [1] beta [2] hnext [3] resid
    double *w = ws->w;
    double *h = ws->h_scal + 8;
    mxp_status s;
    // Timed regions bracket pool events; their times are read at the stream
    // synchronisations the Arnoldi loop makes anyway (no wait of their own).
    std::vector<std::pair<size_t, double *>> pending;
    size_t next_ev = 0;
    auto timed = [&](double *acc, auto &&fn) -> mxp_status {
        cudaEvent_t a = pool_event(ws, next_ev), b = pool_event(ws, next_ev + 1);
        if (a && b) cudaEventRecord(a, st);
        mxp_status q = fn();
        if (a && b) {
            cudaEventRecord(b, st);
            pending.push_back({next_ev, acc});
            next_ev += 2;
        }
        return q;
    };
    auto settle = [&]() {  // after a synchronisation of st
        for (auto &pr : pending) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ws->ev_pool[pr.first], ws->ev_pool[pr.first + 1]);
            *pr.second += t;
        }
        pending.clear();
        next_ev = 0;
    };
    // z = M^{-1} r -> V_0 after normalisation
    s = launch_copy(n, r, V, st);
    if (s == MXP_OK) s = timed(ms_trsv, [&] { return lu_solve_ws(ws, n, LU, lda, V, st); });
    if (s == MXP_OK) s = launch_mdot(n, 1, V, n, V, ws->gpart, sc + 0, 0, st);
    if (s == MXP_OK) s = launch_sqrt(sc + 0, sc + 1, st);
    if (s == MXP_OK) s = launch_vdiv(n, V, sc + 1, V, st);
    if (s == MXP_OK) s = launch_set_g0(m, g, sc + 1, st);
    if (s != MXP_OK) goto out;
    {
        MXP_CUDA(cudaMemcpyAsync(h, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        MXP_CUDA(cudaStreamSynchronize(st));
        settle();
        const double beta = h[0];
        int k = 0;
        if (!(beta > 0.0) || !std::isfinite(beta)) {
            MXP_CUDA(cudaMemsetAsync(r, 0, (size_t)n * sizeof(double), st));
            goto out;
        }
        for (int j = 0; j < m; ++j) {
            double *vj = V + (int64_t)j * n;
            s = timed(ms_gemv, [&] { return residual_gemv(ws, n, seed, dd, 1.0, vj, 0.0, w, st); });
            if (s == MXP_OK) s = timed(ms_trsv, [&] { return lu_solve_ws(ws, n, LU, lda, w, st); });
            // classical Gram-Schmidt, twice
            if (s == MXP_OK) s = launch_mdot(n, j + 1, V, n, w, ws->gpart, hcol, 0, st);
            if (s == MXP_OK) s = launch_vsub(n, j + 1, V, n, hcol, w, st);
            if (s == MXP_OK) s = launch_mdot(n, j + 1, V, n, w, ws->gpart, hcol2, 0, st);
            if (s == MXP_OK) s = launch_vsub(n, j + 1, V, n, hcol2, w, st);
            if (s == MXP_OK) s = launch_axpy(j + 1, 1.0, hcol2, hcol, st);
            if (s == MXP_OK) s = launch_mdot(n, 1, w, n, w, ws->gpart, sc + 0, 0, st);
            if (s == MXP_OK) s = launch_sqrt(sc + 0, sc + 2, st);
            if (s == MXP_OK) s = launch_givens(j, H, ldh, hcol, sc + 2, cs, sn, g, sc + 3, st);
            if (s == MXP_OK) s = launch_vdiv(n, w, sc + 2, V + (int64_t)(j + 1) * n, st);
            if (s != MXP_OK) goto out;
            MXP_CUDA(cudaMemcpyAsync(h + 1, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, st));
            MXP_CUDA(cudaStreamSynchronize(st));
            settle();
            k = j + 1;
            if (!(h[1] > ws->gm_tol * beta)) break;
        }
        *inner_iters += k;
        s = launch_backsolve(k, H, ldh, g, y, st);
        if (s == MXP_OK) {
            cudaError_t e = cudaMemsetAsync(r, 0, (size_t)n * sizeof(double), st);
            if (e != cudaSuccess) s = cuda_fail(e, "gmres: memset");
        }
        if (s == MXP_OK) s = launch_vadd(n, k, V, n, y, r, st);
    }
out:
    return s;
}

extern "C" mxp_status mxp_iterative_refinement(int n, uint64_t seed, const float *d_LU, int64_t lda,
                                               const double *d_d, const double *d_rowsum,
                                               const double *d_rhs, double *d_x, double norma,
                                               int maxit, int method, mxp_workspace *ws,
                                               void *stream, mxp_ir_stats *stats) {
    if (!ws || !d_LU || !d_d || !d_rhs || !d_x) return fail(MXP_INVALID_ARG, "IR: NULL argument");
    if (n > ws->n || lda < n) return fail(MXP_INVALID_ARG, "IR: bad n / lda");
    if (maxit < 1) return fail(MXP_INVALID_ARG, "IR: maxit < 1");
    if (method != MXP_IR_CLASSIC && method != MXP_IR_GMRES) return fail(MXP_INVALID_ARG, "IR: unknown method");
    cudaStream_t st = as_stream(stream);
    double *r = ws->r;
    double *sc = ws->scal;  // [0] normx [1] normr [2] norma [3] normb
    double *h = ws->h_scal;
    cudaEvent_t e0 = ws->ev_ir[0], e1 = ws->ev_ir[1], g0 = ws->ev_ir[2], g1 = ws->ev_ir[3], t0 = ws->ev_ir[4],
                t1 = ws->ev_ir[5];
    double ms_gemv = 0.0, ms_trsv = 0.0;
    bool trsv_pending = false;  // t0..t1 recorded, read at the next synchronisation
    mxp_status s = MXP_OK;
    cudaEventRecord(e0, st);
    MXP_CUDA(cudaMemsetAsync(ws->status, 0, sizeof(DevStatus), st));
    if (norma <= 0.0 && ws->higham) norma = higham_infnorm(n, ws->h_alpha, ws->h_beta);
    if (norma <= 0.0) {
        s = launch_norma(n, d_d, d_rowsum, sc + 2, st);
        if (s != MXP_OK) return s;
    }
    s = launch_infnorm(n, d_rhs, sc + 3, st);
    if (s != MXP_OK) return s;
    MXP_CUDA(cudaMemcpyAsync(h + 2, sc + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MXP_CUDA(cudaStreamSynchronize(st));
    if (norma <= 0.0) norma = h[2];
    const double normb = h[3];
    s = launch_ir_init(n, d_rhs, d_d, d_x, st);
    if (s != MXP_OK) return s;
    const double eps = 0x1p-53;  // DBL_EPSILON / 2
    int it = 0;
    bool converged = false;
    double normr = -1.0, hpl = -1.0, normx = 0.0;
    int gemv_calls = 0, trsv_calls = 0, inner = 0;
    for (it = 0; it < maxit; ++it) {
        s = launch_copy(n, d_rhs, r, st);
        if (s == MXP_OK) s = launch_infnorm(n, d_x, sc + 0, st);
        cudaEventRecord(g0, st);
        if (s == MXP_OK) s = residual_gemv(ws, n, seed, d_d, -1.0, d_x, 1.0, r, st);
        cudaEventRecord(g1, st);
        if (s == MXP_OK) s = launch_infnorm(n, r, sc + 1, st);
        if (s != MXP_OK) return s;
        ++gemv_calls;
        MXP_CUDA(cudaMemcpyAsync(h, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        MXP_CUDA(cudaStreamSynchronize(st));
        ms_gemv += elapsed(g0, g1);
        if (trsv_pending) ms_trsv += elapsed(t0, t1);
        trsv_pending = false;
        normx = h[0];
        normr = h[1];
        hpl = normr / (norma * normx + normb) * 1.0 / ((double)n * eps);
        if (stats && it < 64) {
            stats->history[it] = hpl;
            stats->history_residual[it] = normr;
        }
        if (!std::isfinite(hpl)) {
            s = fail(MXP_NONFINITE, "IR: non-finite residual");
            break;
        }
        if (hpl < 16.0) {
            converged = true;
            break;
        }
        if (method == MXP_IR_GMRES) {
            double mg = 0.0, mt = 0.0;
            const int before = inner;
            s = gmres_correction(n, seed, d_LU, lda, d_d, r, ws, st, &inner, &mg, &mt);
            ms_gemv += mg;
            ms_trsv += mt;
            gemv_calls += inner - before;
            trsv_calls += inner - before + 1;
            if (s == MXP_OK) s = launch_axpy(n, 1.0, r, d_x, st);
            if (s != MXP_OK) return s;
        } else {
            cudaEventRecord(t0, st);
            s = lu_solve_ws(ws, n, d_LU, lda, r, st);
            cudaEventRecord(t1, st);
            if (s == MXP_OK) s = launch_axpy(n, 1.0, r, d_x, st);
            if (s != MXP_OK) return s;
            ++trsv_calls;
            trsv_pending = true;
        }
    }
    cudaEventRecord(e1, st);
    mxp_status rs = read_status(ws, st);
    if (trsv_pending) ms_trsv += elapsed(t0, t1);
    if (stats) {
        stats->iterations = it;
        stats->converged = converged ? 1 : 0;
        stats->residual = normr;
        stats->hpl_harness = hpl;
        stats->norma = norma;
        stats->normb = normb;
        stats->normx = normx;
        stats->ms_total = elapsed(e0, e1);
        stats->ms_gemv = ms_gemv;
        stats->ms_trsv = ms_trsv;
        stats->gemv_calls = gemv_calls;
        stats->trsv_calls = trsv_calls;
        stats->inner_iterations = inner;
    }
    if (s != MXP_OK) return s;
    if (rs != MXP_OK) return rs;
    if (!converged) return fail(MXP_NOT_CONVERGED, "IR: maxit reached without convergence");
    return MXP_OK;
}

extern "C" mxp_status mxp_solve(int n, int b, uint64_t seed, float *d_A, int64_t lda,
                                const double *d_d, const double *d_rowsum, const double *d_rhs,
                                double *d_x, int maxit, int method, mxp_workspace *ws,
                                void *stream, mxp_lu_stats *lu_stats, mxp_ir_stats *ir_stats) {
    mxp_status s = mxp_panel_lu(n, b, d_A, lda, ws, stream, lu_stats);
    if (s != MXP_OK) return s;
    return mxp_iterative_refinement(n, seed, d_A, lda, d_d, d_rowsum, d_rhs, d_x, 0.0, maxit, method,
                                    ws, stream, ir_stats);
}

extern "C" mxp_status mxp_solve_host(int n, int b, uint64_t seed, float *d_A, int64_t lda,
                                     const double *d_d, const double *d_rowsum,
                                     const double *h_rhs, double *h_x, int maxit, int method,
                                     mxp_workspace *ws, void *stream, mxp_lu_stats *lu_stats,
                                     mxp_ir_stats *ir_stats) {
    if (!ws || !h_rhs || !h_x) return fail(MXP_INVALID_ARG, "solve_host: NULL argument");
    if (n > ws->n) return fail(MXP_INVALID_ARG, "solve_host: n larger than the workspace");
    cudaStream_t st = as_stream(stream);
    // rhs and x are staged in the workspace's own vector slots: no allocation
    MXP_CUDA(cudaMemcpyAsync(ws->rhsv, h_rhs, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
    mxp_status s = mxp_solve(n, b, seed, d_A, lda, d_d, d_rowsum, ws->rhsv, ws->xv, maxit, method, ws,
                             stream, lu_stats, ir_stats);
    if (s == MXP_OK || s == MXP_NOT_CONVERGED) {
        cudaError_t e = cudaMemcpyAsync(h_x, ws->xv, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "solve_host: copy of x");
    }
    return s;
}
