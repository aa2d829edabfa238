// mxp_otf_gemv_noalloc: the on-the-fly residual GEMV for callers that cannot
// allocate device memory.
//
// Some callers hold only raw device pointers and cannot create or own an
// mxp_workspace: code dropped into an existing refinement loop that has no
// place to keep one, or applications that forbid device allocation after
// start-up because cudaMalloc / cudaFree may synchronise the whole device and
// stall unrelated streams.  This entry point takes inputs and outputs only;
// the split-K partial sums that mxp_otf_gemv keeps in the workspace live here
// in a file-scope device array of fixed size instead, so the call allocates
// nothing.
//
// Rules of use:
//  * Maximum size: n <= kNoAllocMaxN (262144).  Larger n is rejected with
//    MXP_INVALID_ARG before anything is launched.
//  * The array (kScratchDoubles doubles, 4 MiB) is reserved on every GPU that
//    loads the library and stays reserved until the process exits.
//  * Its device address is looked up (cudaGetSymbolAddress) on the first call
//    made on each device, with that device current; make that first call
//    before any stream capture begins.
//  * The stream must belong to the current device (the array used is the
//    current device's copy); a stream of another device is rejected with
//    MXP_INVALID_ARG.
//  * Every call shares the one array and it keeps the last call's contents.
//    Each call overwrites every partial sum it later reads, so nothing needs
//    clearing between calls; calls that overlap on the GPU (different streams,
//    or different host threads on the same device) race on the array and must
//    be ordered by the caller.
#include <mutex>

#include "mxp_internal.cuh"

namespace mxp {
namespace {

constexpr int64_t kScratchDoubles = int64_t(1) << 19;    // 4 MiB of partial sums
constexpr int64_t kNoAllocMaxN = kScratchDoubles / 2;     // room for at least two column splits
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_gemv_scratch[kScratchDoubles];

std::mutex g_addr_mutex;
double *g_addr[kMaxDevices] = {};

// Device address of g_gemv_scratch on the current device (resolved once per device).
mxp_status scratch_address(double **out) {
    int dev = 0;
    MXP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(MXP_UNSUPPORTED, "otf_gemv_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_gemv_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "otf_gemv_noalloc: cudaGetSymbolAddress");
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return MXP_OK;
}

}  // namespace
}  // namespace mxp

using namespace mxp;

extern "C" mxp_status mxp_otf_gemv_noalloc(int n, uint64_t seed, const double *d_d, double alpha,
                                           const double *d_x, double beta, double *d_y,
                                           void *stream) {
    if (n <= 0 || !d_d || !d_x || !d_y) return fail(MXP_INVALID_ARG, "otf_gemv_noalloc: bad arguments");
    if ((int64_t)n > kNoAllocMaxN)
        return fail(MXP_INVALID_ARG, "otf_gemv_noalloc: n exceeds the fixed scratch (maximum n = 262144); "
                                     "use mxp_otf_gemv with a workspace");
    cudaStream_t st = as_stream(stream);
    if (st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread) {  // those name the current device
        int cur = 0, sdev = 0;
        MXP_CUDA(cudaGetDevice(&cur));
        MXP_CUDA(cudaStreamGetDevice(st, &sdev));
        if (sdev != cur)
            return fail(MXP_INVALID_ARG, "otf_gemv_noalloc: the stream belongs to another device than the current one");
    }
    double *scratch = nullptr;
    mxp_status s = scratch_address(&scratch);
    if (s != MXP_OK) return s;
    const int max_splits = (int)imin64(16, kScratchDoubles / n);
    return launch_otf_gemv(n, seed, d_d, alpha, d_x, beta, d_y, scratch, max_splits, st);
}
