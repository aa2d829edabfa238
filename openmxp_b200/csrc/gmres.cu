// FP64 kernels of GMRES-IR: refinement whose correction equation A d = r is
// solved by GMRES left-preconditioned with the low-precision LU factors
// (M = LU in FP32), with A applied on the fly (otf_gemv) and every vector
// operation, the Arnoldi orthogonalisation (classical Gram-Schmidt, applied
// twice) and the Givens rotations in FP64 on the GPU.  The reference has only
// classic refinement (iterative_refinement.hpp:97-174); this is the GMRES
// alternative its header comment of iterative refinement leaves open.
//
// Basis vectors are rows of V (ldv = n doubles apart).  Reductions are
// two-stage with a fixed order, so results are deterministic.
#include "mxp_internal.cuh"

namespace mxp {

namespace {

constexpr int kDotThreads = 256;

// partial[k * nblk + blockIdx.x] = sum over this block's rows of V[k][i] * w[i], k < nv
__global__ void __launch_bounds__(kDotThreads)
mdot_kernel(int n, int nv, const double *__restrict__ V, int64_t ldv, const double *__restrict__ w,
            double *__restrict__ partial, int nblk) {
    __shared__ double red[kDotThreads / 32];
    const int k = blockIdx.y;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kDotThreads + threadIdx.x; i < n;
         i += (int64_t)nblk * kDotThreads)
        s = __fma_rn(V[(int64_t)k * ldv + i], w[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kDotThreads / 32; ++q) t += red[q];
        partial[(int64_t)k * nblk + blockIdx.x] = t;
    }
}

// out[k] (+)= sum_b partial[k * nblk + b], one warp per k, fixed order.
__global__ void mdot_reduce_kernel(int nv, int nblk, const double *__restrict__ partial,
                                   double *__restrict__ out, int accumulate) {
    const int k = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += 32) s += partial[(int64_t)k * nblk + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[k] = accumulate ? out[k] + s : s;
}

// w[i] -= sum_{k < nv} V[k][i] * h[k]
__global__ void vsub_kernel(int n, int nv, const double *__restrict__ V, int64_t ldv,
                            const double *__restrict__ h, double *__restrict__ w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = w[i];
    for (int k = 0; k < nv; ++k) t = __fma_rn(-V[(int64_t)k * ldv + i], h[k], t);
    w[i] = t;
}

// y[i] += sum_{k < nv} V[k][i] * c[k]
__global__ void vadd_kernel(int n, int nv, const double *__restrict__ V, int64_t ldv,
                            const double *__restrict__ c, double *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = y[i];
    for (int k = 0; k < nv; ++k) t = __fma_rn(V[(int64_t)k * ldv + i], c[k], t);
    y[i] = t;
}

// dst = src / *den   (den on the device: no host round trip)
__global__ void vdiv_kernel(int n, const double *__restrict__ src, const double *__restrict__ den,
                            double *__restrict__ dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i] / *den;
}

// One-thread Arnoldi bookkeeping for column j (0-based):
//   hcol[0..j] holds the projections (already accumulated over both CGS
//   passes), *hnext = ||w||.  Apply the previous rotations, build rotation j,
//   update g, store the column in H (column-major, ldh), report |g[j+1]|.
__global__ void givens_kernel(int j, double *__restrict__ H, int ldh, const double *__restrict__ hcol,
                              const double *__restrict__ hnext, double *__restrict__ cs,
                              double *__restrict__ sn, double *__restrict__ g,
                              double *__restrict__ resid_out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double *col = H + (int64_t)j * ldh;
    for (int i = 0; i <= j; ++i) col[i] = hcol[i];
    double hj1 = *hnext;
    for (int i = 0; i < j; ++i) {
        const double a = col[i], b = col[i + 1];
        col[i] = cs[i] * a + sn[i] * b;
        col[i + 1] = -sn[i] * a + cs[i] * b;
    }
    const double a = col[j], b = hj1;
    const double r = hypot(a, b);
    const double c = r > 0.0 ? a / r : 1.0;
    const double s = r > 0.0 ? b / r : 0.0;
    cs[j] = c;
    sn[j] = s;
    col[j] = r;
    col[j + 1] = 0.0;
    const double gj = g[j];
    g[j] = c * gj;
    g[j + 1] = -s * gj;
    *resid_out = fabs(g[j + 1]);
}

// Solve the k x k upper-triangular H y = g (one thread).
__global__ void backsolve_kernel(int k, const double *__restrict__ H, int ldh,
                                 const double *__restrict__ g, double *__restrict__ y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = k - 1; i >= 0; --i) {
        double t = g[i];
        for (int q = i + 1; q < k; ++q) t -= H[(int64_t)q * ldh + i] * y[q];
        y[i] = t / H[(int64_t)i * ldh + i];
    }
}

__global__ void set_g0_kernel(int m, double *__restrict__ g, const double *__restrict__ beta) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i <= m) g[i] = (i == 0) ? *beta : 0.0;
}

__global__ void sqrt_kernel(const double *__restrict__ in, double *__restrict__ out) {
    if (threadIdx.x == 0) *out = sqrt(*in);
}

}  // namespace

int gmres_dot_blocks(int n) { return (int)imin64(cdiv(n, kDotThreads), 2 * num_sms()); }

// out[0..nv) (+)= V[0..nv) . w
mxp_status launch_mdot(int n, int nv, const double *V, int64_t ldv, const double *w,
                       double *partial, double *out, int accumulate, cudaStream_t st) {
    const int nblk = gmres_dot_blocks(n);
    mdot_kernel<<<dim3(nblk, nv), kDotThreads, 0, st>>>(n, nv, V, ldv, w, partial, nblk);
    MXP_LAUNCHED();
    mdot_reduce_kernel<<<nv, 32, 0, st>>>(nv, nblk, partial, out, accumulate);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_vsub(int n, int nv, const double *V, int64_t ldv, const double *h, double *w,
                       cudaStream_t st) {
    vsub_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, nv, V, ldv, h, w);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_vadd(int n, int nv, const double *V, int64_t ldv, const double *c, double *y,
                       cudaStream_t st) {
    vadd_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, nv, V, ldv, c, y);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_vdiv(int n, const double *src, const double *den, double *dst, cudaStream_t st) {
    vdiv_kernel<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(n, src, den, dst);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_givens(int j, double *H, int ldh, const double *hcol, const double *hnext,
                         double *cs, double *sn, double *g, double *resid_out, cudaStream_t st) {
    givens_kernel<<<1, 32, 0, st>>>(j, H, ldh, hcol, hnext, cs, sn, g, resid_out);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_backsolve(int k, const double *H, int ldh, const double *g, double *y,
                            cudaStream_t st) {
    backsolve_kernel<<<1, 32, 0, st>>>(k, H, ldh, g, y);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_set_g0(int m, double *g, const double *beta, cudaStream_t st) {
    set_g0_kernel<<<(unsigned)cdiv(m + 1, 128), 128, 0, st>>>(m, g, beta);
    MXP_LAUNCHED();
    return MXP_OK;
}

mxp_status launch_sqrt(const double *in, double *out, cudaStream_t st) {
    sqrt_kernel<<<1, 32, 0, st>>>(in, out);
    MXP_LAUNCHED();
    return MXP_OK;
}

}  // namespace mxp
