// Test infrastructure only.  Compiles the reference's own CPU pieces of the
// solve path in place, from the reference tree (-I <reference>/src), and
// exposes them with C linkage so the oracle can be pinned against them.
// Nothing here is shipped or measured; the output lands in oracle/_ref/.
//
// Pieces: the LCG generator (hpl_rand.hpp), the CPU on-the-fly GEMV kernel
// (otf_gemv.cpp through svesim.hpp / fp16sim.hpp on x86), and the CPU no-pivot
// LU (sgetrf_nopiv.cpp, naive and the 6-wide OpenMP variant).
#define __HPLAI_DEVICE_MACROS__ 1
#define __host__
#define __device__
#include <cstddef>
#include <cstdint>
int grank = 0;  // declared extern by hpl_rand.hpp:10
#include "hpl_rand.hpp"
#include "otf_gemv.cpp"
#include "sgetrf_nopiv.cpp"

extern "C" {
// fill_one_panel_with_rand (hpl_rand.hpp:158-198): FP32 block with the CPU
// calc_diag-order diagonal when the block is square and on the diagonal.
void ref_fill_one_panel_f32(int n, int i0, int j0, int nrow, int ncol, float *a, size_t lda,
                            uint64_t seed, int calc_diag) {
    fill_one_panel_with_rand<float>(n, i0, j0, nrow, ncol, a, lda, seed, calc_diag != 0);
}
// panel_fill_one_with_rand (hpl_rand.hpp:80-129) in FP64: used for the RHS,
// i.e. column j0 = n of the stream (matgen.hpp:419-436).
void ref_panel_fill_f64(int n, int i0, int j0, int nrow, int ncol, double *a, size_t lda,
                        uint64_t seed) {
    panel_fill_one_with_rand<double>(n, i0, j0, nrow, ncol, a, lda, seed, false);
}
double ref_calc_diag(int i, int n, uint64_t seed) { return calc_diag(i, n, seed); }
double ref_mat_elem(int n, int i, int j, int seed) { return mat_elem(n, i, j, seed); }
void ref_rand_pow(uint64_t a, uint64_t c, uint64_t e, uint64_t *oa, uint64_t *oc) {
    RandCoeff r = RandCoeff{a, c}.pow(e);
    *oa = r.a;
    *oc = r.c;
}
void ref_sgetrf_nopiv_naive(int m, int n, float *a, size_t lda) { sgetrf_nopiv_naive(m, n, a, lda); }
void ref_sgetrf_nopiv_tuned(int n, float *a, size_t lda) { sgetrf_nopiv_tuned(n, a, lda); }
unsigned short ref_fp16_bits(float f) {
    fp16 h(f);
    return h.x;
}
}
