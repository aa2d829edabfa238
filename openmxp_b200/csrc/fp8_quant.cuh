// E4M3 quantization with one power-of-two scale per 128 x 128 tile, shared by
// the panel-cast kernels (casts.cu) and the epilogue of the tensor-core TRSM
// product that writes the FP8 L panel directly (schur_tc.cu): both must give
// the same bytes for the same FP32 values.
#pragma once

#include <cuda_fp8.h>
#include <stdint.h>

namespace mxp {

// Largest e with amax * 2^e <= 448, clamped to [-126, 126]; 0 for a zero or
// non-finite amax.  Mirrors orc_e4m3_scale_exp of the oracle bit for bit.
__device__ __forceinline__ int e4m3_scale_exp(float amax) {
    if (!(amax > 0.0f) || !(amax < 3.0e38f)) return 0;
    int ea = (int)((__float_as_uint(amax) >> 23) & 0xffu) - 127;
    if (ea < -126) ea = -126;
    int e = 8 - ea;
    if ((double)amax * exp2((double)e) > 448.0) e -= 1;
    e = max(-126, min(126, e));
    return e;
}

// 2^e as a float (e in [-126, 126])
__device__ __forceinline__ float e4m3_scale_up(int e) { return __int_as_float((e + 127) << 23); }

__device__ __forceinline__ uint8_t to_e4m3(float x) {
    return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}

}  // namespace mxp
