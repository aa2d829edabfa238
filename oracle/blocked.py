"""Numpy restatement of the blocked no-pivot LU as the product runs it at its
full block size: FP32 diagonal-block LU, panel TRSM by inverse (FP32
triangular inverses by doubling, the large doubling levels and the panel
products as low-precision products with FP32 accumulation), panel casts and
the Schur update C -= quant(L) quant(U^T)^T.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of mxp_panel_lu
and mxp_getrf_nopiv_inv at block sizes where the C restatement
(oracle/mxp_oracle.c) is too slow.  The product path never calls it.

What each step restates:
- diagonal block: orc_getrf_nopiv_blocked (C, 64-column steps, the
  sgetrf_nopiv_naive operation order of sgetrf_nopiv.cpp:27-61 inside);
- TRSM by inverse: update_left_panels_wGPU_alt / update_right_panels_wGPU_alt
  (panel_trf_gdirect.hpp:73-142): an FP32 inverse of the diagonal triangle,
  then one GEMM of the panel against it.  The reference casts both operands
  to FP16; the product uses BF16, as one product ("single", 2^-9 operand
  rounding) or as three split products hi*hi + hi*lo + lo*hi accumulated in
  one FP32 sum ("split", near FP32).  "fp32" keeps the reference's plain
  STRSM (panel_trf.hpp:188-246);
- triangular inverses: orc_tri_inverses (C) for the 64 x 64 blocks and the
  FP32 doubling levels below `inv_tc`; the levels from `inv_tc` up as
  low-precision products in the TRSM's form, as the product runs them on
  its tensor cores;
- casts and Schur update: the quantisers below (bit-exact restatements of
  the casts, pinned against the C oracle's scalar conversions by
  tests/test_oracle_blocked.py) and FP32 matrix products of the dequantised
  operands: FP16, BF16 and scaled E4M3 products are exact in FP32, so only
  the order of the FP32 sums differs from the tensor cores'
  (panel_trf.hpp:825-837, rocm_device_macros.h:267-268).
The schedule is the reference's one panel per step; the product's merged
groups give every element the same updates in the same order of panels.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

FORM_FP16, FORM_BF16X2, FORM_FP8, FORM_FP32 = 0, 1, 2, 3
FORM_BF16 = 4  # one BF16 product (the single-product TRSM by inverse)
TRSM_FORMS = {"split": FORM_BF16X2, "single": FORM_BF16}


# ---------------------------------------------------------------------------
# quantisers: dequantised FP32 values (and the E4M3 bytes / UE8M0 scales)
# ---------------------------------------------------------------------------
def f16_round(x: np.ndarray) -> np.ndarray:
    """FP32 -> FP16 round to nearest even (subnormals kept, overflow to inf) -> FP32."""
    with np.errstate(over="ignore"):
        return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 round to nearest even -> FP32 (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = (u + np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32).reshape(np.shape(x))


def e4m3_round(v: np.ndarray) -> np.ndarray:
    """FP32 -> E4M3 (bias 7, max 448, round to nearest even, saturating) -> FP32."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    a = np.abs(v)
    u = a.view(np.uint32)
    normal = ((u + np.uint32(0x7FFFF) + ((u >> np.uint32(20)) & np.uint32(1))) & np.uint32(0xFFF00000)).view(
        np.float32)
    normal = np.minimum(normal, np.float32(448.0))
    sub = (np.rint(a * np.float32(512.0)) / np.float32(512.0)).astype(np.float32)
    out = np.where(a >= np.float32(2.0 ** -6), normal, sub).astype(np.float32)
    return np.copysign(out, v).astype(np.float32)


_E4M3_POS = None


def e4m3_bytes(v: np.ndarray) -> np.ndarray:
    """The E4M3 byte of each FP32 value (sign of the input kept for zeros)."""
    global _E4M3_POS
    if _E4M3_POS is None:
        vals = np.array([O.lib().orc_e4m32f(c) for c in range(0x7F)], np.float32)  # 0x00..0x7e
        _E4M3_POS = vals
    q = np.abs(e4m3_round(v))
    code = np.searchsorted(_E4M3_POS, q).astype(np.uint8)
    return code | (np.signbit(np.asarray(v, np.float32)).astype(np.uint8) << np.uint8(7))


def e4m3_scale_exp(amax: np.ndarray) -> np.ndarray:
    """Largest e with amax * 2^e <= 448 per tile (0 for amax == 0); clamp +-126."""
    amax = np.asarray(amax, np.float32)
    ea = ((amax.view(np.uint32) >> np.uint32(23)) & np.uint32(0xFF)).astype(np.int64) - 127
    ea = np.maximum(ea, -126)
    e = 8 - ea
    e = np.where(np.ldexp(amax, e.astype(np.int32)) > np.float32(448.0), e - 1, e)
    e = np.clip(e, -126, 126)
    return np.where(amax > 0, e, 0).astype(np.int64)


def fp8_panel(P: np.ndarray):
    """E4M3 copy of a panel in (row, K) orientation with one power-of-two scale
    per 128 x 128 tile: (dequantised FP32 values, bytes, UE8M0 scale bytes
    127 - e of shape (ceil(m/128), ceil(K/128)))."""
    P = np.asarray(P, np.float32)
    m, K = P.shape
    mt, kt = -(-m // 128), -(-K // 128)
    pad = np.zeros((mt * 128, kt * 128), np.float32)
    pad[:m, :K] = np.abs(P)
    amax = pad.reshape(mt, 128, kt, 128).max(axis=(1, 3))
    e = e4m3_scale_exp(amax)
    efull = np.repeat(np.repeat(e, 128, axis=0), 128, axis=1)[:m, :K].astype(np.int32)
    scaled = np.ldexp(P, efull).astype(np.float32)
    deq = np.ldexp(e4m3_round(scaled), -efull).astype(np.float32)
    return deq, e4m3_bytes(scaled), (127 - e).astype(np.uint8)


def q_operand(form: int, P: np.ndarray, right: bool) -> np.ndarray:
    """Dequantised tensor-core operand of a panel in (row, K) orientation, by
    the C oracle's OpenMP quantiser (the scalar conversions the numpy ones
    below are pinned to).  BF16X2 lays out three K segments: hi|hi|lo for the
    left operand and hi|lo|hi for the right one, so one product gives
    hi*hi + hi*lo + lo*hi."""
    P = np.asarray(P, np.float32)
    m, K = P.shape
    if form not in (FORM_FP32, FORM_FP16, FORM_BF16, FORM_BF16X2, FORM_FP8):
        raise ValueError(f"unknown form {form}")
    out = np.empty((m, K * (3 if form == FORM_BF16X2 else 1)), np.float32, order="F")
    if not (m and K):
        return out
    s0, s1 = P.strides
    if s0 == 4 and s1 % 4 == 0 and s1 >= 4 * m:      # columns strided: a view of a column-major matrix
        ld, rowmajor = s1 // 4, 0
    elif s1 == 4 and s0 % 4 == 0 and s0 >= 4 * K:    # rows strided: the transpose of such a view
        ld, rowmajor = s0 // 4, 1
    else:
        P = np.asfortranarray(P)
        ld, rowmajor = m, 0
    O.lib().orc_quantise(form, int(right), m, K, P.ctypes.data, ld, rowmajor, out.ctypes.data)
    return out


def q_operand_np(form: int, P: np.ndarray, right: bool) -> np.ndarray:
    """q_operand by the vectorised numpy quantisers (used to pin them)."""
    P = np.asarray(P, np.float32)
    if form == FORM_FP32:
        return np.array(P, np.float32)
    if form == FORM_FP16:
        return f16_round(P)
    if form == FORM_BF16:
        return bf16_round(P)
    if form == FORM_BF16X2:
        hi = bf16_round(P)
        lo = bf16_round(P - hi)
        return np.concatenate([hi, lo, hi] if right else [hi, hi, lo], axis=1)
    if form == FORM_FP8:
        return fp8_panel(P)[0]
    raise ValueError(f"unknown form {form}")


def qgemm(form: int, P: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """P (m x K) times Q (K x n) with both operands quantised to `form` and the
    products summed in FP32 (C = acc of the product's store mode)."""
    lq = q_operand(form, P, right=False)
    rq = q_operand(form, np.asarray(Q, np.float32).T, right=True)
    return np.asfortranarray((rq @ lq.T).T, np.float32)


def _ptr(A: np.ndarray, i: int = 0, j: int = 0) -> int:
    assert A.flags.f_contiguous and A.dtype == np.float32
    return A.ctypes.data + 4 * (i + j * A.shape[0])


# ---------------------------------------------------------------------------
# diagonal block: LU and triangular inverses
# ---------------------------------------------------------------------------
def inv_tc_start(b: int, inv_tc: int) -> int:
    """First doubling level run as low-precision products (0: none), as the
    product decides it: only when two blocks of that size fit in b."""
    return inv_tc if inv_tc > 0 and 2 * inv_tc <= b else 0


def tri_inverses(A: np.ndarray, r: int, b: int, inv_tc: int = 1024, tform: int = FORM_BF16X2):
    """(inv(U), inv(L)) of the factored b x b diagonal block of A at (r, r)."""
    XU = np.zeros((b, b), np.float32, order="F")
    XL = np.zeros((b, b), np.float32, order="F")
    s0 = inv_tc_start(b, inv_tc)
    O.lib().orc_tri_inverses(b, _ptr(A, r, r), A.shape[0], XU.ctypes.data, XL.ctypes.data, b, s0)
    if s0:
        D = A[r:r + b, r:r + b]
        S = s0
        while S < b:
            npair = b // (2 * S)
            c = b - npair * 2 * S - S
            for p in range(npair + 1):
                s2 = S if p < npair else c
                if s2 <= 0:
                    break
                r0, r1 = p * 2 * S, p * 2 * S + S
                T = qgemm(tform, D[r0:r0 + S, r1:r1 + s2], XU[r1:r1 + s2, r1:r1 + s2])
                XU[r0:r0 + S, r1:r1 + s2] = -qgemm(tform, XU[r0:r0 + S, r0:r0 + S], T)
                T = qgemm(tform, D[r1:r1 + s2, r0:r0 + S], XL[r0:r0 + S, r0:r0 + S])
                XL[r1:r1 + s2, r0:r0 + S] = -qgemm(tform, XL[r1:r1 + s2, r1:r1 + s2], T)
            S *= 2
    return XU, XL


def getrf_nopiv_inv(A: np.ndarray, inv_tc: int = 1024, tform: int = FORM_BF16X2):
    """In-place LU of the square F-ordered FP32 block A plus its inverses
    (oracle of mxp_getrf_nopiv_inv).  Returns (info, XU, XL)."""
    n = A.shape[0]
    info = O.lib().orc_getrf_nopiv_blocked(n, _ptr(A), n)
    if info:
        return info, None, None
    XU, XL = tri_inverses(A, 0, n, inv_tc, tform)
    return 0, XU, XL


# ---------------------------------------------------------------------------
# whole blocked LU
# ---------------------------------------------------------------------------
def panel_lu(A: np.ndarray, b: int, form: int = FORM_FP16, trsm: str = "split", inv_tc: int = 1024,
             chunk: int = 4096, keep_panels: bool = False):
    """Blocked no-pivot LU of the F-ordered FP32 matrix A in place.

    form: the Schur operands (FP16, BF16X2, FP8); trsm: "split", "single" or
    "fp32" (plain STRSM).  Returns 0, or 1 + the global index of the first
    bad pivot.  keep_panels: also return the FP32 L and U^T panels of every
    step (for checks of the product's low-precision panel copies)."""
    assert A.flags.f_contiguous and A.dtype == np.float32
    n = A.shape[0]
    nb = n // b
    lib = O.lib()
    panels = []
    for k in range(nb):
        kk = k * b
        info = lib.orc_getrf_nopiv_blocked(b, _ptr(A, kk, kk), n)
        if info:
            return (kk + info, panels) if keep_panels else kk + info
        m = n - kk - b
        if m <= 0:
            break
        if trsm == "fp32":
            lib.orc_trsm_runn(m, b, _ptr(A, kk, kk), n, _ptr(A, kk + b, kk), n)
            lib.orc_trsm_llnu(b, m, _ptr(A, kk, kk), n, _ptr(A, kk, kk + b), n)
        else:
            tform = TRSM_FORMS[trsm]
            XU, XL = tri_inverses(A, kk, b, inv_tc, tform)
            A[kk + b:, kk:kk + b] = qgemm(tform, A[kk + b:, kk:kk + b], XU)
            A[kk:kk + b, kk + b:] = qgemm(tform, XL, A[kk:kk + b, kk + b:])
        L = A[kk + b:, kk:kk + b]
        Ut = A[kk:kk + b, kk + b:].T
        if keep_panels:
            panels.append((np.array(L), np.array(Ut)))
        lq = q_operand(form, L, right=False)
        rq = q_operand(form, Ut, right=True)
        for c0 in range(0, m, chunk):
            c1 = min(m, c0 + chunk)
            # (R L^T)^T: the product comes out column-major like A
            A[kk + b:, kk + b + c0:kk + b + c1] -= (rq[c0:c1] @ lq.T).T
    return (0, panels) if keep_panels else 0
