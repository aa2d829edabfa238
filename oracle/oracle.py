"""ctypes view of the CPU oracle (oracle/mxp_oracle.c) and of the reference's
own CPU pieces compiled in place (oracle/_ref/libmxpref.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker -- never on the product
path of openmxp_b200.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libmxpref.so")

DIAG_ROWSUM = 0
DIAG_055_PLUS1 = 1
FORM_FP16, FORM_BF16X2, FORM_FP8, FORM_FP32 = 0, 1, 2, 3

_lib = None
_ref = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="F_CONTIGUOUS")
_vp = C.c_void_p


def build() -> None:
    """Compile the oracle (oracle/_ref is built by __graft_entry__.build)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        i64, u64, i32, dbl = C.c_int64, C.c_uint64, C.c_int, C.c_double
        L.orc_elem.argtypes = [i32, u64, i64, i64]
        L.orc_elem.restype = dbl
        L.orc_state.argtypes = [i32, u64, i64, i64]
        L.orc_state.restype = u64
        L.orc_aff_pow.argtypes = [u64, u64, u64, _vp, _vp]
        L.orc_matgen.argtypes = [i32, u64, i32, _vp, i64, _vp, _vp, _vp]
        L.orc_rowsum_row.argtypes = [i32, u64, i64]
        L.orc_rowsum_row.restype = dbl
        L.orc_matgen_f64.argtypes = [i32, u64, _vp, _vp, i64]
        L.orc_rowsum_cpu_order.argtypes = [i32, u64, i64]
        L.orc_rowsum_cpu_order.restype = dbl
        L.orc_f2h.argtypes = [C.c_float]
        L.orc_f2h.restype = C.c_uint16
        L.orc_h2f.argtypes = [C.c_uint16]
        L.orc_h2f.restype = C.c_float
        L.orc_f2bf.argtypes = [C.c_float]
        L.orc_f2bf.restype = C.c_uint16
        L.orc_f2e4m3.argtypes = [C.c_float]
        L.orc_f2e4m3.restype = C.c_uint8
        L.orc_e4m32f.argtypes = [C.c_uint8]
        L.orc_e4m32f.restype = C.c_float
        L.orc_e4m3_scale_exp.argtypes = [C.c_float]
        L.orc_e4m3_scale_exp.restype = i32
        L.orc_getrf_nopiv.argtypes = [i32, i32, _vp, i64]
        L.orc_getrf_nopiv.restype = i32
        L.orc_trsm_runn.argtypes = [i32, i32, _vp, i64, _vp, i64]
        L.orc_trsm_llnu.argtypes = [i32, i32, _vp, i64, _vp, i64]
        L.orc_getrf_nopiv_blocked.argtypes = [i32, _vp, i64]
        L.orc_getrf_nopiv_blocked.restype = i32
        L.orc_tri_inverses.argtypes = [i32, _vp, i64, _vp, _vp, i64, i32]
        L.orc_quantise.argtypes = [i32, i32, i32, i32, _vp, i64, i32, _vp]
        L.orc_higham_beta.argtypes = [i32, dbl, dbl]
        L.orc_higham_beta.restype = dbl
        L.orc_higham_matgen.argtypes = [i32, dbl, dbl, _vp, i64, _vp]
        L.orc_higham_matgen_cols.argtypes = [i32, dbl, dbl, i64, i64, _vp, i64]
        L.orc_higham_gemv.argtypes = [i32, dbl, dbl, dbl, _vp, dbl, _vp]
        L.orc_higham_matgen_f64.argtypes = [i32, dbl, dbl, _vp, i64]
        L.orc_higham_infnorm.argtypes = [i32, dbl, dbl]
        L.orc_higham_infnorm.restype = dbl
        L.orc_schur_update.argtypes = [i32, i32, i32, i32, _vp, i64, _vp, i64, _vp, i64]
        L.orc_panel_lu.argtypes = [i32, i32, _vp, i64, i32]
        L.orc_panel_lu.restype = i32
        L.orc_otf_gemv.argtypes = [i32, u64, _vp, dbl, _vp, dbl, _vp]
        L.orc_lu_solve.argtypes = [i32, _vp, i64, _vp]
        L.orc_lu_solve_ref1x1.argtypes = [i32, i32, _vp, i64, _vp]
        L.orc_infnorm.argtypes = [i32, _vp]
        L.orc_infnorm.restype = dbl
        L.orc_ir_classic.argtypes = [i32, i32, u64, _vp, i64, _vp, _vp, _vp, _vp, i32, i32,
                                     _vp, _vp, _vp]
        L.orc_ir_classic.restype = i32
        L.orc_solve.argtypes = [i32, i32, u64, i32, i32, i32, _vp, _vp]
        L.orc_solve.restype = i32
        L.orc_solve_ex.argtypes = [i32, i32, u64, i32, i32, i32, _vp, _vp, _vp, _vp]
        L.orc_solve_ex.restype = i32
        L.orc_num_threads.restype = i32
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref() -> C.CDLL:
    """The reference's own compiled CPU pieces (present only where the
    reference tree was available to build them)."""
    global _ref
    if _ref is None:
        R = C.CDLL(REF_PATH)
        i32, u64, sz, dbl = C.c_int, C.c_uint64, C.c_size_t, C.c_double
        R.ref_fill_one_panel_f32.argtypes = [i32, i32, i32, i32, i32, _vp, sz, u64, i32]
        R.ref_panel_fill_f64.argtypes = [i32, i32, i32, i32, i32, _vp, sz, u64]
        R.ref_calc_diag.argtypes = [i32, i32, u64]
        R.ref_calc_diag.restype = dbl
        R.ref_mat_elem.argtypes = [i32, i32, i32, i32]
        R.ref_mat_elem.restype = dbl
        R.ref_rand_pow.argtypes = [u64, u64, u64, _vp, _vp]
        R.ref_sgetrf_nopiv_naive.argtypes = [i32, i32, _vp, sz]
        R.ref_sgetrf_nopiv_tuned.argtypes = [i32, _vp, sz]
        R.ref_fp16_bits.argtypes = [C.c_float]
        R.ref_fp16_bits.restype = C.c_uint16
        R.otf_gemv_kernel.argtypes = [C.c_int64, i32, i32, dbl, _vp, _vp, u64]
        R.ref_getrf_diag.argtypes = [i32, _vp, C.c_int64]
        R.ref_getrf_diag.restype = i32
        R.ref_otf_gemv.argtypes = [i32, i32, u64, _vp, dbl, _vp, dbl, _vp]
        R.ref_higham_gemv.argtypes = [i32, i32, dbl, dbl, dbl, _vp, _vp]
        R.higham_mat_comp_beta.argtypes = [i32, dbl, dbl]
        R.higham_mat_comp_beta.restype = dbl
        _ref = R
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ----------------------------------------------------------------------------
# numpy-level helpers
# ----------------------------------------------------------------------------

def matgen(n: int, seed: int, diag_rule: int = DIAG_ROWSUM, with_matrix: bool = True):
    """(A float32 Fortran-ordered n x n, d, rowsum, rhs) in the GPU-pinned order."""
    A = np.empty((n, n), dtype=np.float32, order="F") if with_matrix else None
    d = np.empty(n, np.float64)
    rs = np.empty(n, np.float64)
    b = np.empty(n, np.float64)
    lib().orc_matgen(n, seed, diag_rule, _p(A) if A is not None else None, n, _p(d), _p(rs), _p(b))
    return A, d, rs, b


def matgen_f64(n: int, seed: int, d: np.ndarray) -> np.ndarray:
    """FP64 matrix the refinement solves (FP64 generator values, d on the diagonal)."""
    A = np.empty((n, n), dtype=np.float64, order="F")
    lib().orc_matgen_f64(n, seed, _p(d), _p(A), n)
    return A


def panel_lu(A: np.ndarray, b: int, form: int = FORM_FP16) -> int:
    assert A.flags.f_contiguous and A.dtype == np.float32
    n = A.shape[0]
    return lib().orc_panel_lu(n, b, _p(A), n, form)


def otf_gemv(n, seed, d, alpha, x, beta, y):
    lib().orc_otf_gemv(n, seed, _p(d), alpha, _p(x), beta, _p(y))
    return y


def lu_solve(LU: np.ndarray, x: np.ndarray) -> np.ndarray:
    n = LU.shape[0]
    lib().orc_lu_solve(n, _p(LU), n, _p(x))
    return x


def ir_classic(n, b, seed, LU, d, rowsum, rhs, maxit=50, ref1x1=False):
    x = np.empty(n, np.float64)
    resid = np.zeros(1)
    hpl = np.zeros(1)
    hist = np.zeros(maxit)
    it = lib().orc_ir_classic(n, b, seed, _p(LU), n, _p(d),
                              _p(rowsum) if rowsum is not None else None, _p(rhs), _p(x),
                              maxit, int(ref1x1), _p(resid), _p(hpl), _p(hist))
    return it, x, float(resid[0]), float(hpl[0]), hist


def solve(n, b, seed, diag_rule=DIAG_ROWSUM, form=FORM_FP16, maxit=50, ref_kernels=False):
    """Whole CPU solve (generation excluded from t_lu / t_ir).  ref_kernels:
    the diagonal blocks by the reference's compiled sgetrf_nopiv_omp<6> and the
    residual by its compiled otf_gemv_kernel (oracle/_ref), the rest by the
    oracle's restatement."""
    x = np.empty(n, np.float64)
    st = np.zeros(5)
    if ref_kernels:
        R = ref()
        rc = lib().orc_solve_ex(n, b, seed, diag_rule, form, maxit, _p(x), _p(st),
                                C.cast(R.ref_getrf_diag, C.c_void_p), C.cast(R.ref_otf_gemv, C.c_void_p))
    else:
        rc = lib().orc_solve(n, b, seed, diag_rule, form, maxit, _p(x), _p(st))
    return rc, x, {"t_lu": st[0], "t_ir": st[1], "resid": st[2], "hpl": st[3], "iters": int(st[4])}


def f2h_array(a: np.ndarray) -> np.ndarray:
    f = np.vectorize(lambda v: lib().orc_f2h(float(v)), otypes=[np.uint16])
    return f(a)


def f2bf_array(a: np.ndarray) -> np.ndarray:
    f = np.vectorize(lambda v: lib().orc_f2bf(float(v)), otypes=[np.uint16])
    return f(a)


def bf2f_array(a: np.ndarray) -> np.ndarray:
    return (a.astype(np.uint32) << 16).view(np.float32)


def f2e4m3_array(a: np.ndarray) -> np.ndarray:
    f = np.vectorize(lambda v: lib().orc_f2e4m3(float(v)), otypes=[np.uint8])
    return f(a)


def kmajor_panel(form: int, P: np.ndarray, right: bool):
    """Oracle of mxp_panel_cast_{left,right}: P is the m x b panel in
    row = output-row orientation (L column panel, or U^T for the right panel).
    Returns (raw K-major array, scales or None)."""
    m, b = P.shape
    P = np.asarray(P, np.float32)
    if form == FORM_FP16:
        return f2h_array(P), None
    if form == FORM_BF16X2:
        hi = f2bf_array(P)
        lo = f2bf_array((P - bf2f_array(hi)).astype(np.float32))
        segs = [hi, lo, hi] if right else [hi, hi, lo]
        return np.concatenate(segs, axis=1), None
    mt, kt = -(-m // 128), -(-b // 128)
    out = np.zeros((m, b), np.uint8)
    sc = np.zeros((mt, kt), np.uint8)
    for ti in range(mt):
        for tk in range(kt):
            blk = P[ti * 128:(ti + 1) * 128, tk * 128:(tk + 1) * 128]
            e = lib().orc_e4m3_scale_exp(float(np.max(np.abs(blk))) if blk.size else 0.0)
            sc[ti, tk] = 127 - e
            out[ti * 128:(ti + 1) * 128, tk * 128:(tk + 1) * 128] = f2e4m3_array(
                (blk * np.float32(2.0 ** e)).astype(np.float32))
    return out, sc


def schur_update(form: int, C: np.ndarray, L: np.ndarray, U: np.ndarray) -> np.ndarray:
    """C -= quant(L) quant(U^T)^T with FP32 accumulation (C, L, U Fortran float32)."""
    m, K = L.shape
    n = U.shape[1]
    C = np.asfortranarray(C.astype(np.float32, copy=True))
    L = np.asfortranarray(L, dtype=np.float32)
    U = np.asfortranarray(U, dtype=np.float32)
    lib().orc_schur_update(form, m, n, K, L.ctypes.data, m, U.ctypes.data, K, C.ctypes.data, m)
    return C


# ----------------------------------------------------------------------------
# Higham's HPL-AI matrix
# ----------------------------------------------------------------------------
def higham_params(n: int, cond: float, rho: float):
    """(alpha, beta) with alpha = rho * beta for cond(A, inf) = cond."""
    beta = lib().orc_higham_beta(n, cond, rho)
    return rho * beta, beta


def higham_matgen(n: int, alpha: float, beta: float, with_matrix: bool = True):
    """(A float32 Fortran-ordered, d float64)."""
    A = np.empty((n, n), np.float32, order="F") if with_matrix else None
    d = np.empty(n, np.float64)
    lib().orc_higham_matgen(n, alpha, beta, _p(A) if A is not None else None, n, _p(d))
    return A, d


def higham_matrix_f64(n: int, alpha: float, beta: float) -> np.ndarray:
    """The FP64 matrix the residual uses (entries regenerated in FP64)."""
    A = np.empty((n, n), np.float64, order="F")
    lib().orc_higham_matgen_f64(n, alpha, beta, _p(A), n)
    return A


def higham_gemv(n, alpha, beta, a, x, b, y):
    lib().orc_higham_gemv(n, alpha, beta, a, _p(x), b, _p(y))
    return y

