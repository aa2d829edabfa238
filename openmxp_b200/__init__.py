"""openmxp_b200: B200-native single-GPU HPL-MxP solve path.

Python mirror of the reference's host interface for the path (panel_matgen_dev,
panel_lu_async_wGPU, iterative_refinement2, otf_gemv, the panel casts and the
Schur gemm_ex), calling the CUDA library libmxp.so through its C ABI
(include/mxp.h).  torch provides device memory and streams only.  There is no
CPU fallback: every call fails loudly when the extension is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmxp.so")

# enums of include/mxp.h
OK, INVALID_ARG, ZERO_PIVOT, NONFINITE, NOT_CONVERGED, TIMEOUT, CUDA_ERROR, UNSUPPORTED, NO_MEMORY = range(9)
FORM_FP16, FORM_BF16X2, FORM_FP8 = 0, 1, 2
FORMS = {"fp16": FORM_FP16, "bf16x2": FORM_BF16X2, "fp8": FORM_FP8}
DIAG_ROWSUM, DIAG_055_PLUS1 = 0, 1
IR_CLASSIC, IR_GMRES = 0, 1
STATUS_NAMES = ["OK", "INVALID_ARG", "ZERO_PIVOT", "NONFINITE", "NOT_CONVERGED", "TIMEOUT",
                "CUDA_ERROR", "UNSUPPORTED", "NO_MEMORY"]


class MxpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")


class LuStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_diag_lu", C.c_double), ("ms_trsm", C.c_double),
                ("ms_cast", C.c_double), ("ms_schur", C.c_double), ("info", C.c_int),
                ("schur_launches", C.c_int), ("ms_trsm_inv", C.c_double), ("ms_trsm_gemm", C.c_double),
                ("overlapped_diag", C.c_int), ("pad", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class IrStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("hpl_harness", C.c_double), ("norma", C.c_double), ("normb", C.c_double),
                ("normx", C.c_double), ("ms_total", C.c_double), ("ms_gemv", C.c_double),
                ("ms_trsv", C.c_double), ("gemv_calls", C.c_int), ("trsv_calls", C.c_int),
                ("inner_iterations", C.c_int), ("history", C.c_double * 64),
                ("history_residual", C.c_double * 64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("history")}
        d["history"] = [self.history[i] for i in range(min(64, self.iterations + 1))]
        return d


class PanelView(C.Structure):
    _fields_ = [("data", C.c_void_p), ("ld", C.c_int64), ("slot_k", C.c_int64), ("esize", C.c_int),
                ("slots", C.c_int), ("rows", C.c_int64), ("scales", C.c_void_p), ("sc_ld", C.c_int),
                ("sc_slot", C.c_int)]


class BatchResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("info", C.c_int), ("pad", C.c_int),
                ("hpl_harness", C.c_double), ("residual", C.c_double)]


class BatchStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("b", C.c_int), ("tile_n", C.c_int), ("stages", C.c_int),
                ("autotuned", C.c_int), ("grid", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_vp, _i32, _i64, _u64, _dbl = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double

# name -> (restype, argtypes); mirrors include/mxp.h
_SIGS = {
    "mxp_version": (C.c_char_p, []),
    "mxp_last_error_string": (C.c_char_p, []),
    "mxp_workspace_create": (_i32, [_i32, _i32, _i32, _i32, C.POINTER(_vp)]),
    "mxp_workspace_destroy": (_i32, [_vp]),
    "mxp_workspace_bytes": (C.c_size_t, [_i32, _i32, _i32]),
    "mxp_workspace_set_option": (_i32, [_vp, _i32, _i32]),
    "mxp_workspace_panel_view": (_i32, [_vp, _i32, C.POINTER(PanelView)]),
    "mxp_matgen": (_i32, [_i32, _u64, _i32, _vp, _i64, _vp, _vp, _vp, _vp]),
    "mxp_matgen_f64": (_i32, [_i32, _u64, _i32, _vp, _i64, _vp]),
    "mxp_getrf_nopiv": (_i32, [_i32, _vp, _i64, _vp, _vp]),
    "mxp_getrf_nopiv_inv": (_i32, [_i32, _vp, _i64, _vp, _vp, _i64, _vp, _vp]),
    "mxp_trsm_right_upper": (_i32, [_i32, _i32, _vp, _i64, _vp, _i64, _vp]),
    "mxp_trsm_left_lower_unit": (_i32, [_i32, _i32, _vp, _i64, _vp, _i64, _vp]),
    "mxp_half_conversion_left": (_i32, [_vp, _i32, _i32, _i64, _vp, _i64, _vp]),
    "mxp_half_conversion_right_trans": (_i32, [_vp, _i32, _i32, _i64, _vp, _i64, _vp]),
    "mxp_panel_cast_left": (_i32, [_i32, _i32, _i32, _vp, _i64, _vp, _i64, _vp, _vp]),
    "mxp_panel_cast_right": (_i32, [_i32, _i32, _i32, _vp, _i64, _vp, _i64, _vp, _vp]),
    "mxp_schur_update": (_i32, [_i32, _i32, _i32, _i32, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _i64,
                                _vp, _vp]),
    "mxp_panel_lu": (_i32, [_i32, _i32, _vp, _i64, _vp, _vp, C.POINTER(LuStats)]),
    "mxp_otf_gemv": (_i32, [_i32, _u64, _vp, _dbl, _vp, _dbl, _vp, _vp, _vp]),
    "mxp_lu_solve": (_i32, [_i32, _vp, _i64, _vp, _vp, _vp]),
    "mxp_iterative_refinement": (_i32, [_i32, _u64, _vp, _i64, _vp, _vp, _vp, _vp, _dbl, _i32,
                                        _i32, _vp, _vp, C.POINTER(IrStats)]),
    "mxp_solve": (_i32, [_i32, _i32, _u64, _vp, _i64, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp,
                         C.POINTER(LuStats), C.POINTER(IrStats)]),
    "mxp_solve_host": (_i32, [_i32, _i32, _u64, _vp, _i64, _vp, _vp, _vp, _vp, _i32, _i32, _vp,
                              _vp, C.POINTER(LuStats), C.POINTER(IrStats)]),
    "mxp_infnorm": (_i32, [_i32, _vp, C.POINTER(_dbl), _vp, _vp]),
    "mxp_check_reciprocal": (_i32, [C.POINTER(_u64), C.POINTER(_u64)]),
    "mxp_trsm_inv_right_upper": (_i32, [_i32, _i32, _vp, _i64, _vp, _i64, _i32, _vp, _vp]),
    "mxp_trsm_inv_left_lower": (_i32, [_i32, _i32, _vp, _i64, _vp, _i64, _i32, _vp, _vp]),
    "mxp_local_extent": (_i32, [_i32, _i32, _i32, _i32, C.POINTER(_i64)]),
    "mxp_matgen_local": (_i32, [_i32, _i32, _u64, _i32, _i32, _i32, _i32, _vp, _vp, _i64, _vp]),
    "mxp_otf_gemv_local": (_i32, [_i32, _i32, _u64, _i32, _i32, _i32, _i32, _vp, _dbl, _vp, _vp, _vp]),
    "mxp_block_gemv": (_i32, [_i32, _i32, _dbl, _vp, _i64, _vp, _dbl, _vp, _vp]),
    "mxp_batch_sizes": (_i32, [_i32, _u64, C.POINTER(C.c_int)]),
    "mxp_batch_partition": (_i32, [_i32, C.POINTER(C.c_int), _i32, C.POINTER(C.c_int)]),
    "mxp_batch_create": (_i32, [_i32, C.POINTER(C.c_int), C.POINTER(C.c_uint64), _i32, C.POINTER(_vp)]),
    "mxp_batch_destroy": (_i32, [_vp]),
    "mxp_batch_layout": (_i32, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "mxp_batch_matgen": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "mxp_batch_set_config": (_i32, [_vp, _i32, _i32, _i32]),
    "mxp_batch_autotune": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _vp, C.POINTER(BatchStats)]),
    "mxp_batch_solve": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _vp, C.POINTER(BatchStats)]),
    "mxp_batch_results": (_i32, [_vp, C.POINTER(BatchResult)]),
    "mxp_higham_params": (_i32, [_i32, _dbl, _dbl, C.POINTER(_dbl), C.POINTER(_dbl)]),
    "mxp_matgen_higham": (_i32, [_i32, _dbl, _dbl, _u64, _vp, _i64, _vp, _vp, _vp]),
    "mxp_higham_gemv": (_i32, [_i32, _dbl, _dbl, _dbl, _vp, _dbl, _vp, _vp]),
    "mxp_higham_infnorm": (_i32, [_i32, _dbl, _dbl, C.POINTER(_dbl)]),
    "mxp_workspace_set_matrix_higham": (_i32, [_vp, _dbl, _dbl]),
    "mxp_kernel_launches": (_i64, []),
    "mxp_reset_kernel_launches": (None, []),
}


def lib() -> C.CDLL:
    """Load libmxp.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m openmxp_b200.build` "
                              "(or __graft_entry__.build()) first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise MxpError(status, lib().mxp_last_error_string().decode())


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


# ---------------------------------------------------------------------------
# workspace (LRPanels / Workspace of the reference, panel.hpp:169-187, 321-454)
# ---------------------------------------------------------------------------
OPT_TRSM_TENSOR = 1
OPT_GMRES_RESTART = 2
OPT_GMRES_TOL_EXP = 3
OPT_MERGE_PANELS = 4
OPT_SCHUR_PAIR = 5
OPT_DIAG_COOP = 6
OPT_TRSM_PAIR = 7
OPT_TEST_WITHHOLD_FLAG = 8
OPT_OVERLAP_DIAG = 9
OPT_OVERLAP_MIN = 10
OPT_TRSM_SINGLE = 11
OPT_MERGE_DEPTH = 12
OPT_INV_TC = 13
OPT_TRSV_INV = 14
OPT_FP8_FUSED_CAST = 15
OPT_TRSM_COUNTER = 16


class Workspace:
    def __init__(self, n: int, b: int, form: int | str = FORM_FP16, device: int = 0,
                 trsm_tensor: bool = True, merge_panels: bool = True, schur_pair: bool = False,
                 diag_coop: bool = True, overlap_diag: int | None = None,
                 overlap_min: int | None = None, trsm_single: bool | None = None,
                 merge_depth: int | None = None):
        if isinstance(form, str):
            form = FORMS[form]
        self.n, self.b, self.form, self.device = n, b, form, device
        h = _vp()
        check(lib().mxp_workspace_create(n, b, form, device, C.byref(h)))
        self.handle = h
        self.set_option(OPT_TRSM_TENSOR, int(trsm_tensor))
        self.set_option(OPT_MERGE_PANELS, int(merge_panels))
        self.set_option(OPT_SCHUR_PAIR, int(schur_pair))
        self.set_option(OPT_DIAG_COOP, int(diag_coop))
        if overlap_diag is not None:
            self.set_option(OPT_OVERLAP_DIAG, int(overlap_diag))
        if overlap_min is not None:
            self.set_option(OPT_OVERLAP_MIN, int(overlap_min))
        if trsm_single is not None:
            self.set_option(OPT_TRSM_SINGLE, int(trsm_single))
        if merge_depth is not None:
            self.set_option(OPT_MERGE_DEPTH, int(merge_depth))

    def set_option(self, key: int, value: int) -> None:
        check(lib().mxp_workspace_set_option(self.handle, key, value))

    def set_matrix_higham(self, alpha: float, beta: float) -> None:
        """Refine against Higham's matrix (alpha, beta); (0, 0): the LCG matrix."""
        check(lib().mxp_workspace_set_matrix_higham(self.handle, alpha, beta))

    def panel_view(self, side: int) -> dict:
        """Device location of the low-precision L (side 0) or R (side 1) panel
        slots (mxp_workspace_panel_view)."""
        v = PanelView()
        check(lib().mxp_workspace_panel_view(self.handle, side, C.byref(v)))
        return {k: getattr(v, k) for k, _ in PanelView._fields_}

    def close(self):
        if self.handle:
            lib().mxp_workspace_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def bytes(n: int, b: int, form: int = FORM_FP16) -> int:
        return int(lib().mxp_workspace_bytes(n, b, form))


# ---------------------------------------------------------------------------
# matrices (Panels at a 1x1 grid: one column-major n x n FP32 matrix)
# ---------------------------------------------------------------------------
@dataclass
class Problem:
    n: int
    seed: int
    diag_rule: int
    A: "object"        # torch float32, n*lda elements, column-major
    lda: int
    d: "object"        # torch float64 [n]
    rowsum: "object"   # torch float64 [n]
    rhs: "object"      # torch float64 [n]

    def matrix(self):
        """A as an (n x n) torch view with A[i, j] = a_ij (column-major storage)."""
        return self.A.view(self.n, self.lda)[:, : self.n].t()


def panel_matgen(n: int, seed: int = 42, diag_rule: int = DIAG_ROWSUM, device=None,
                 A=None, lda: int | None = None, stream=None) -> Problem:
    """panel_matgen_dev + panel_colvgen (matgen.hpp:84-117, 419-436)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    lda = n if lda is None else lda
    if A is None:
        A = torch.empty(n * lda, dtype=torch.float32, device=dev)
    d = torch.empty(n, dtype=torch.float64, device=dev)
    rs = torch.empty(n, dtype=torch.float64, device=dev)
    rhs = torch.empty(n, dtype=torch.float64, device=dev)
    check(lib().mxp_matgen(n, seed, diag_rule, _ptr(A), lda, _ptr(d), _ptr(rs), _ptr(rhs),
                           _stream(stream)))
    return Problem(n, seed, diag_rule, A, lda, d, rs, rhs)


def matgen_f64(n: int, seed: int = 42, diag_rule: int = DIAG_ROWSUM, A=None, lda: int | None = None,
               stream=None):
    """The FP64 system refinement solves (FP64 off-diagonals, diagonal d), column-major."""
    import torch
    lda = n if lda is None else lda
    if A is None:
        A = torch.empty(n * lda, dtype=torch.float64,
                        device=torch.device("cuda", torch.cuda.current_device()))
    check(lib().mxp_matgen_f64(n, seed, diag_rule, _ptr(A), lda, _stream(stream)))
    return A


# ---------------------------------------------------------------------------
# Higham's HPL-AI matrix (HMGen, highammgen.hpp:4-30)
# ---------------------------------------------------------------------------
def higham_params(n: int, cond: float = 1e3, rho: float = 0.5):
    """(alpha, beta) of Higham's matrix for the estimated cond(A, inf) = cond."""
    a, b = C.c_double(), C.c_double()
    check(lib().mxp_higham_params(n, cond, rho, C.byref(a), C.byref(b)))
    return a.value, b.value


def higham_matgen(n: int, alpha: float, beta: float, seed: int = 42, device=None, stream=None) -> Problem:
    """pmatgen(HMGen) + pdiaggen (matgen.hpp:157-208, 399-417) and the LCG
    right-hand side of `seed`.  The Problem carries .alpha / .beta."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    A = torch.empty(n * n, dtype=torch.float32, device=dev)
    d = torch.empty(n, dtype=torch.float64, device=dev)
    rhs = torch.empty(n, dtype=torch.float64, device=dev)
    check(lib().mxp_matgen_higham(n, alpha, beta, seed, _ptr(A), n, _ptr(d), _ptr(rhs), _stream(stream)))
    p = Problem(n, seed, DIAG_ROWSUM, A, n, d, None, rhs)
    p.alpha, p.beta = alpha, beta
    return p


def higham_gemv(n, alpha, beta, a, x, b, y, stream=None):
    check(lib().mxp_higham_gemv(n, alpha, beta, a, _ptr(x), b, _ptr(y), _stream(stream)))


def higham_infnorm(n: int, alpha: float, beta: float) -> float:
    out = C.c_double()
    check(lib().mxp_higham_infnorm(n, alpha, beta, C.byref(out)))
    return out.value


def regenerate(p: Problem, stream=None) -> None:
    """Refill p.A (and d / rowsum / rhs) in place."""
    if getattr(p, "alpha", None) is not None:
        check(lib().mxp_matgen_higham(p.n, p.alpha, p.beta, p.seed, _ptr(p.A), p.lda, _ptr(p.d), _ptr(p.rhs),
                                      _stream(stream)))
        return
    check(lib().mxp_matgen(p.n, p.seed, p.diag_rule, _ptr(p.A), p.lda, _ptr(p.d), _ptr(p.rowsum),
                           _ptr(p.rhs), _stream(stream)))


# ---------------------------------------------------------------------------
# LU (panel_lu_async_wGPU, panel_trf.hpp:470-867)
# ---------------------------------------------------------------------------
def panel_lu(p: Problem, b: int, ws: Workspace, stream=None) -> dict:
    st = LuStats()
    check(lib().mxp_panel_lu(p.n, b, _ptr(p.A), p.lda, ws.handle, _stream(stream), C.byref(st)))
    return st.as_dict()


def getrf_nopiv(A, n: int, lda: int, ws: Workspace, stream=None) -> None:
    check(lib().mxp_getrf_nopiv(n, _ptr(A), lda, ws.handle, _stream(stream)))


def getrf_nopiv_inv(A, n: int, lda: int, XU, XL, ldx: int, ws: Workspace, stream=None) -> None:
    """In-place no-pivot LU of A plus inv(U) -> XU and inv(L) -> XL."""
    check(lib().mxp_getrf_nopiv_inv(n, _ptr(A), lda, _ptr(XU), _ptr(XL), ldx, ws.handle, _stream(stream)))


def trsm_right_upper(m, n, U, ldu, B, ldb, stream=None):
    check(lib().mxp_trsm_right_upper(m, n, _ptr(U), ldu, _ptr(B), ldb, _stream(stream)))


def trsm_left_lower_unit(m, n, L, ldl, B, ldb, stream=None):
    check(lib().mxp_trsm_left_lower_unit(m, n, _ptr(L), ldl, _ptr(B), ldb, _stream(stream)))


def trsm_inv_right_upper(m, b, XU, ldx, B, ldb, ws: "Workspace", single: bool = False, stream=None):
    """B (m x b) <- B * XU on the tensor cores (the reference's Alt-TRSM)."""
    check(lib().mxp_trsm_inv_right_upper(m, b, _ptr(XU), ldx, _ptr(B), ldb, int(single), ws.handle,
                                         _stream(stream)))


def trsm_inv_left_lower(b, m, XL, ldx, B, ldb, ws: "Workspace", single: bool = False, stream=None):
    """B (b x m) <- XL * B on the tensor cores (the reference's Alt-TRSM)."""
    check(lib().mxp_trsm_inv_left_lower(b, m, _ptr(XL), ldx, _ptr(B), ldb, int(single), ws.handle,
                                        _stream(stream)))


def half_conversion_left(Cm, m, b, plda, lp, lplda, stream=None):
    check(lib().mxp_half_conversion_left(_ptr(Cm), m, b, plda, _ptr(lp), lplda, _stream(stream)))


def half_conversion_right_trans(Cm, b, m, plda, rp, rplda, stream=None):
    check(lib().mxp_half_conversion_right_trans(_ptr(Cm), b, m, plda, _ptr(rp), rplda, _stream(stream)))


def panel_cast_left(form, m, b, A, lda, out, ldk, scales=None, stream=None):
    check(lib().mxp_panel_cast_left(form, m, b, _ptr(A), lda, _ptr(out), ldk, _ptr(scales),
                                    _stream(stream)))


def panel_cast_right(form, m, b, A, lda, out, ldk, scales=None, stream=None):
    check(lib().mxp_panel_cast_right(form, m, b, _ptr(A), lda, _ptr(out), ldk, _ptr(scales),
                                     _stream(stream)))


def schur_update(form, m, n, k, Lp, ldl, Rp, ldr, Cm, ldc, ws: Workspace, lscales=None,
                 rscales=None, stream=None):
    check(lib().mxp_schur_update(form, m, n, k, _ptr(Lp), ldl, _ptr(lscales), _ptr(Rp), ldr,
                                 _ptr(rscales), _ptr(Cm), ldc, ws.handle, _stream(stream)))


# ---------------------------------------------------------------------------
# refinement (iterative_refinement2, iterative_refinement.hpp:97-174)
# ---------------------------------------------------------------------------
def otf_gemv(n, seed, d, alpha, x, beta, y, ws: Workspace, stream=None):
    check(lib().mxp_otf_gemv(n, seed, _ptr(d), alpha, _ptr(x), beta, _ptr(y), ws.handle,
                             _stream(stream)))


def lu_solve(LU, n, lda, x, ws: Workspace, stream=None):
    check(lib().mxp_lu_solve(n, _ptr(LU), lda, _ptr(x), ws.handle, _stream(stream)))


def iterative_refinement(p: Problem, ws: Workspace, x=None, maxit: int = 50,
                         method: int = IR_CLASSIC, stream=None, raise_on_fail: bool = True):
    import torch
    if x is None:
        x = torch.empty(p.n, dtype=torch.float64, device=p.A.device)
    st = IrStats()
    rs = p.rowsum if p.diag_rule != DIAG_ROWSUM else None
    s = lib().mxp_iterative_refinement(p.n, p.seed, _ptr(p.A), p.lda, _ptr(p.d), _ptr(rs),
                                       _ptr(p.rhs), _ptr(x), 0.0, maxit, method, ws.handle,
                                       _stream(stream), C.byref(st))
    if raise_on_fail:
        check(s)
    return x, st.as_dict(), s


def solve(p: Problem, b: int, ws: Workspace, x=None, maxit: int = 50, method: int = IR_CLASSIC,
          stream=None):
    """LU then refinement: the timed region of main.cpp:617-657."""
    import torch
    if x is None:
        x = torch.empty(p.n, dtype=torch.float64, device=p.A.device)
    lst, ist = LuStats(), IrStats()
    rs = p.rowsum if p.diag_rule != DIAG_ROWSUM else None
    check(lib().mxp_solve(p.n, b, p.seed, _ptr(p.A), p.lda, _ptr(p.d), _ptr(rs), _ptr(p.rhs),
                          _ptr(x), maxit, method, ws.handle, _stream(stream), C.byref(lst),
                          C.byref(ist)))
    return x, lst.as_dict(), ist.as_dict()


def solve_host(p: Problem, b: int, ws: Workspace, h_rhs, h_x, maxit: int = 50,
               method: int = IR_CLASSIC, stream=None):
    """End-to-end call with host buffers (pinned torch CPU tensors)."""
    lst, ist = LuStats(), IrStats()
    rs = p.rowsum if p.diag_rule != DIAG_ROWSUM else None
    check(lib().mxp_solve_host(p.n, b, p.seed, _ptr(p.A), p.lda, _ptr(p.d), _ptr(rs), _ptr(h_rhs),
                               _ptr(h_x), maxit, method, ws.handle, _stream(stream), C.byref(lst),
                               C.byref(ist)))
    return lst.as_dict(), ist.as_dict()


def infnorm(x, ws: Workspace, stream=None) -> float:
    out = C.c_double(0.0)
    check(lib().mxp_infnorm(x.numel(), _ptr(x), C.byref(out), ws.handle, _stream(stream)))
    return out.value


def check_reciprocal() -> tuple[int, int]:
    """(mismatches, inputs checked) of the library's branch-free FP32
    reciprocal against the CUDA runtime's IEEE reciprocal (mxp_check_reciprocal)."""
    bad, n = _u64(0), _u64(0)
    check(lib().mxp_check_reciprocal(C.byref(bad), C.byref(n)))
    return int(bad.value), int(n.value)


def kernel_launches() -> int:
    return int(lib().mxp_kernel_launches())


def reset_kernel_launches() -> None:
    lib().mxp_reset_kernel_launches()


def hpl_flops(n: int) -> float:
    """Credited FLOPs of main.cpp:663: 2/3 n^3 + 3/2 n^2."""
    return 2.0 / 3.0 * n ** 3 + 1.5 * n ** 2


# ---------------------------------------------------------------------------
# batched form: many systems of uneven orders in one persistent launch
# ---------------------------------------------------------------------------
def batch_partition(sizes, nparts: int) -> list:
    """Part (0 .. nparts-1) of each system: largest first, each to the part with
    the least n^3 work so far (mxp_batch_partition)."""
    n = len(sizes)
    out = (C.c_int * n)()
    check(lib().mxp_batch_partition(n, (C.c_int * n)(*sizes), nparts, out))
    return list(out)


def batch_sizes(count: int, size_seed: int = 3) -> list:
    """Orders 128 * (2 + floor((v + 0.5) * 31)) from the generator stream of size_seed."""
    out = (C.c_int * count)()
    check(lib().mxp_batch_sizes(count, size_seed, out))
    return list(out)


class Batch:
    """count systems (orders n_list, generator seeds seeds) packed in one set of
    device buffers: A (FP32 matrices), d, rhs, x (FP64 vectors)."""

    def __init__(self, n_list, seeds, device: int = 0):
        import torch
        self.count = len(n_list)
        self.n = list(n_list)
        self.seeds = list(seeds)
        h = _vp()
        ns = (C.c_int * self.count)(*self.n)
        ss = (C.c_uint64 * self.count)(*self.seeds)
        check(lib().mxp_batch_create(self.count, ns, ss, device, C.byref(h)))
        self.handle = h
        mf, vd = C.c_int64(), C.c_int64()
        ao, vo = (C.c_int64 * self.count)(), (C.c_int64 * self.count)()
        check(lib().mxp_batch_layout(h, C.byref(mf), C.byref(vd), ao, vo))
        self.a_off, self.v_off = list(ao), list(vo)
        dev = torch.device("cuda", device)
        self.A = torch.empty(mf.value, dtype=torch.float32, device=dev)
        self.d = torch.empty(vd.value, dtype=torch.float64, device=dev)
        self.rhs = torch.empty(vd.value, dtype=torch.float64, device=dev)
        self.x = torch.empty(vd.value, dtype=torch.float64, device=dev)

    def matrix(self, i: int):
        """System i's matrix as an (n x n) torch view with [r, c] = a_rc."""
        n = self.n[i]
        return self.A[self.a_off[i]:self.a_off[i] + n * n].view(n, n).t()

    def vec(self, t, i: int):
        return t[self.v_off[i]:self.v_off[i] + self.n[i]]

    def matgen(self, stream=None) -> None:
        check(lib().mxp_batch_matgen(self.handle, _ptr(self.A), _ptr(self.d), _ptr(self.rhs), _stream(stream)))

    def set_config(self, b: int, tile_n: int = 256, stages: int = 4) -> None:
        check(lib().mxp_batch_set_config(self.handle, b, tile_n, stages))

    def autotune(self, sample: int = 0, stream=None) -> dict:
        st = BatchStats()
        check(lib().mxp_batch_autotune(self.handle, _ptr(self.A), _ptr(self.d), _ptr(self.rhs), _ptr(self.x),
                                       sample, _stream(stream), C.byref(st)))
        return st.as_dict()

    def solve(self, maxit: int = 50, stream=None) -> dict:
        st = BatchStats()
        check(lib().mxp_batch_solve(self.handle, _ptr(self.A), _ptr(self.d), _ptr(self.rhs), _ptr(self.x),
                                    maxit, _stream(stream), C.byref(st)))
        return st.as_dict()

    def results(self) -> list:
        out = (BatchResult * self.count)()
        check(lib().mxp_batch_results(self.handle, out))
        return [{k: getattr(r, k) for k, _ in BatchResult._fields_ if k != "pad"} for r in out]

    def close(self) -> None:
        if self.handle:
            lib().mxp_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
