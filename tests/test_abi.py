"""The C-ABI library loads without a GPU, exports every function declared in
include/mxp.h, and rejects bad arguments on the host before touching CUDA."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mxp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mxp_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("mxp_matgen", "mxp_panel_lu", "mxp_schur_update", "mxp_otf_gemv",
                 "mxp_iterative_refinement", "mxp_solve", "mxp_solve_host"):
        assert must in names


def test_library_exports_every_declared_symbol(mxp):
    L = mxp.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_sizes(mxp):
    assert b"sm_100a" in mxp.lib().mxp_version()
    # C3: FP16 panels 4 x (N-B) x B x 2 bytes, vectors, and the inverses of
    # the 48 diagonal blocks kept for the refinement (2 x N x B x 4 bytes)
    nbytes = mxp.Workspace.bytes(122880, 2560, mxp.FORM_FP16)
    assert 2.4e9 + 2 * 122880 * 2560 * 4 < nbytes < 10e9
    assert mxp.Workspace.bytes(122880, 2560, mxp.FORM_BF16X2) > 2.9 * 2.4e9


def test_host_side_argument_checks(mxp):
    L = mxp.lib()
    h = C.c_void_p()
    assert L.mxp_workspace_create(0, 64, 0, 0, C.byref(h)) == mxp.INVALID_ARG
    assert L.mxp_workspace_create(128, 256, 0, 0, C.byref(h)) == mxp.INVALID_ARG
    assert L.mxp_workspace_create(128, 64, 9, 0, C.byref(h)) == mxp.INVALID_ARG
    assert L.mxp_matgen(0, 1, 0, None, 1, None, None, None, None) == mxp.INVALID_ARG
    assert L.mxp_matgen(16, 1, 5, None, 16, None, None, None, None) == mxp.INVALID_ARG
    assert L.mxp_panel_lu(128, 64, None, 128, None, None, None) == mxp.INVALID_ARG
    assert b"NULL" in L.mxp_last_error_string()
    assert L.mxp_otf_gemv(16, 1, None, 1.0, None, 0.0, None, None, None) == mxp.INVALID_ARG
    with pytest.raises(mxp.MxpError) as e:
        mxp.check(mxp.INVALID_ARG)
    assert "INVALID_ARG" in str(e.value)


def test_panel_cast_argument_checks(mxp):
    L = mxp.lib()
    # ldk smaller than the K extent of the form (3b for BF16X2)
    assert L.mxp_panel_cast_left(1, 16, 64, None, 16, None, 128, None, None) == mxp.INVALID_ARG
    assert L.mxp_panel_cast_left(2, 16, 64, None, 16, None, 64, None, None) == mxp.INVALID_ARG  # FP8 needs scales
    assert L.mxp_panel_cast_right(7, 16, 64, None, 64, None, 64, None, None) == mxp.INVALID_ARG


def test_flop_credit():
    import bench
    assert bench.hpl_flops(8192) == pytest.approx(3.666e11, rel=1e-3)
    assert bench.hpl_flops(122880) == pytest.approx(1.2370e15, rel=1e-4)
    assert bench.schur_flops(122880, 2560, 1) == pytest.approx(1.20e15, rel=2e-2)
