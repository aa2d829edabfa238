"""Single-product TRSM by inverse (MXP_OPT_TRSM_SINGLE): the panel solves
X_L = A21 inv(U11) and X_U = inv(L11) A12 as one BF16 x BF16 -> FP32
tensor-core product each (K = b) instead of the three split-BF16 products.
The operand rounding (2^-9 relative) bounds the factor error; the solve must
still reach the scaled-residual threshold through refinement."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [0, 2])
@pytest.mark.parametrize("n,b,seed", [(1024, 128, 7), (2048, 256, 11), (1536, 512, 42)])
def test_single_trsm_factors(mxp, orc, torch_cuda, form, n, b, seed):
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form, trsm_single=True)
    mxp.panel_lu(p, b, ws)
    got = to_np_colmajor(p.A, n, n, n)
    A, _, _, _ = orc.matgen(n, seed, 0)
    assert orc.panel_lu(A, b, form) == 0
    # BF16 operands: a few 2^-9 relative per product
    assert rel_fro(got, A) <= 1e-2
    low = np.tril(np.ones((n, n), bool), -1)
    assert rel_fro(got[low], A[low]) <= 1e-2


def test_single_trsm_differs_from_split(mxp, torch_cuda):
    # the option really changes the path: factors differ from the split form's
    n, b = 1024, 128
    p1 = mxp.panel_matgen(n, 3)
    p2 = mxp.panel_matgen(n, 3)
    mxp.panel_lu(p1, b, mxp.Workspace(n, b, 0))
    mxp.panel_lu(p2, b, mxp.Workspace(n, b, 0, trsm_single=True))
    a1 = to_np_colmajor(p1.A, n, n, n)
    a2 = to_np_colmajor(p2.A, n, n, n)
    assert not np.array_equal(a1, a2)
    assert rel_fro(a2, a1) <= 1e-2


@pytest.mark.parametrize("form", [0, 2])
@pytest.mark.parametrize("method", [0, 1])
def test_single_trsm_solve(mxp, torch_cuda, form, method):
    n, b = 4096, 256
    p = mxp.panel_matgen(n, 21)
    ws = mxp.Workspace(n, b, form, trsm_single=True)
    _, lu, ir = mxp.solve(p, b, ws, method=method)
    assert ir["converged"]
    assert ir["hpl_harness"] < 16.0
