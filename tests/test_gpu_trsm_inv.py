"""mxp_trsm_inv_right_upper / mxp_trsm_inv_left_lower: the panel TRSM as a
tensor-core product with the triangle's inverse (the reference's Alt-TRSM,
panel_trf_gdirect.hpp:73-142), against the oracle's restatement of the same
product (oracle/blocked.py qgemm: the same BF16 or split-BF16 operands, FP32
sums).  The operands are bit-identical, only the order of the FP32 sums
differs, so every entry agrees within 1e-4 of the sum of its terms' sizes;
and the result solves the triangular system as the plain FP32 STRSM does, to
the product's precision."""
import numpy as np
import pytest

from oracle import blocked as Bk
from tests.gpu_util import from_np_colmajor, rel_fro, to_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("m,b", [(2560, 512), (3000, 1024), (700, 256)])
def test_trsm_inv_both_sides(mxp, orc, torch_cuda, single, m, b):
    torch = torch_cuda
    n = m + b
    A, _, _, _ = orc.matgen(n, 13)
    D = np.asfortranarray(A[:b, :b])
    dD = from_np_colmajor(torch, D)
    XU = torch.empty(b * b, device="cuda")
    XL = torch.empty(b * b, device="cuda")
    ws = mxp.Workspace(n, b, 0, trsm_single=single)
    mxp.getrf_nopiv_inv(dD, b, b, XU, XL, b, ws)
    LU = to_np_colmajor(dD, b, b, b)
    xu, xl = to_np_colmajor(XU, b, b, b), to_np_colmajor(XL, b, b, b)
    tform = Bk.FORM_BF16 if single else Bk.FORM_BF16X2
    # right side: the L panel below the block
    P = np.asfortranarray(A[b:, :b])
    dP = from_np_colmajor(torch, P, ld=m + 5)
    mxp.trsm_inv_right_upper(m, b, XU, b, dP, m + 5, ws, single=single)
    got = to_np_colmajor(dP, m, b, m + 5)
    want = Bk.qgemm(tform, P, xu)
    bound = np.abs(Bk.q_operand(tform, P, False)) @ np.abs(Bk.q_operand(tform, xu.T, True)).T
    assert np.all(np.abs(got.astype(np.float64) - want) <= 1e-4 * bound + 1e-30)
    # the plain FP32 STRSM gives the same panel to the product's precision
    ref = P.copy(order="F")
    orc.lib().orc_trsm_runn(m, b, np.asfortranarray(LU).ctypes.data, b, ref.ctypes.data, m)
    assert rel_fro(got, ref) <= (1e-2 if single else 1e-4)
    # left side: the U panel right of the block
    Q = np.asfortranarray(A[:b, b:])
    dQ = from_np_colmajor(torch, Q, ld=b + 3)
    mxp.trsm_inv_left_lower(b, m, XL, b, dQ, b + 3, ws, single=single)
    got = to_np_colmajor(dQ, b, m, b + 3)
    want = Bk.qgemm(tform, xl, Q)
    bound = np.abs(Bk.q_operand(tform, xl, False)) @ np.abs(Bk.q_operand(tform, Q.T, True)).T
    assert np.all(np.abs(got.astype(np.float64) - want) <= 1e-4 * bound + 1e-30)
    ref = Q.copy(order="F")
    orc.lib().orc_trsm_llnu(b, m, np.asfortranarray(LU).ctypes.data, b, ref.ctypes.data, b)
    assert rel_fro(got, ref) <= (1e-2 if single else 1e-4)
    ws.close()


def test_trsm_inv_rejects_long_panel(mxp, torch_cuda):
    torch = torch_cuda
    ws = mxp.Workspace(1024, 256, 0)
    X = torch.zeros(256 * 256, device="cuda")
    B = torch.zeros(1024 * 256, device="cuda")
    with pytest.raises(mxp.MxpError):
        mxp.trsm_inv_right_upper(1000, 256, X, 256, B, 1000, ws)  # m > n - b
    ws.close()
