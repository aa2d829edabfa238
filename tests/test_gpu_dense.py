"""FP32 diagonal LU and panel TRSMs vs the oracle (tolerance: FP32 rounding
of a different but equivalent summation order)."""
import numpy as np
import pytest

from tests.gpu_util import from_np_colmajor, to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coop", [True, False])
@pytest.mark.parametrize("n,pad", [(64, 0), (200, 7), (512, 0), (1000, 24), (2560, 0)])
def test_getrf_nopiv(mxp, orc, torch_cuda, n, pad, coop):
    """coop: the single cooperative launch (grid barriers) vs one launch per 64 columns."""
    torch = torch_cuda
    A, _, _, _ = orc.matgen(n, 5)
    dA = from_np_colmajor(torch, A, ld=n + pad)
    ws = mxp.Workspace(n, n, 0, diag_coop=coop)
    mxp.getrf_nopiv(dA, n, n + pad, ws)
    got = to_np_colmajor(dA, n, n, n + pad)
    ref = A.copy(order="F")
    assert orc.lib().orc_getrf_nopiv(n, n, ref.ctypes.data, n) == 0
    assert rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("coop", [True, False])
@pytest.mark.parametrize("n", [64, 200, 1000, 2560])
def test_getrf_nopiv_inv(mxp, orc, torch_cuda, n, coop):
    """LU plus both triangular inverses: X_U U = I and X_L L = I to FP32 accuracy."""
    torch = torch_cuda
    A, _, _, _ = orc.matgen(n, 3)
    dA = from_np_colmajor(torch, A)
    XU = torch.full((n * n,), float("nan"), dtype=torch.float32, device="cuda")
    XL = torch.full((n * n,), float("nan"), dtype=torch.float32, device="cuda")
    ws = mxp.Workspace(max(n, 128), n, 0, diag_coop=coop)
    ws.set_option(mxp.OPT_INV_TC, 0)  # every level in FP32 (the tensor-core levels: below)
    mxp.getrf_nopiv_inv(dA, n, n, XU, XL, n, ws)
    LU = to_np_colmajor(dA, n, n, n).astype(np.float64)
    U = np.triu(LU)
    L = np.tril(LU, -1) + np.eye(n)
    xu = to_np_colmajor(XU, n, n, n).astype(np.float64)
    xl = to_np_colmajor(XL, n, n, n).astype(np.float64)
    assert np.array_equal(np.tril(xu, -1), np.zeros((n, n)))
    assert np.array_equal(np.triu(xl, 1), np.zeros((n, n)))
    assert np.abs(xu @ U - np.eye(n)).max() < 1e-5
    assert np.abs(xl @ L - np.eye(n)).max() < 1e-5
    ref = A.copy(order="F")
    assert orc.lib().orc_getrf_nopiv(n, n, ref.ctypes.data, n) == 0
    assert rel_fro(LU, ref) < 1e-6


@pytest.mark.parametrize("coop", [True, False])
def test_getrf_zero_pivot_reported(mxp, orc, torch_cuda, coop):
    torch = torch_cuda
    n = 128
    A, _, _, _ = orc.matgen(n, 5)
    A[70, 70] = 0.0
    A[70, :] = 0.0           # row 70 all zero -> pivot 70 is exactly zero
    dA = from_np_colmajor(torch, A)
    ws = mxp.Workspace(n, n, 0, diag_coop=coop)
    with pytest.raises(mxp.MxpError) as e:
        mxp.getrf_nopiv(dA, n, n, ws)
    assert e.value.status == mxp.ZERO_PIVOT


@pytest.mark.parametrize("m,n", [(1000, 64), (333, 200), (4096, 256)])
def test_trsm_right_upper(mxp, orc, torch_cuda, m, n):
    torch = torch_cuda
    U, _, _, _ = orc.matgen(n, 9)
    assert orc.lib().orc_getrf_nopiv(n, n, U.ctypes.data, n) == 0
    rng = np.random.default_rng(m)
    B = rng.uniform(-0.5, 0.5, (m, n)).astype(np.float32)
    dU = from_np_colmajor(torch, U)
    dB = from_np_colmajor(torch, B, ld=m + 1)
    mxp.trsm_right_upper(m, n, dU, n, dB, m + 1)
    got = to_np_colmajor(dB, m, n, m + 1)
    ref = np.asfortranarray(B.copy())
    orc.lib().orc_trsm_runn(m, n, U.ctypes.data, n, ref.ctypes.data, m)
    assert rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("m,n", [(64, 1000), (200, 333), (256, 4096)])
def test_trsm_left_lower_unit(mxp, orc, torch_cuda, m, n):
    torch = torch_cuda
    Lm, _, _, _ = orc.matgen(m, 9)
    assert orc.lib().orc_getrf_nopiv(m, m, Lm.ctypes.data, m) == 0
    rng = np.random.default_rng(n)
    B = rng.uniform(-0.5, 0.5, (m, n)).astype(np.float32)
    dL = from_np_colmajor(torch, Lm)
    dB = from_np_colmajor(torch, B)
    mxp.trsm_left_lower_unit(m, n, dL, m, dB, m)
    got = to_np_colmajor(dB, m, n, m)
    ref = np.asfortranarray(B.copy())
    orc.lib().orc_trsm_llnu(m, n, Lm.ctypes.data, m, ref.ctypes.data, m)
    assert rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("n,start,single", [(512, 128, False), (1000, 128, False), (2560, 1024, False),
                                            (2560, 512, False), (1536, 256, True)])
def test_getrf_nopiv_inv_tensor_levels(mxp, orc, torch_cuda, n, start, single):
    """The large doubling levels of the inverses as tensor-core products
    (MXP_OPT_INV_TC): split-BF16 products keep X U = I to ~1e-5 (about 16
    mantissa bits per operand); one BF16 product to ~1e-2.  The LU itself is
    unchanged and the zero triangles stay exactly zero."""
    torch = torch_cuda
    A, _, _, _ = orc.matgen(n, 3)
    dA = from_np_colmajor(torch, A)
    XU = torch.full((n * n,), float("nan"), dtype=torch.float32, device="cuda")
    XL = torch.full((n * n,), float("nan"), dtype=torch.float32, device="cuda")
    ws = mxp.Workspace(n, n, 0, trsm_single=single)
    ws.set_option(mxp.OPT_INV_TC, start)
    mxp.getrf_nopiv_inv(dA, n, n, XU, XL, n, ws)
    LU = to_np_colmajor(dA, n, n, n).astype(np.float64)
    U = np.triu(LU)
    L = np.tril(LU, -1) + np.eye(n)
    xu = to_np_colmajor(XU, n, n, n).astype(np.float64)
    xl = to_np_colmajor(XL, n, n, n).astype(np.float64)
    assert np.array_equal(np.tril(xu, -1), np.zeros((n, n)))
    assert np.array_equal(np.triu(xl, 1), np.zeros((n, n)))
    tol = 1e-2 if single else 1e-4
    assert np.abs(xu @ U - np.eye(n)).max() < tol
    assert np.abs(xl @ L - np.eye(n)).max() < tol
    ref = A.copy(order="F")
    assert orc.lib().orc_getrf_nopiv(n, n, ref.ctypes.data, n) == 0
    assert rel_fro(LU, ref) < 1e-6


def test_inv_tc_option_bounds(mxp, torch_cuda):
    ws = mxp.Workspace(512, 128, 0)
    for bad in (-1, 64, 300):
        with pytest.raises(mxp.MxpError):
            ws.set_option(mxp.OPT_INV_TC, bad)
    ws.set_option(mxp.OPT_INV_TC, 0)


def test_branch_free_reciprocal(mxp, torch_cuda):
    """The 64 x 64 LU forms its multipliers with a branch-free FP32 reciprocal
    (FP64 Newton steps from the hardware approximation, rounded once); it must
    equal the CUDA runtime's IEEE round-to-nearest reciprocal bit for bit on
    every normal input checked (all signs and exponents, 65536 mantissas each)."""
    bad, n = mxp.check_reciprocal()
    assert n == 2 * 254 * 65536
    assert bad == 0
