"""Higham's HPL-AI matrix family on the GPU against the oracle: parameters,
the FP32 matrix and FP64 diagonal bit for bit, the FP64 residual GEMV bit for
bit (the same sums in the same order), and a whole solve -- the blocked LU of
the Higham matrix, refined against it -- to scaled residual < 16 with the
forward error of an FP64 solve; the factors are checked as the reference's
panel_check does (panel_check.hpp:66-110: L's strictly lower entries against
alpha, U's strictly upper ones against beta, U's diagonal against 1)."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,cond,rho", [(1000, 1e3, 0.5), (4096, 1e4, 0.125), (61440, 1e6, 0.5),
                                        (122880, 1e4, 0.5)])
def test_params_match_oracle(mxp, orc, n, cond, rho):
    a, b = mxp.higham_params(n, cond, rho)
    assert b == orc.lib().orc_higham_beta(n, cond, rho)
    assert a == rho * b


@pytest.mark.parametrize("n", [1000, 4097])
def test_matgen_bit_exact(mxp, orc, torch_cuda, n):
    a, b = mxp.higham_params(n, 1e3, 0.5)
    p = mxp.higham_matgen(n, a, b, seed=42)
    A, d = orc.higham_matgen(n, a, b)
    got = to_np_colmajor(p.A, n, n, n)
    assert np.array_equal(got.view(np.uint32), A.view(np.uint32))
    assert np.array_equal(p.d.cpu().numpy(), d)
    _, _, _, rhs = orc.matgen(n, 42, with_matrix=False)
    assert np.array_equal(p.rhs.cpu().numpy(), rhs)


def test_matgen_beyond_one_launch(mxp, orc, torch_cuda):
    """n > 65535 columns: the fill runs in two launches; the last columns
    against the oracle's column fill."""
    torch = torch_cuda
    n = 65600
    a, b = mxp.higham_params(n, 1e3, 0.5)
    A = torch.empty(n * n, dtype=torch.float32, device="cuda")
    mxp.check(mxp.lib().mxp_matgen_higham(n, a, b, 1, A.data_ptr(), n, None, None,
                                          torch.cuda.current_stream().cuda_stream))
    j0, nc = 65500, 100
    got = A[j0 * n:(j0 + nc) * n].view(nc, n).cpu().numpy().T
    want = np.empty((n, nc), np.float32, order="F")
    orc.lib().orc_higham_matgen_cols(n, a, b, j0, nc, want.ctypes.data, n)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    del A


@pytest.mark.parametrize("n,rho,alpha,beta_y", [(1000, 0.5, -1.0, 1.0), (3000, 1.0, 0.5, 0.0),
                                                (4096, 0.125, 1.0, -2.0)])
def test_gemv_bit_exact(mxp, orc, torch_cuda, n, rho, alpha, beta_y):
    torch = torch_cuda
    a, b = mxp.higham_params(n, 1e3, rho)
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y.copy()).cuda()
    mxp.higham_gemv(n, a, b, alpha, dx, beta_y, dy)
    want = orc.higham_gemv(n, a, b, alpha, x, beta_y, y.copy())
    assert np.array_equal(dy.cpu().numpy(), want)


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,cond", [(2048, 256, 1e3), (4096, 512, 1e4)])
def test_solve_higham(mxp, orc, torch_cuda, form, n, b, cond):
    a, be = mxp.higham_params(n, cond, 0.5)
    p = mxp.higham_matgen(n, a, be, seed=7)
    ws = mxp.Workspace(n, b, form)
    ws.set_matrix_higham(a, be)
    x, lst, ist = mxp.solve(p, b, ws)
    assert ist["converged"] == 1 and ist["hpl_harness"] < 16.0
    assert ist["norma"] == mxp.higham_infnorm(n, a, be)
    assert ist["norma"] == pytest.approx(orc.lib().orc_higham_infnorm(n, a, be), rel=1e-13)
    LU = to_np_colmajor(p.A, n, n, n).astype(np.float64)
    low, up = np.tril(np.ones((n, n), bool), -1), np.triu(np.ones((n, n), bool), 1)
    # panel_check: the factors of A = L U are alpha / beta / 1
    tol = 2e-1 if form == 2 else 1e-2
    assert np.max(np.abs(LU[low] - a)) / a <= tol
    assert np.max(np.abs(LU[up] - be)) / be <= tol
    assert np.max(np.abs(np.diag(LU) - 1.0)) <= tol
    A64 = orc.higham_matrix_f64(n, a, be)
    _, _, _, rhs = orc.matgen(n, 7, with_matrix=False)
    xt = np.linalg.solve(A64, rhs)
    xs = x.cpu().numpy()
    assert np.max(np.abs(xs - xt)) / np.max(np.abs(xt)) < 1e-10
    # back to the LCG matrix on the same workspace
    ws.set_matrix_higham(0.0, 0.0)
    q = mxp.panel_matgen(n, 5)
    _, _, ist2 = mxp.solve(q, b, ws)
    assert ist2["converged"] == 1


def test_bad_higham_arguments(mxp, torch_cuda):
    with pytest.raises(mxp.MxpError):
        mxp.higham_params(1, 1e3, 0.5)
    ws = mxp.Workspace(256, 64, 0)
    with pytest.raises(mxp.MxpError):
        ws.set_matrix_higham(-1.0, 1.0)
