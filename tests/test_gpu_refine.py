"""FP64 refinement pieces and the whole solve vs the oracle / an FP64 LU."""
import numpy as np
import pytest

from tests.gpu_util import from_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,seed,alpha,beta", [(1000, 42, -1.0, 1.0), (2048, 7, 0.5, 0.0),
                                               (4096, 11, -1.0, 2.0), (300, 3, 1.0, -1.0)])
def test_otf_gemv(mxp, orc, torch_cuda, n, seed, alpha, beta):
    torch = torch_cuda
    _, d, _, _ = orc.matgen(n, seed, with_matrix=False)
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    ws = mxp.Workspace(n, min(n, 64), 0)
    dd = torch.from_numpy(d).cuda()
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y.copy()).cuda()
    mxp.otf_gemv(n, seed, dd, alpha, dx, beta, dy, ws)
    got = dy.cpu().numpy()
    want = orc.otf_gemv(n, seed, d, alpha, x, beta, y.copy())
    scale = np.abs(alpha) * (np.abs(orc.matgen_f64(n, seed, d)) @ np.abs(x)) + np.abs(beta * y)
    assert np.all(np.abs(got - want) <= 1e-14 * scale + 1e-300)


@pytest.mark.parametrize("n", [64, 1000, 4096, 5000])
def test_lu_solve(mxp, orc, torch_cuda, n):
    torch = torch_cuda
    A, _, _, _ = orc.matgen(n, 5)
    assert orc.lib().orc_getrf_nopiv(n, n, A.ctypes.data, n) == 0
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    dLU = from_np_colmajor(torch, A)
    dx = torch.from_numpy(x.copy()).cuda()
    ws = mxp.Workspace(n, min(n, 64), 0)
    mxp.lu_solve(dLU, n, n, dx, ws)
    got = dx.cpu().numpy()
    want = orc.lu_solve(A, x.copy())
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed,rule", [(1024, 128, 42, 0), (2048, 256, 7, 0), (2048, 256, 11, 1),
                                           (4096, 512, 7, 0)])
def test_solve_converges_and_forward_error(mxp, orc, torch_cuda, form, n, b, seed, rule):
    p = mxp.panel_matgen(n, seed, rule)
    ws = mxp.Workspace(n, b, form)
    x, lst, ist = mxp.solve(p, b, ws)
    assert ist["converged"] == 1 and ist["hpl_harness"] < 16.0
    xs = x.cpu().numpy()
    # FP64 oracle: LU of the FP64 matrix the residual uses
    _, d, rs, rhs = orc.matgen(n, seed, rule, with_matrix=False)
    A64 = orc.matgen_f64(n, seed, d)
    xt = np.linalg.solve(A64, rhs)
    fwd = np.max(np.abs(xs - xt)) / np.max(np.abs(xt))
    assert fwd < 1e-10
    # same iteration count as the oracle's classic IR on its own factors (+-1)
    A, _, _, _ = orc.matgen(n, seed, rule)
    orc.panel_lu(A, b, form)
    it, *_ = orc.ir_classic(n, b, seed, A, d, rs if rule else None, rhs)
    assert abs(ist["iterations"] - it) <= (1 if form != 2 else 2)


def test_ir_not_converged_status(mxp, torch_cuda):
    p = mxp.panel_matgen(1024, 42)
    ws = mxp.Workspace(1024, 128, 0)
    mxp.panel_lu(p, 128, ws)
    x, st, s = mxp.iterative_refinement(p, ws, maxit=1, raise_on_fail=False)
    assert s == mxp.NOT_CONVERGED and st["converged"] == 0


def test_solve_host_matches_device(mxp, torch_cuda):
    torch = torch_cuda
    n, b = 2048, 256
    p1 = mxp.panel_matgen(n, 42)
    ws = mxp.Workspace(n, b, 0)
    x1, _, _ = mxp.solve(p1, b, ws)
    p2 = mxp.panel_matgen(n, 42)
    h_rhs = p2.rhs.cpu().pin_memory()
    h_x = torch.empty(n, dtype=torch.float64).pin_memory()
    mxp.solve_host(p2, b, ws, h_rhs, h_x)
    assert torch.equal(h_x, x1.cpu())


@pytest.mark.parametrize("form", [0, 2])
@pytest.mark.parametrize("n,b,seed,rule", [(2048, 256, 42, 0), (2048, 256, 11, 1)])
def test_gmres_ir(mxp, orc, torch_cuda, form, n, b, seed, rule):
    """GMRES-IR (LU-preconditioned FP64 GMRES for the correction) reaches the
    threshold and the same forward error as the FP64 oracle solve."""
    p = mxp.panel_matgen(n, seed, rule)
    ws = mxp.Workspace(n, b, form)
    x, lst, ist = mxp.solve(p, b, ws, method=mxp.IR_GMRES)
    assert ist["converged"] == 1 and ist["hpl_harness"] < 16.0
    assert ist["inner_iterations"] >= 1
    _, d, rs, rhs = orc.matgen(n, seed, rule, with_matrix=False)
    xt = np.linalg.solve(orc.matgen_f64(n, seed, d), rhs)
    assert np.max(np.abs(x.cpu().numpy() - xt)) / np.max(np.abs(xt)) < 1e-10


def test_gmres_options(mxp, torch_cuda):
    ws = mxp.Workspace(1024, 128, 0)
    ws.set_option(mxp.OPT_GMRES_RESTART, 2)
    ws.set_option(mxp.OPT_GMRES_TOL_EXP, 4)
    p = mxp.panel_matgen(1024, 42)
    x, lst, ist = mxp.solve(p, 128, ws, method=mxp.IR_GMRES)
    assert ist["converged"] == 1
    with pytest.raises(mxp.MxpError):
        ws.set_option(mxp.OPT_GMRES_RESTART, 99)
