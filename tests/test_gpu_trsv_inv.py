"""Refinement solves with the inverses of the diagonal blocks that the LU
keeps (MXP_OPT_TRSV_INV): the same result as exact block substitution on the
GPU's own factors (to ~1e-14 with near-FP32 inverses), deterministic, and the
same refinement outcome as the chain-of-64-row-blocks solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _factor(mxp, n, b, form, seed=42, **kw):
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form, **kw)
    mxp.panel_lu(p, b, ws)
    return p, ws


# (n, b, form, trsm_single, tolerance relative to max |x|).  Each diagonal
# block is solved as t1 = X v, t = t1 + X (v - T t1) with the stored inverse X,
# so the error is of the order of the square of X's relative error: near-FP32
# inverses (split-BF16 products for the doubling levels >= 1024 at b = 2560)
# leave ~1e-14; one BF16 product for those levels (trsm_single) ~2^-9 per
# entry before the refinement step.
CASES = [(1024, 128, 0, False, 1e-12), (2048, 256, 2, False, 1e-12), (4096, 512, 0, False, 1e-12),
         (2048, 256, 1, False, 1e-12), (5120, 2560, 0, False, 1e-12), (5120, 2560, 2, True, 1e-8)]


@pytest.mark.parametrize("n,b,form,single,tol", CASES)
def test_lu_solve_with_stored_inverses(mxp, orc, torch_cuda, n, b, form, single, tol):
    torch = torch_cuda
    p, ws = _factor(mxp, n, b, form, trsm_single=single)
    LU = np.asfortranarray(p.A.view(n, n).cpu().numpy().T)
    rng = np.random.default_rng(n + form)
    x = rng.standard_normal(n)
    want = orc.lu_solve(LU.copy(order="F"), x.copy())
    dx = torch.from_numpy(x.copy()).cuda()
    mxp.lu_solve(p.A, n, n, dx, ws)                 # stored inverses (the factor of the last LU)
    got_inv = dx.cpu().numpy()
    dx = torch.from_numpy(x.copy()).cuda()
    mxp.lu_solve(p.A, n, n, dx, ws)                 # deterministic: the same bits again
    assert np.array_equal(dx.cpu().numpy(), got_inv)
    ws.set_option(mxp.OPT_TRSV_INV, 0)               # the chain of 64-row blocks
    dx = torch.from_numpy(x.copy()).cuda()
    mxp.lu_solve(p.A, n, n, dx, ws)
    got_chain = dx.cpu().numpy()
    scale = np.max(np.abs(want))
    assert np.max(np.abs(got_chain - want)) <= 1e-12 * scale
    err = np.max(np.abs(got_inv - want)) / scale
    assert err <= tol, err
    ws.close()


def test_stored_inverses_belong_to_the_last_lu(mxp, orc, torch_cuda):
    """A factor in another buffer is solved by the chain kernel (exact)."""
    torch = torch_cuda
    n, b = 1024, 128
    p, ws = _factor(mxp, n, b, 0)
    q = mxp.panel_matgen(n, 7)
    ws2 = mxp.Workspace(n, b, 0, trsm_tensor=False)   # no inverses kept: plain LU
    mxp.panel_lu(q, b, ws2)
    LU = np.asfortranarray(q.A.view(n, n).cpu().numpy().T)
    x = np.random.default_rng(5).standard_normal(n)
    dx = torch.from_numpy(x.copy()).cuda()
    mxp.lu_solve(q.A, n, n, dx, ws)                  # ws holds the inverses of p's factor
    want = orc.lu_solve(LU.copy(order="F"), x.copy())
    assert np.max(np.abs(dx.cpu().numpy() - want)) <= 1e-12 * np.max(np.abs(want))
    ws.close()
    ws2.close()


@pytest.mark.parametrize("form,single", [(0, False), (2, True)])
def test_refinement_same_outcome_both_solves(mxp, orc, torch_cuda, form, single):
    n, b = 5120, 2560
    res = {}
    for inv in (1, 0):
        p = mxp.panel_matgen(n, 7)
        ws = mxp.Workspace(n, b, form, trsm_single=single)
        ws.set_option(mxp.OPT_TRSV_INV, inv)
        x, lst, ist = mxp.solve(p, b, ws)
        assert ist["converged"] == 1 and ist["hpl_harness"] < 16.0
        res[inv] = (ist["iterations"], x.cpu().numpy())
        ws.close()
    assert abs(res[1][0] - res[0][0]) <= 1
    _, d, _, rhs = orc.matgen(n, 7, with_matrix=False)
    xt = np.linalg.solve(orc.matgen_f64(n, 7, d), rhs)
    for inv in (1, 0):
        assert np.max(np.abs(res[inv][1] - xt)) / np.max(np.abs(xt)) < 1e-10
