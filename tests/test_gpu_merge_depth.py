"""Merged schedule with D panels per trailing pass (MXP_OPT_MERGE_DEPTH = D, 3
or 4): each panel of a group updates the column and row blocks of the group's
later panels, then one pass with K = D b applies the group.  The factors must match
the oracle's restatement of the reference's one-panel-per-step LU to the same
bar as the default schedule."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [3, 4])
@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed", [(1024, 128, 7), (2048, 256, 11), (1792, 256, 3), (1280, 256, 5),
                                      (2560, 512, 42)])
def test_depth_factors(mxp, orc, torch_cuda, depth, form, n, b, seed):
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form, merge_depth=depth)
    st = mxp.panel_lu(p, b, ws)
    got = to_np_colmajor(p.A, n, n, n)
    A, _, _, _ = orc.matgen(n, seed, 0)
    assert orc.panel_lu(A, b, form) == 0
    assert rel_fro(got, A) <= 1e-3
    low = np.tril(np.ones((n, n), bool), -1)
    assert rel_fro(got[low], A[low]) <= 1e-3
    # groups of D: 2 (D - 1) updates inside and one trailing pass; a last
    # full group has no trailing matrix and no row blocks (D - 1 launches); a
    # tail of t < D panels updates t - 1 column blocks
    q, t = divmod(n // b, depth)
    want = (2 * depth - 1) * q + (-depth if t == 0 else t - 1)
    assert st["schur_launches"] == want


@pytest.mark.parametrize("depth", [1, 2, 3, 4])
def test_depth_solve_converges(mxp, torch_cuda, depth):
    n, b = 3072, 256
    p = mxp.panel_matgen(n, 13)
    ws = mxp.Workspace(n, b, 2, merge_depth=depth, trsm_single=True)
    _, lu, ir = mxp.solve(p, b, ws)
    assert ir["converged"] and ir["hpl_harness"] < 16.0


def test_depth_option_bounds(mxp, torch_cuda):
    ws = mxp.Workspace(512, 128, 0)
    for bad in (0, 5):
        with pytest.raises(mxp.MxpError):
            ws.set_option(mxp.OPT_MERGE_DEPTH, bad)
