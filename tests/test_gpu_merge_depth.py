"""Merged schedule with three panels per trailing pass (MXP_OPT_MERGE_DEPTH = 3):
each panel of a group updates the column and row blocks of the group's later
panels, then one pass with K = 3b applies the group.  The factors must match
the oracle's restatement of the reference's one-panel-per-step LU to the same
bar as the default schedule."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed", [(1024, 128, 7), (2048, 256, 11), (1792, 256, 3), (1280, 256, 5),
                                      (2560, 512, 42)])
def test_depth3_factors(mxp, orc, torch_cuda, form, n, b, seed):
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form, merge_depth=3)
    st = mxp.panel_lu(p, b, ws)
    got = to_np_colmajor(p.A, n, n, n)
    A, _, _, _ = orc.matgen(n, seed, 0)
    assert orc.panel_lu(A, b, form) == 0
    assert rel_fro(got, A) <= 1e-3
    low = np.tril(np.ones((n, n), bool), -1)
    assert rel_fro(got[low], A[low]) <= 1e-3
    # groups of three: 2 + 2 updates inside and one trailing pass (5 launches);
    # a last full group has no trailing matrix and no row blocks (2); a tail
    # of two panels updates one column block (1); a tail of one, nothing
    q, t = divmod(n // b, 3)
    want = 5 * q + {0: -3, 1: 0, 2: 1}[t]
    assert st["schur_launches"] == want


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_depth_solve_converges(mxp, torch_cuda, depth):
    n, b = 3072, 256
    p = mxp.panel_matgen(n, 13)
    ws = mxp.Workspace(n, b, 2, merge_depth=depth, trsm_single=True)
    _, lu, ir = mxp.solve(p, b, ws)
    assert ir["converged"] and ir["hpl_harness"] < 16.0


def test_depth_option_bounds(mxp, torch_cuda):
    ws = mxp.Workspace(512, 128, 0)
    for bad in (0, 4):
        with pytest.raises(mxp.MxpError):
            ws.set_option(mxp.OPT_MERGE_DEPTH, bad)
