"""Whole blocked LU (mxp_panel_lu) vs the oracle's restatement of
panel_lu_async_wGPU with the same precision form.  Factor bar for the FP16
forms: relative Frobenius distance of the factors <= 1e-3."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("trsm_tensor,merge,coop", [(True, True, True), (True, False, True),
                                                   (False, True, True), (True, True, False)])
@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed,rule", [(512, 64, 42, 0), (1024, 128, 7, 0), (2048, 256, 11, 1),
                                           (1536, 512, 42, 0), (1280, 256, 3, 0)])
def test_panel_lu_factors(mxp, orc, torch_cuda, form, n, b, seed, rule, trsm_tensor, merge, coop):
    torch = torch_cuda
    p = mxp.panel_matgen(n, seed, rule)
    ws = mxp.Workspace(n, b, form, trsm_tensor=trsm_tensor, merge_panels=merge, diag_coop=coop)
    st = mxp.panel_lu(p, b, ws)
    got = to_np_colmajor(p.A, n, n, n)
    A, _, _, _ = orc.matgen(n, seed, rule)
    assert orc.panel_lu(A, b, form) == 0
    err = rel_fro(got, A)
    assert err <= 1e-3
    # off-diagonal factor entries are tiny next to the diagonal; check them alone too
    low = np.tril(np.ones((n, n), bool), -1)
    assert rel_fro(got[low], A[low]) <= 1e-3
    up = np.triu(np.ones((n, n), bool), 1)
    assert rel_fro(got[up], A[up]) <= 1e-3
    nb = n // b
    if not merge or (form == 2 and b % 128):
        assert st["schur_launches"] == nb - 1
    else:  # pairs: col block + row block + merged trailing; an odd tail pass
        assert st["schur_launches"] >= nb - 1


def test_panel_lu_rejects_bad_block(mxp, torch_cuda):
    p = mxp.panel_matgen(256, 1)
    ws = mxp.Workspace(256, 64, 0)
    with pytest.raises(mxp.MxpError) as e:
        mxp.panel_lu(p, 96, ws)
    assert e.value.status == mxp.INVALID_ARG
