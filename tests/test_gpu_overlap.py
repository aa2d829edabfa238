"""Diagonal factorisation of the next panel pair run beside the trailing pass
(MXP_OPT_OVERLAP_DIAG): the trailing pass is split into the next diagonal
block's corner, then two launches that claim the remaining tiles from one
counter (the second on the SMs the factorisation used).  Every tile is the
same arithmetic whichever CTA or launch computes it, and the cooperative
factorisation's result does not depend on its grid size, so the factors
must be bit-identical to the sequential schedule's."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor, rel_fro

pytestmark = pytest.mark.gpu


def _lu(mxp, n, b, seed, rule, form, **opts):
    p = mxp.panel_matgen(n, seed, rule)
    ws = mxp.Workspace(n, b, form, **opts)
    st = mxp.panel_lu(p, b, ws)
    return to_np_colmajor(p.A, n, n, n), st


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed,rule,sms", [(3072, 256, 42, 0, 16), (4096, 256, 7, 1, 8),
                                               (5120, 512, 11, 0, 32), (2816, 256, 3, 0, 74)])
def test_overlap_bit_identical(mxp, torch_cuda, form, n, b, seed, rule, sms):
    ref, st0 = _lu(mxp, n, b, seed, rule, form, merge_depth=2)
    got, st1 = _lu(mxp, n, b, seed, rule, form, merge_depth=2, overlap_diag=sms, overlap_min=2)
    assert st0["overlapped_diag"] == 0
    # pairs (k, k+1) whose trailing matrix has >= 2 blocks beyond the pair
    nb = n // b
    expect = sum(1 for k in range(0, nb, 2) if nb - k - 2 >= 2)
    assert st1["overlapped_diag"] == expect
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("form", [0, 2])
def test_overlap_depth3_bit_identical(mxp, torch_cuda, form):
    n, b = 4096, 256
    ref, _ = _lu(mxp, n, b, 17, 0, form, merge_depth=3)
    got, st = _lu(mxp, n, b, 17, 0, form, merge_depth=3, overlap_diag=24, overlap_min=2)
    # groups (0,1,2), (3,4,5), ... with >= 2 blocks of trailing matrix after them
    nb = n // b
    assert st["overlapped_diag"] == sum(1 for k in range(0, nb, 3) if nb - k - 3 >= 2)
    assert np.array_equal(got, ref)


def test_overlap_matches_oracle(mxp, orc, torch_cuda):
    n, b, seed = 2048, 256, 5
    got, st = _lu(mxp, n, b, seed, 0, 0, overlap_diag=20, overlap_min=2)
    assert st["overlapped_diag"] > 0
    A, _, _, _ = orc.matgen(n, seed, 0)
    assert orc.panel_lu(A, b, 0) == 0
    assert rel_fro(got, A) <= 1e-3


def test_overlap_solve_converges(mxp, torch_cuda):
    n, b = 4096, 256
    p = mxp.panel_matgen(n, 9)
    ws = mxp.Workspace(n, b, 2, overlap_diag=16, overlap_min=2)
    _, lu, ir = mxp.solve(p, b, ws)
    assert ir["converged"]
    assert lu["overlapped_diag"] > 0


def test_overlap_off_when_blocks_unaligned(mxp, torch_cuda):
    # the skipped corner must be whole 128 x 256 tiles: b = 128 falls back
    got, st = _lu(mxp, 1536, 128, 4, 0, 0, overlap_diag=16, overlap_min=2)
    ref, _ = _lu(mxp, 1536, 128, 4, 0, 0)
    assert st["overlapped_diag"] == 0
    assert np.array_equal(got, ref)


def test_overlap_option_bounds(mxp, torch_cuda):
    ws = mxp.Workspace(1024, 256, 0)
    with pytest.raises(mxp.MxpError):
        ws.set_option(mxp.OPT_OVERLAP_DIAG, -1)
    with pytest.raises(mxp.MxpError):
        ws.set_option(mxp.OPT_OVERLAP_DIAG, 1000)
    with pytest.raises(mxp.MxpError):
        ws.set_option(mxp.OPT_OVERLAP_MIN, 1)
    ws.set_option(mxp.OPT_OVERLAP_DIAG, 0)
