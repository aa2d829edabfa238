"""mxp_matgen vs the oracle (itself pinned to the reference generator): bit-exact."""
import json
import os

import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,seed,rule,pad", [(256, 42, 0, 0), (1000, 7, 0, 3), (2048, 11, 1, 0),
                                             (777, 3, 0, 0), (64, 1000, 1, 17)])
def test_matgen_bitexact(mxp, orc, torch_cuda, n, seed, rule, pad):
    torch = torch_cuda
    p = mxp.panel_matgen(n, seed, rule, lda=n + pad)
    torch.cuda.synchronize()
    A = to_np_colmajor(p.A, n, n, n + pad)
    Ao, do, rso, bo = orc.matgen(n, seed, rule)
    assert np.array_equal(A.view(np.uint32), Ao.view(np.uint32))
    assert np.array_equal(p.d.cpu().numpy().view(np.uint64), do.view(np.uint64))
    assert np.array_equal(p.rowsum.cpu().numpy().view(np.uint64), rso.view(np.uint64))
    assert np.array_equal(p.rhs.cpu().numpy().view(np.uint64), bo.view(np.uint64))


def test_matgen_large_samples(mxp, orc, torch_cuda):
    """Sampled elements at N = 61440 (the plain-form configuration) against the
    values the reference generator produced (tests/golden/golden.json)."""
    torch = torch_cuda
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
    s = [g for g in gold["samples"] if g["n"] == 61440][0]
    n, seed = s["n"], s["seed"]
    p = mxp.panel_matgen(n, seed)
    torch.cuda.synchronize()
    M = p.A.view(n, n)  # M[j, i] = a_ij
    for (i, j), hx in zip(s["ij"], s["f64_hex"]):
        if i == j:
            continue
        assert M[j, i].item() == np.float32(float.fromhex(hx))
    rhs = p.rhs.cpu().numpy()
    for r, hx in zip(s["rhs_rows"], s["rhs_f64_hex"]):
        assert rhs[r] == float.fromhex(hx)
    d = p.d.cpu().numpy()
    for i in (0, 1, n // 2, n - 1):
        dv = orc.lib().orc_rowsum_row(n, seed, i)
        assert d[i] == dv
        assert M[i, i].item() == np.float32(dv)
    del p, M
    torch.cuda.empty_cache()


def test_matgen_rejects_bad_args(mxp):
    import ctypes as C
    assert mxp.lib().mxp_matgen(0, 1, 0, None, 1, None, None, None, None) == mxp.INVALID_ARG
    assert mxp.lib().mxp_matgen(16, 1, 7, None, 16, None, None, None, None) == mxp.INVALID_ARG
