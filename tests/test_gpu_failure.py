"""Failure detection without a GPU fault: a bounded device wait is made to run
out (a completion flag that nothing sets) and the call must come back with
MXP_TIMEOUT after about the 2 s bound, leaving the context usable."""
import time

import numpy as np
import pytest

from tests.gpu_util import from_np_colmajor

pytestmark = pytest.mark.gpu


def test_trsv_wait_times_out_then_recovers(mxp, orc, torch_cuda):
    torch = torch_cuda
    n = 512
    A, _, _, _ = orc.matgen(n, 5)
    assert orc.lib().orc_getrf_nopiv(n, n, A.ctypes.data, n) == 0
    dLU = from_np_colmajor(torch, A)
    x = np.random.default_rng(3).standard_normal(n)
    ws = mxp.Workspace(n, 64, 0)

    ws.set_option(mxp.OPT_TEST_WITHHOLD_FLAG, 3)  # row block 3 never publishes
    dx = torch.from_numpy(x.copy()).cuda()
    t0 = time.perf_counter()
    with pytest.raises(mxp.MxpError) as e:
        mxp.lu_solve(dLU, n, n, dx, ws)
    dt = time.perf_counter() - t0
    assert e.value.status == mxp.TIMEOUT
    assert 1.5 < dt < 60.0

    # the option applies to one call; the same workspace and context solve correctly
    dx = torch.from_numpy(x.copy()).cuda()
    mxp.lu_solve(dLU, n, n, dx, ws)
    want = orc.lu_solve(A, x.copy())
    got = dx.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    ws.close()
