"""The FP64 system generator (mxp_matgen_f64) and the FP64 forward-error
reference (openmxp_b200.forward_error) against the oracle and numpy."""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,seed,rule,pad", [(256, 42, 0, 0), (777, 7, 1, 5)])
def test_matgen_f64_bitexact(mxp, orc, torch_cuda, n, seed, rule, pad):
    torch = torch_cuda
    A = mxp.matgen_f64(n, seed, rule, lda=n + pad)
    torch.cuda.synchronize()
    A64 = to_np_colmajor(A, n, n, n + pad)
    _, d, _, _ = orc.matgen(n, seed, rule)
    Ao = orc.matgen_f64(n, seed, d)
    assert np.array_equal(A64.view(np.uint64), Ao.view(np.uint64))


@pytest.mark.parametrize("n,block,rule", [(1024, 256, 0), (1000, 384, 1)])
def test_reference_solution_matches_numpy(mxp, orc, torch_cuda, n, block, rule):
    from openmxp_b200 import forward_error as fe
    torch = torch_cuda
    seed = 5
    p = mxp.panel_matgen(n, seed, rule)
    x = fe.reference_solution(n, seed, rule, p.rhs, block=block)
    torch.cuda.synchronize()
    _, d, _, b = orc.matgen(n, seed, rule)
    Ao = orc.matgen_f64(n, seed, d)
    xn = np.linalg.solve(Ao, b)
    assert np.max(np.abs(x.cpu().numpy() - xn)) / np.max(np.abs(xn)) < 1e-13


def test_solve_forward_error_fp16_fp8(mxp, torch_cuda):
    """Forward error of the FP16 and FP8 forms against the FP64 reference."""
    from openmxp_b200 import forward_error as fe
    n, b, seed = 4096, 512, 9
    p = mxp.panel_matgen(n, seed)
    x_ref = fe.reference_solution(n, seed, 0, p.rhs, block=1024)
    for form in (mxp.FORM_FP16, mxp.FORM_FP8):
        mxp.regenerate(p)
        ws = mxp.Workspace(n, b, form)
        x, _, ist = mxp.solve(p, b, ws)
        assert ist["converged"] == 1 and ist["hpl_harness"] < 16
        assert fe.forward_error(x, x_ref) < 1e-10
        ws.close()
