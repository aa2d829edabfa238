"""FP8 form: the TRSM-by-inverse products that form each L and U panel also
write their E4M3 copies and per-tile scales (MXP_OPT_FP8_FUSED_CAST).  Those
bytes must be the ones the FP8 panel casts make from the stored FP32 panels,
so the whole factorisation is bit-identical with the option on and off."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("n,b,seed", [(2048, 256, 7), (2560, 512, 11), (3584, 256, 5), (5120, 2560, 7)])
def test_fused_l_panel_cast_is_bit_identical(mxp, torch_cuda, single, n, b, seed):
    out = {}
    for fused in (1, 0):
        p = mxp.panel_matgen(n, seed)
        ws = mxp.Workspace(n, b, mxp.FORM_FP8, trsm_single=single)
        ws.set_option(mxp.OPT_FP8_FUSED_CAST, fused)
        mxp.panel_lu(p, b, ws)
        torch.cuda.synchronize()
        out[fused] = p.A.clone()
        ws.close()
    assert torch.equal(out[1].view(torch.int32), out[0].view(torch.int32))


def test_fused_solve_converges(mxp, torch_cuda):
    n, b = 3072, 256
    p = mxp.panel_matgen(n, 13)
    ws = mxp.Workspace(n, b, mxp.FORM_FP8, trsm_single=True)
    _, lu, ir = mxp.solve(p, b, ws)
    assert ir["converged"] == 1 and ir["hpl_harness"] < 16.0
