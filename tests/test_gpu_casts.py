"""Panel casts vs the oracle: bit-exact for every form and both layouts."""
import numpy as np
import pytest

from tests.gpu_util import from_np_colmajor

pytestmark = pytest.mark.gpu


def _panel(rng, m, b, scale=1e-4):
    P = (rng.standard_normal((m, b)) * scale).astype(np.float32)
    P[0, 0] = 3e-8      # FP16 subnormal range
    P[-1, -1] = 7e-6
    return P


@pytest.mark.parametrize("m,b", [(64, 64), (200, 96), (1000, 256)])
def test_reference_layout_casts(mxp, orc, torch_cuda, m, b):
    torch = torch_cuda
    rng = np.random.default_rng(m + b)
    Lp = _panel(rng, m, b)
    dL = from_np_colmajor(torch, Lp, ld=m + 5)
    out = torch.zeros(m * b + 8, dtype=torch.int16, device="cuda")
    mxp.half_conversion_left(dL, m, b, m + 5, out, m)
    torch.cuda.synchronize()
    got = out[: m * b].cpu().numpy().view(np.uint16).reshape(b, m).T
    assert np.array_equal(got, orc.f2h_array(Lp))
    # right: U block b x m -> rp[k * rplda + j] = U(k, j)
    U = _panel(rng, b, m)
    dU = from_np_colmajor(torch, U, ld=b + 3)
    outr = torch.zeros(b * m + 8, dtype=torch.int16, device="cuda")
    mxp.half_conversion_right_trans(dU, b, m, b + 3, outr, m)
    torch.cuda.synchronize()
    gotr = outr[: b * m].cpu().numpy().view(np.uint16).reshape(b, m)  # [k, j]
    assert np.array_equal(gotr, orc.f2h_array(U))


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("m,b", [(128, 128), (300, 256), (1, 64), (515, 384)])
def test_kmajor_casts(mxp, orc, torch_cuda, form, m, b):
    torch = torch_cuda
    rng = np.random.default_rng(7 * m + b + form)
    L = _panel(rng, m, b, 1e-3)
    L[: min(m, 128), : min(b, 128)] *= 1e-3  # a tile with a different scale
    U = _panel(rng, b, m, 0.5)
    Kx = 3 * b if form == 1 else b
    es = 1 if form == 2 else 2
    ldk = -(-Kx // (16 // es)) * (16 // es)
    dt = torch.uint8 if es == 1 else torch.int16
    sc_n = (-(-m // 128)) * (-(-b // 128))
    for right, P, src_ld in ((False, L, m + 2), (True, U, b + 6)):
        dP = from_np_colmajor(torch, P, ld=src_ld)
        out = torch.zeros(m * ldk + 16, dtype=dt, device="cuda")
        sc = torch.zeros(sc_n + 16, dtype=torch.uint8, device="cuda")
        fn = mxp.panel_cast_right if right else mxp.panel_cast_left
        fn(form, m, b, dP, src_ld, out, ldk, sc if form == 2 else None)
        torch.cuda.synchronize()
        raw = out[: m * ldk].cpu().numpy()
        raw = raw.view(np.uint8 if es == 1 else np.uint16).reshape(m, ldk)[:, :Kx]
        want, wsc = orc.kmajor_panel(form, U.T if right else L, right)
        assert np.array_equal(raw, want), f"form {form} right={right}"
        if form == 2:
            assert np.array_equal(sc[:sc_n].cpu().numpy().reshape(wsc.shape), wsc)
