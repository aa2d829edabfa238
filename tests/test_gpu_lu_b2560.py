"""mxp_panel_lu at the benched block size (B = 2560) against the oracle's
restatement of the same algorithm (oracle/blocked.py): FP32 diagonal LU,
TRSM by inverse with the triangular-inverse levels from 1024 on the tensor
cores, panel casts, Schur update.  The three arms are configured exactly as
bench.py runs them:

- plain FP16 form: split-BF16 TRSM products (near FP32), groups of 4 panels;
- FP8 form: single BF16 TRSM product, E4M3 panels written by the TRSM
  products' epilogues (MXP_OPT_FP8_FUSED_CAST on);
- BF16X2 form: split-BF16 TRSM products.

N = 10240 is one full group of four panels; N = 12800 is a group plus a
one-panel tail.  Bars: relative Frobenius distance <= 1e-3 (the factor bar
the FP16 forms are held to) overall and on the strict lower and upper parts, and
element-wise: every entry of a strict part within 1e-3 of that part's
largest entry for the split-BF16 TRSM, within 2 * 2^-8 of it for the single
BF16 product (the GPU and the oracle reach each operand through different
Schur summation orders, so the same entry may round to neighbouring BF16
values: one BF16 ulp, 2^-8 relative, in each of the two operands).  The
low-precision panel copies the Schur update reads are checked byte for byte
against the oracle's casts of the factors' FP32 panels."""
import numpy as np
import pytest

from oracle import blocked as Bk
from tests.gpu_util import panel_slot, rel_fro, to_np_colmajor

pytestmark = pytest.mark.gpu

B = 2560
ELEM_TOL = {"split": 1e-3, "single": 2.0 * 2.0 ** -8}
ARMS = {  # name: (form, workspace trsm_single, oracle trsm)
    "fp16_split": (0, False, "split"),
    "fp8_single_fused": (2, True, "single"),
    "bf16x2_split": (1, False, "split"),
}


def _factor(mxp, n, seed, arm, opts=None):
    form, single, _ = ARMS[arm]
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, B, form, trsm_single=single)
    for k, v in (opts or {}).items():
        ws.set_option(k, v)
    st = mxp.panel_lu(p, B, ws)
    return p, ws, st


def _parts(n):
    return np.tril(np.ones((n, n), bool), -1), np.triu(np.ones((n, n), bool), 1)


@pytest.mark.parametrize("arm", list(ARMS))
@pytest.mark.parametrize("n,seed", [(10240, 7), (12800, 42)])
def test_factors_b2560(mxp, orc, torch_cuda, arm, n, seed):
    form, _, trsm = ARMS[arm]
    p, ws, st = _factor(mxp, n, seed, arm)
    got = to_np_colmajor(p.A, n, n, n)
    ws.close()
    del p
    A, _, _, _ = orc.matgen(n, seed)
    assert Bk.panel_lu(A, B, form, trsm=trsm, inv_tc=1024) == 0
    low, up = _parts(n)
    assert rel_fro(got, A) <= 1e-3
    for part in (low, up):
        g, w = got[part].astype(np.float64), A[part].astype(np.float64)
        assert rel_fro(g, w) <= 1e-3
        assert np.max(np.abs(g - w)) <= ELEM_TOL[trsm] * np.max(np.abs(w))
    # the diagonal (the U pivots) too, entry by entry
    dg, dw = np.diag(got).astype(np.float64), np.diag(A).astype(np.float64)
    assert np.max(np.abs(dg - dw) / np.abs(dw)) <= 1e-5


@pytest.mark.parametrize("arm", list(ARMS))
@pytest.mark.parametrize("n", [10240, 12800])
def test_panel_copies_b2560(mxp, orc, torch_cuda, arm, n):
    """The low-precision L and R panels left in the workspace's slots are the
    oracle's casts of the factor's own FP32 panels, byte for byte (for FP8:
    the E4M3 bytes and UE8M0 scales the TRSM epilogues wrote)."""
    torch = torch_cuda
    form, _, _ = ARMS[arm]
    p, ws, _ = _factor(mxp, n, 11, arm)
    got = to_np_colmajor(p.A, n, n, n)
    lv, rv = ws.panel_view(0), ws.panel_view(1)
    nb = n // B
    slots = min(nb - 1, 4)  # slot s holds panel s of the first group (the tail writes none)
    for s in range(slots):
        m = n - (s + 1) * B
        Lp = got[(s + 1) * B:, s * B:(s + 1) * B]
        Rp = got[s * B:(s + 1) * B, (s + 1) * B:].T
        kext = 3 * B if form == 1 else B
        for view, P, right in ((lv, Lp, False), (rv, Rp, True)):
            raw, sc = panel_slot(torch, view, s, s * B, m, kext)
            if form == 2:
                _, want_b, want_s = Bk.fp8_panel(P)
                assert np.array_equal(raw, want_b), (arm, s, right)
                assert np.array_equal(sc, want_s), (arm, s, right)
            elif form == 0:
                want = np.ascontiguousarray(P, np.float32).astype(np.float16).view(np.uint16)
                assert np.array_equal(raw.view(np.uint16), want), (arm, s, right)
            else:
                q = Bk.q_operand(1, P, right)
                want = (np.ascontiguousarray(q).view(np.uint32) >> 16).astype(np.uint16)
                assert np.array_equal(raw.view(np.uint16), want), (arm, s, right)
    ws.close()


@pytest.mark.parametrize("arm", ["fp16_split", "fp8_single_fused"])
def test_trsm_tile_counter_bit_identical(mxp, torch_cuda, arm):
    """TRSM-by-inverse tiles claimed from the device counter (default) or in
    static round robin: the same factors and FP8 panel bytes and scales."""
    torch = torch_cuda
    n = 10240
    out = {}
    for ctr in (1, 0):
        p, ws, _ = _factor(mxp, n, 5, arm, {mxp.OPT_TRSM_COUNTER: ctr})
        torch.cuda.synchronize()
        lv, rv = ws.panel_view(0), ws.panel_view(1)
        kext = B
        pans = [panel_slot(torch, v, s, s * B, n - (s + 1) * B, kext) for v in (lv, rv) for s in range(3)]
        out[ctr] = (p.A.clone(), pans)
        ws.close()
    assert torch.equal(out[1][0].view(torch.int32), out[0][0].view(torch.int32))
    for (a, sa), (b, sb) in zip(out[1][1], out[0][1]):
        assert np.array_equal(a, b)
        assert (sa is None and sb is None) or np.array_equal(sa, sb)


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("n,seed", [(2560, 7), (2048, 3)])
def test_inverses_tensor_levels(mxp, orc, torch_cuda, single, n, seed):
    """mxp_getrf_nopiv_inv at the benched block size: the LU and both
    triangular inverses, whose doubling levels from 1024 run as tensor-core
    products (split BF16, or one BF16 product for the single-product TRSM),
    against the oracle's restatement of the same levels."""
    torch = torch_cuda
    p = mxp.panel_matgen(n, seed)
    XU = torch.empty(n * n, device="cuda")
    XL = torch.empty(n * n, device="cuda")
    ws = mxp.Workspace(n, n, 0, trsm_single=single)
    mxp.getrf_nopiv_inv(p.A, n, n, XU, XL, n, ws)
    got_lu = to_np_colmajor(p.A, n, n, n)
    gu, gl = to_np_colmajor(XU, n, n, n), to_np_colmajor(XL, n, n, n)
    A, _, _, _ = orc.matgen(n, seed)
    info, wu, wl = Bk.getrf_nopiv_inv(A, 1024, Bk.FORM_BF16 if single else Bk.FORM_BF16X2)
    assert info == 0
    # the diagonal-block LU itself: FP32, same 64-column blocking
    assert rel_fro(got_lu, A) <= 1e-6
    tol = 2e-3 if single else 1e-4
    for g, w in ((gu, wu), (gl, wl)):
        assert rel_fro(g, w) <= tol
        assert np.max(np.abs(g.astype(np.float64) - w)) <= tol * np.max(np.abs(w))


@pytest.mark.parametrize("single", [False, True])
def test_inverse_chains_concurrent_bit_identical(mxp, torch_cuda, single):
    """The U and L tensor-core inverse chains run on two streams when the
    workspace has room for a second pair of operand casts (n >= 3b), one after
    the other otherwise: the same products either way, so the same bits."""
    torch = torch_cuda
    n = B
    out = []
    for ws_n in (3 * B, B):  # concurrent chains, then serial
        p = mxp.panel_matgen(n, 9)
        XU = torch.empty(n * n, device="cuda")
        XL = torch.empty(n * n, device="cuda")
        ws = mxp.Workspace(ws_n, B, 0, trsm_single=single)
        mxp.getrf_nopiv_inv(p.A, n, n, XU, XL, n, ws)
        torch.cuda.synchronize()
        out.append((p.A.clone(), XU, XL))
        ws.close()
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
