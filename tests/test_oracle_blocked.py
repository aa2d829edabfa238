"""The numpy restatement of the blocked LU at the product's block size
(oracle/blocked.py) pinned on the CPU: its vectorised quantisers bit-exact
against the C oracle's scalar conversions (themselves pinned against F16C and
the reference's fp16sim), its plain-STRSM form against orc_panel_lu, and the
TRSM by inverse against the plain triangular solve."""
import numpy as np
import pytest

from oracle import blocked as Bk


def _random_floats(rng, count):
    """Finite FP32 values over the whole exponent range, plus edge cases."""
    u = rng.integers(0, 2 ** 32, count, dtype=np.uint64).astype(np.uint32)
    x = u.view(np.float32)
    x = x[np.isfinite(x)]
    edges = np.array([0.0, -0.0, 1.0, -1.0, 448.0, 449.0, 464.0, 465.0, 480.0, 2 ** -6, 2 ** -9, 2 ** -10,
                      3 * 2 ** -10, 65504.0, 65520.0, 6.1e-5, 5.96e-8, 2.98e-8, 1e-40], np.float32)
    return np.concatenate([x, edges, -edges])


def test_f16_round_bit_exact(orc):
    rng = np.random.default_rng(1)
    x = _random_floats(rng, 20000)
    got = Bk.f16_round(x).view(np.uint32)
    want = np.array([orc.lib().orc_h2f(orc.lib().orc_f2h(float(v))) for v in x], np.float32).view(np.uint32)
    assert np.array_equal(got, want)


def test_bf16_round_bit_exact(orc):
    rng = np.random.default_rng(2)
    x = _random_floats(rng, 20000)
    x = x[np.abs(x) < 3.3e38]
    got = Bk.bf16_round(x).view(np.uint32)
    want = (np.array([orc.lib().orc_f2bf(float(v)) for v in x], np.uint32) << 16)
    assert np.array_equal(got, want)


def test_e4m3_bit_exact(orc):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(8000) * 10.0 ** rng.uniform(-4, 2.7, 8000),
                        rng.uniform(-2 ** -5, 2 ** -5, 4000), _random_floats(rng, 4000)]).astype(np.float32)
    x = x[np.abs(x) < 1e6]
    want_b = np.array([orc.lib().orc_f2e4m3(float(v)) for v in x], np.uint8)
    assert np.array_equal(Bk.e4m3_bytes(x), want_b)
    want_v = np.array([orc.lib().orc_e4m32f(int(c)) for c in want_b], np.float32)
    assert np.array_equal(Bk.e4m3_round(x).view(np.uint32) & 0x7FFFFFFF, want_v.view(np.uint32) & 0x7FFFFFFF)


def test_e4m3_scale_exp(orc):
    rng = np.random.default_rng(4)
    a = np.concatenate([np.abs(rng.standard_normal(3000)) * 10.0 ** rng.uniform(-30, 30, 3000),
                        [0.0, 448.0, 449.0, 1.0, 1.75, 1.76, 3.5, 1e-38]]).astype(np.float32)
    want = np.array([orc.lib().orc_e4m3_scale_exp(float(v)) for v in a])
    assert np.array_equal(Bk.e4m3_scale_exp(a), want)


@pytest.mark.parametrize("m,K", [(300, 200), (128, 128), (257, 64)])
def test_fp8_panel_matches_c_cast(orc, m, K):
    rng = np.random.default_rng(m + K)
    P = (rng.standard_normal((m, K)) * 10.0 ** rng.uniform(-6, 1, (m, 1))).astype(np.float32)
    deq, byts, sc = Bk.fp8_panel(P)
    want_b, want_s = orc.kmajor_panel(2, P, right=False)
    assert np.array_equal(byts, want_b)
    assert np.array_equal(sc, want_s)


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("n,b,seed", [(512, 128, 42), (768, 256, 7)])
def test_blocked_fp32_trsm_matches_c_oracle(orc, form, n, b, seed):
    A1, _, _, _ = orc.matgen(n, seed)
    A2 = A1.copy(order="F")
    assert orc.panel_lu(A1, b, form) == 0
    assert Bk.panel_lu(A2, b, form, trsm="fp32") == 0
    low = np.tril(np.ones((n, n), bool), -1)
    d = np.abs(A2.astype(np.float64) - A1)
    # same algorithm, FP32 sums in another order
    assert np.linalg.norm(d[low]) <= 1e-5 * np.linalg.norm(A1[low])
    assert np.linalg.norm(d) <= 1e-6 * np.linalg.norm(A1)


@pytest.mark.parametrize("trsm,tol", [("split", 1e-5), ("single", 5e-3)])
@pytest.mark.parametrize("n,b,inv_tc", [(1024, 512, 128), (2048, 1024, 256), (1536, 256, 1024)])
def test_trsm_by_inverse_close_to_strsm(orc, trsm, tol, n, b, inv_tc):
    A1, _, _, _ = orc.matgen(n, 11)
    A2 = A1.copy(order="F")
    assert Bk.panel_lu(A1, b, 0, trsm="fp32") == 0
    assert Bk.panel_lu(A2, b, 0, trsm=trsm, inv_tc=inv_tc) == 0
    low = np.tril(np.ones((n, n), bool), -1)
    up = np.triu(np.ones((n, n), bool), 1)
    for part in (low, up):
        assert np.linalg.norm((A2 - A1)[part]) <= tol * np.linalg.norm(A1[part])


@pytest.mark.parametrize("b,inv_tc,tform,tol", [(2560, 1024, 1, 2e-7), (2560, 1024, 4, 2e-3),
                                                (1280, 0, 1, 2e-7), (2048, 512, 1, 2e-7)])
def test_tri_inverses(orc, b, inv_tc, tform, tol):
    A, _, _, _ = orc.matgen(b, 5)
    info, XU, XL = Bk.getrf_nopiv_inv(A, inv_tc, tform)
    assert info == 0
    U = np.triu(A).astype(np.float64)
    L = np.tril(A, -1).astype(np.float64) + np.eye(b)
    # X T = I scaled by the magnitude of the inverse's rows
    assert np.max(np.abs(XU @ U - np.eye(b))) <= tol
    assert np.max(np.abs(XL @ L - np.eye(b))) <= tol
    assert np.all(np.tril(XU, -1) == 0) and np.all(np.triu(XL, 1) == 0)


def test_c_quantiser_equals_numpy_on_views(orc):
    """q_operand (the C oracle's OpenMP quantiser, fed strided views in place)
    and the numpy quantisers give the same bits in every form."""
    rng = np.random.default_rng(9)
    big = np.asfortranarray((rng.standard_normal((1100, 500)) * 10.0 ** rng.uniform(-6, 1, (1100, 1)))
                            .astype(np.float32))
    for P in (big[100:, 50:450], big[100:1000, 50:450].T, big[::2, ::3]):
        for form in (0, 1, 2, 3, 4):
            for right in (False, True):
                a = Bk.q_operand(form, P, right)
                b = np.asfortranarray(Bk.q_operand_np(form, P, right))
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (form, right)
