"""tcgen05 Schur update (casts + mxp_schur_update) vs the oracle's
quantise-then-FP32-accumulate restatement.  Tolerance: FP32 accumulation of
K terms in a different order, bounded by 1e-5 * sum_k |l_ik r_jk|."""
import numpy as np
import pytest

from tests.gpu_util import from_np_colmajor, to_np_colmajor

pytestmark = pytest.mark.gpu

FORMS = [0, 1, 2]  # FP16, BF16X2, FP8 (block-scaled)


def _run(mxp, torch, form, m, n, K, seed=0, pair=True):
    rng = np.random.default_rng(seed + 31 * m + n + K + form)
    L = (rng.standard_normal((m, K)) * 1e-2).astype(np.float32)
    U = (rng.standard_normal((K, n)) * 0.5).astype(np.float32)
    Cm = rng.standard_normal((m, n)).astype(np.float32)
    ldc = m + 3
    dL = from_np_colmajor(torch, L, ld=m)
    dU = from_np_colmajor(torch, U, ld=K)
    dC = from_np_colmajor(torch, Cm, ld=ldc)
    Kx = 3 * K if form == 1 else K
    es = 1 if form == 2 else 2
    ldk = -(-Kx // (16 // es)) * (16 // es)
    dt = torch.uint8 if es == 1 else torch.int16
    Lp = torch.zeros(m * ldk + 64, dtype=dt, device="cuda")
    Rp = torch.zeros(n * ldk + 64, dtype=dt, device="cuda")
    ls = torch.zeros(((m + 127) // 128) * ((K + 127) // 128) + 16, dtype=torch.uint8, device="cuda")
    rs = torch.zeros(((n + 127) // 128) * ((K + 127) // 128) + 16, dtype=torch.uint8, device="cuda")
    ws = mxp.Workspace(max(m, n, K) + K, K, form, schur_pair=pair)
    mxp.panel_cast_left(form, m, K, dL, m, Lp, ldk, ls if form == 2 else None)
    mxp.panel_cast_right(form, n, K, dU, K, Rp, ldk, rs if form == 2 else None)
    mxp.schur_update(form, m, n, K, Lp, ldk, Rp, ldk, dC, ldc, ws, ls if form == 2 else None,
                     rs if form == 2 else None)
    torch.cuda.synchronize()
    return L, U, Cm, to_np_colmajor(dC, m, n, ldc)


@pytest.mark.parametrize("pair", [True, False])
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("m,n,K", [(128, 256, 64), (300, 500, 128), (1, 1, 64), (129, 257, 192),
                                   (1024, 1024, 256), (257, 300, 2560), (2048, 1536, 1024)])
def test_schur_vs_oracle(mxp, orc, torch_cuda, form, m, n, K, pair):
    L, U, Cm, got = _run(mxp, torch_cuda, form, m, n, K, pair=pair)
    want = orc.schur_update(form, Cm, L, U)
    bound = np.abs(L.astype(np.float64)) @ np.abs(U.astype(np.float64))
    err = np.abs(got.astype(np.float64) - want.astype(np.float64))
    assert np.all(err <= 1e-5 * bound + 1e-6 * np.abs(want) + 1e-30), float(np.max(err - 1e-5 * bound))


@pytest.mark.parametrize("pair", [True, False])
def test_schur_exact_small_integers(mxp, orc, torch_cuda, pair):
    """Integer-valued operands make every product and partial sum exact in
    FP32, so the tensor-core result must equal the oracle bit for bit: a
    direct check of the descriptor / swizzle / TMEM-lane mapping."""
    torch = torch_cuda
    m, n, K = 384, 512, 320
    rng = np.random.default_rng(2)
    L = rng.integers(-3, 4, (m, K)).astype(np.float32)
    U = rng.integers(-3, 4, (K, n)).astype(np.float32)
    Cm = rng.integers(-1000, 1000, (m, n)).astype(np.float32)
    dL = from_np_colmajor(torch, L)
    dU = from_np_colmajor(torch, U)
    dC = from_np_colmajor(torch, Cm)
    Lp = torch.zeros(m * K, dtype=torch.int16, device="cuda")
    Rp = torch.zeros(n * K, dtype=torch.int16, device="cuda")
    ws = mxp.Workspace(1024, K, 0, schur_pair=pair)
    mxp.panel_cast_left(0, m, K, dL, m, Lp, K)
    mxp.panel_cast_right(0, n, K, dU, K, Rp, K)
    mxp.schur_update(0, m, n, K, Lp, K, Rp, K, dC, m, ws)
    torch.cuda.synchronize()
    got = to_np_colmajor(dC, m, n, m)
    want = Cm - L @ U
    assert np.array_equal(got, want)


def _tiles(rng, rows, cols, scales):
    """Integer-valued blocks in [-7, 7] times a per-128x128-tile power of two."""
    a = rng.integers(-7, 8, (rows, cols)).astype(np.float32)
    for ti in range(-(-rows // 128)):
        for tk in range(-(-cols // 128)):
            a[ti * 128:(ti + 1) * 128, tk * 128:(tk + 1) * 128] *= np.float32(scales[(ti + tk) % len(scales)])
    return a


@pytest.mark.parametrize("K", [384, 640, 1152])
@pytest.mark.parametrize("pair", [True, False])
def test_schur_fp8_exact_tile_scales(mxp, orc, torch_cuda, pair, K):
    """FP8 with different power-of-two scales per 128x128 tile: every value is
    exact in E4M3 after scaling, every product and sum exact in FP32, so the
    block-scaled MMA must reproduce C - L U^T bit for bit.  Pins the scale-
    factor layout (rows, k-blocks, both operands, stage groups: 3, 5 and 9
    K stages)."""
    torch = torch_cuda
    rng = np.random.default_rng(3)
    m, n = 384, 512
    L = _tiles(rng, m, K, [1.0, 0.125, 0.25, 2.0])
    Ut = _tiles(rng, n, K, [0.5, 1.0, 4.0])      # R = U^T, rows n
    U = np.asfortranarray(Ut.T)
    Cm = rng.integers(-1000, 1000, (m, n)).astype(np.float32)
    dL = from_np_colmajor(torch, L)
    dU = from_np_colmajor(torch, U)
    dC = from_np_colmajor(torch, Cm)
    Lp = torch.zeros(m * K, dtype=torch.uint8, device="cuda")
    Rp = torch.zeros(n * K, dtype=torch.uint8, device="cuda")
    kt = -(-K // 128)
    ls = torch.zeros(3 * kt + 16, dtype=torch.uint8, device="cuda")
    rs = torch.zeros(4 * kt + 16, dtype=torch.uint8, device="cuda")
    ws = mxp.Workspace(1024, 128, 2, schur_pair=pair)
    mxp.panel_cast_left(2, m, K, dL, m, Lp, K, ls)
    mxp.panel_cast_right(2, n, K, dU, K, Rp, K, rs)
    mxp.schur_update(2, m, n, K, Lp, K, Rp, K, dC, m, ws, ls, rs)
    torch.cuda.synchronize()
    got = to_np_colmajor(dC, m, n, m)
    want = Cm - (L.astype(np.float64) @ U.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got, want)


def test_schur_rejects_bad_ld(mxp, torch_cuda):
    torch = torch_cuda
    ws = mxp.Workspace(256, 64, 0)
    buf = torch.zeros(1 << 16, dtype=torch.int16, device="cuda")
    C = torch.zeros(256 * 256, dtype=torch.float32, device="cuda")
    with pytest.raises(mxp.MxpError) as e:
        mxp.schur_update(0, 128, 128, 64, buf, 60, buf, 64, C, 256, ws)  # ldl < K
    assert e.value.status == mxp.INVALID_ARG
    with pytest.raises(mxp.MxpError):
        mxp.schur_update(0, 128, 128, 64, buf, 68, buf, 68, C, 256, ws)  # ld*2 not 16B multiple
