"""Live comparisons of the oracle with the reference's own CPU code compiled
in place (oracle/_ref).  Skipped where the reference tree was not available
to build it (e.g. on the GPU box, which relies on the committed fixtures)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("n,seed", [(64, 1), (300, 42), (777, 7)])
def test_generator_vs_reference(orc, n, seed):
    R = orc.ref()
    A, d, rs, rhs = orc.matgen(n, seed)
    Ar = np.zeros((n, n), np.float32, order="F")
    R.ref_fill_one_panel_f32(n, 0, 0, n, n, Ar.ctypes.data, n, seed, 1)
    off = ~np.eye(n, dtype=bool)
    assert np.array_equal(A[off].view(np.uint32), Ar[off].view(np.uint32))
    assert np.array_equal(np.diag(A), np.diag(Ar))
    br = np.zeros(n)
    R.ref_panel_fill_f64(n, 0, n, n, 1, br.ctypes.data, n, seed)
    assert np.array_equal(rhs, br)


def test_subblock_offsets_vs_reference(orc):
    R = orc.ref()
    n, seed = 1000, 11
    A, _, _, _ = orc.matgen(n, seed)
    blk = np.zeros((37, 53), np.float32, order="F")
    R.ref_fill_one_panel_f32(n, 300, 600, 37, 53, blk.ctypes.data, 37, seed, 0)
    assert np.array_equal(blk, A[300:337, 600:653])


def test_fp16_random_vs_f16c(orc):
    R = orc.ref()
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.standard_normal(3000) * 1e-5, rng.standard_normal(3000) * 1e3]).astype(np.float32)
    for v in xs:
        assert orc.lib().orc_f2h(float(v)) == R.ref_fp16_bits(float(v))


def test_otf_gemv_vs_reference_kernel(orc):
    R = orc.ref()
    n, seed = 512, 42
    rng = np.random.default_rng(1)
    _, d, _, _ = orc.matgen(n, seed, with_matrix=False)
    x = rng.standard_normal(n)
    # oracle full GEMV
    y = np.zeros(n)
    orc.otf_gemv(n, seed, d, 1.0, x, 0.0, y)
    # reference off-diagonal block kernel on one block row + explicit diagonal block
    i0, mb = 128, 64
    yr = np.zeros(mb)
    st = orc.lib().orc_state(n, seed, i0, 0)
    R.otf_gemv_kernel(n, mb, i0, 1.0, x.ctypes.data, yr.ctypes.data, st)  # columns [0, i0)
    st = orc.lib().orc_state(n, seed, i0, i0 + mb)
    xr = x[i0 + mb:].copy()
    R.otf_gemv_kernel(n, mb, n - i0 - mb, 1.0, xr.ctypes.data, yr.ctypes.data, st)
    Ad = np.array([[d[i0 + i] if i == j else orc.lib().orc_elem(n, seed, i0 + i, i0 + j)
                    for j in range(mb)] for i in range(mb)])
    yr += Ad @ x[i0:i0 + mb]
    assert np.allclose(yr, y[i0:i0 + mb], rtol=1e-13, atol=1e-12)


def test_sgetrf_vs_reference(orc):
    R = orc.ref()
    n = 320
    A, _, _, _ = orc.matgen(n, 3)
    a1 = A.copy(order="F")
    a2 = A.copy(order="F")
    R.ref_sgetrf_nopiv_naive(n, n, a1.ctypes.data, n)
    assert orc.lib().orc_getrf_nopiv(n, n, a2.ctypes.data, n) == 0
    # same algorithm and order; the reference build may contract a*b+c into FMAs,
    # so compare at the reference self-test's tolerance (sgetrf_nopiv.cpp:1004-1011)
    assert np.max(np.abs(a1 - a2)) <= 1e-4


def test_ir_1x1_reference_behaviour(orc):
    """The reference's 1x1 block substitution (suspected defect) converges more
    slowly than exact substitution; the product path uses the exact one."""
    n, b = 1024, 128
    A, d, rs, rhs = orc.matgen(n, 42)
    assert orc.panel_lu(A, b) == 0
    it_exact, *_ = orc.ir_classic(n, b, 42, A, d, None, rhs)
    it_ref, *_ = orc.ir_classic(n, b, 42, A, d, None, rhs, ref1x1=True)
    assert 0 <= it_exact < it_ref


@pytest.mark.parametrize("n,b,seed", [(512, 128, 42), (1024, 256, 7), (640, 320, 11)])
def test_reference_otf_gemv_driver(orc, n, b, seed):
    """ref_otf_gemv (the reference's otf_gemv_kernel driven block by block as
    panel_gemv.hpp:310-338 does) against the oracle's residual GEMV: the same
    FP64 products summed in another order."""
    R = orc.ref()
    _, d, _, rhs = orc.matgen(n, seed, with_matrix=False)
    x = np.random.default_rng(n).standard_normal(n)
    y1, y2 = rhs.copy(), rhs.copy()
    orc.otf_gemv(n, seed, d, -1.0, x, 1.0, y1)
    R.ref_otf_gemv(n, b, seed, d.ctypes.data, -1.0, x.ctypes.data, 1.0, y2.ctypes.data)
    scale = np.abs(orc.matgen_f64(n, seed, d)) @ np.abs(x) + np.abs(rhs)
    assert np.all(np.abs(y1 - y2) <= 1e-14 * scale)


@pytest.mark.parametrize("n", [256, 640])
def test_reference_tuned_getrf(orc, n):
    R = orc.ref()
    A, _, _, _ = orc.matgen(n, 3)
    A1, A2 = A.copy(order="F"), A.copy(order="F")
    assert orc.lib().orc_getrf_nopiv(n, n, A1.ctypes.data, n) == 0
    assert R.ref_getrf_diag(n, A2.ctypes.data, n) == 0
    assert np.linalg.norm(A1 - A2) <= 1e-6 * np.linalg.norm(A1)


def test_cpu_solve_with_reference_kernels(orc):
    """The CPU baseline's solve with the reference's compiled diagonal LU and
    residual kernel converges like the oracle's own."""
    rc1, x1, st1 = orc.solve(2048, 256, 42)
    rc2, x2, st2 = orc.solve(2048, 256, 42, ref_kernels=True)
    assert rc1 >= 0 and rc2 >= 0 and abs(rc1 - rc2) <= 1
    assert st2["hpl"] < 16.0
    assert np.max(np.abs(x1 - x2)) <= 1e-10 * np.max(np.abs(x1))
