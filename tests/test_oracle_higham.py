"""The oracle of Higham's HPL-AI matrix family on the CPU: its parameter
search bit-exact against the reference's own higham_mat_comp_beta compiled in
place (oracle/_ref), its matrix equal to L U with the stated structure, and
its residual GEMV against the reference's hmg_gemv_* kernels driven as
otf_gemv(HMGen) does."""
import numpy as np
import pytest

from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n", [100, 1000, 4096, 20000, 37000])
@pytest.mark.parametrize("cond", [1e2, 1e4, 1e6])
@pytest.mark.parametrize("rho", [0.5, 0.125])
def test_beta_bit_exact_vs_reference(orc, n, cond, rho):
    assert orc.lib().orc_higham_beta(n, cond, rho) == orc.ref().higham_mat_comp_beta(n, cond, rho)


@pytest.mark.parametrize("n,cond,rho", [(200, 1e3, 0.5), (513, 1e4, 0.125), (1000, 1e2, 1.0)])
def test_matrix_is_lu_product(orc, n, cond, rho):
    a, b = orc.higham_params(n, cond, rho)
    A = orc.higham_matrix_f64(n, a, b)
    L = np.eye(n) + a * np.tril(np.ones((n, n)), -1)
    U = np.eye(n) + b * np.triu(np.ones((n, n)), 1)
    assert np.max(np.abs(L @ U - A)) <= 4e-16 * np.max(np.abs(A))
    A32, d = orc.higham_matgen(n, a, b)
    assert np.max(np.abs(A32 - A) / A) <= 2 ** -23
    assert np.array_equal(d, np.diag(A))
    assert orc.lib().orc_higham_infnorm(n, a, b) == pytest.approx(np.max(A.sum(axis=1)), rel=1e-14)


def test_column_fill_matches_whole_fill(orc):
    n = 700
    a, b = orc.higham_params(n, 1e3, 0.5)
    A, _ = orc.higham_matgen(n, a, b)
    cols = np.empty((n, 37), np.float32, order="F")
    orc.lib().orc_higham_matgen_cols(n, a, b, 600, 37, cols.ctypes.data, n)
    assert np.array_equal(cols, A[:, 600:637])


def test_gemv_matches_dense_product(orc):
    n = 777
    a, b = orc.higham_params(n, 1e3, 0.5)
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    got = orc.higham_gemv(n, a, b, -1.0, x, 0.5, y.copy())
    want = 0.5 * y - orc.higham_matrix_f64(n, a, b) @ x
    assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))


@needs_ref
@pytest.mark.parametrize("n,b", [(1024, 128), (768, 256)])
def test_gemv_vs_reference_kernels(orc, n, b):
    """rho = 1 (alpha = beta): the reference's kernels and the oracle agree to
    FP64 rounding.  rho != 1: the reference's diagonal-block kernel uses alpha
    and beta in each other's places; its result is the product with that
    matrix, which the oracle's element formula reproduces with the two
    parameters swapped inside the diagonal blocks."""
    R = orc.ref()
    x = np.random.default_rng(n).standard_normal(n)
    for rho in (1.0, 0.5):
        a, be = orc.higham_params(n, 1e3, rho)
        y_ref = np.zeros(n)
        R.ref_higham_gemv(n, b, a, be, 1.0, x.ctypes.data, y_ref.ctypes.data)
        A = orc.higham_matrix_f64(n, a, be)
        if rho != 1.0:
            swapped = orc.higham_matrix_f64(n, be, a)  # the entry formulas with alpha and beta exchanged
            for q in range(0, n, b):
                A[q:q + b, q:q + b] = swapped[q:q + b, q:q + b]
        assert np.max(np.abs(y_ref - A @ x)) <= 1e-14 * np.max(np.abs(y_ref))
    y_orc = orc.higham_gemv(n, a, be, 1.0, x, 0.0, np.zeros(n))
    assert np.max(np.abs(y_orc - y_ref)) > 1e-6 * np.max(np.abs(y_ref))
