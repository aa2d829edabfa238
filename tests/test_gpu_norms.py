"""The refinement's norms and scaled-residual bookkeeping against the oracle.

- mxp_infnorm is colv_infnorm_h (panel_norm.hpp:35-58): a maximum of
  absolute values, which is exact, so the result must equal the oracle's
  bit for bit;
- ||A||inf is hpl_infnorm (panel_norm.hpp:129-135), 2 max(d) for the row-sum
  diagonal, and max(rowsum + d) for the weaker stress diagonal (whose A is no
  longer 2 d in row norm): bit for bit;
- ||b||inf and ||x||inf: bit for bit;
- the scaled residual |r|/(|A||x| + |b|)/(n eps/2) (iterative_refinement.hpp:
  156-165) recomputed from the reported norms: bit for bit;
- the first evaluation (x0 = b ./ d, iterative_refinement.hpp:142-143): its
  residual is not small, so the GPU's and the oracle's sums of the same
  N terms in other orders agree to FP64 rounding (<= 1e-12 relative).
  Later evaluations are not compared value by value: once the solution is
  accurate, r is itself at the level of the rounding noise of the GEMV (a
  scaled residual below 16 means exactly that), so two correct summation
  orders give residual norms that differ by O(1).  Instead the oracle
  refines the GPU's own factors and must take the same number of corrections,
  and the GPU's final x must pass the oracle's residual test.
"""
import numpy as np
import pytest

from tests.gpu_util import to_np_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 1000, 4097, 65537])
def test_infnorm_bit_exact(mxp, orc, torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) * 10.0 ** rng.uniform(-8, 8, n)
    x[rng.integers(n)] = -3.0e9
    ws = mxp.Workspace(max(n, 64), 64, 0)
    got = mxp.infnorm(torch.from_numpy(x).cuda(), ws)
    want = orc.lib().orc_infnorm(n, x.ctypes.data)
    assert got == want == np.max(np.abs(x))


@pytest.mark.parametrize("form", [0, 2])
@pytest.mark.parametrize("n,b,seed,rule", [(2048, 256, 7, 0), (3072, 256, 11, 1), (4096, 512, 42, 0),
                                           (5120, 2560, 3, 0)])
def test_refinement_norms_and_history(mxp, orc, torch_cuda, form, n, b, seed, rule):
    p = mxp.panel_matgen(n, seed, rule)
    ws = mxp.Workspace(n, b, form, trsm_single=(form == 2))
    mxp.panel_lu(p, b, ws)
    LU = np.asfortranarray(to_np_colmajor(p.A, n, n, n))
    x, ist, _ = mxp.iterative_refinement(p, ws)
    xs = x.cpu().numpy()
    _, d, rs, rhs = orc.matgen(n, seed, rule, with_matrix=False)
    norma = 2.0 * np.max(d) if rule == 0 else np.max(rs + d)
    assert ist["norma"] == norma
    assert ist["normb"] == np.max(np.abs(rhs))
    assert ist["normx"] == np.max(np.abs(xs))
    eps = 2.0 ** -53
    hpl = ist["residual"] / (ist["norma"] * ist["normx"] + ist["normb"]) * 1.0 / (n * eps)
    assert hpl == ist["hpl_harness"]
    assert ist["converged"] == 1 and ist["hpl_harness"] < 16.0
    # the oracle refining the GPU's factors
    it, _, _, _, hist = orc.ir_classic(n, b, seed, LU, d, rs if rule else None, rhs)
    assert it == ist["iterations"]
    assert abs(ist["history"][0] - hist[0]) <= 1e-12 * hist[0]
    # the GPU's solution through the oracle's residual
    r = rhs.copy()
    orc.otf_gemv(n, seed, d, -1.0, xs, 1.0, r)
    assert np.max(np.abs(r)) / (norma * np.max(np.abs(xs)) + np.max(np.abs(rhs))) / (n * eps) < 16.0
