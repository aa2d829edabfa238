"""The device pieces of the 2D block-cyclic driver on one GPU, and the driver
itself on a one-process grid (the multi-process schedule is covered by the
gloo tests on the CPU; every call here has one GPU).

- mxp_matgen_local: every process's local matrix of a P x Q grid, generated
  coordinate by coordinate, equals bit for bit the matching blocks of
  mxp_matgen's whole matrix;
- mxp_otf_gemv_local: the partial GEMVs of all coordinates add up to
  mxp_otf_gemv's product (FP64 rounding of different summation orders);
- mxp_block_gemv against an FP64 torch product;
- BlockCyclicSolver on a 1 x 1 grid with the CUDA backend: factors bit for bit
  equal to mxp_panel_lu run with the same steps (one panel per Schur pass;
  STRSM panels, or panels by inverse on the tensor cores with the separate
  FP8 cast), with the look-ahead schedule on and off, refinement to scaled
  residual < 16, and the solution against an FP64 solve."""
import numpy as np
import pytest

from tests.gpu_util import rel_fro, to_np_colmajor

pytestmark = pytest.mark.gpu


def _local_blocks(full, n, b, P, Q, pr, pc):
    rows = [I for I in range(n // b) if I % P == pr]
    cols = [J for J in range(n // b) if J % Q == pc]
    ri = np.concatenate([np.arange(I * b, (I + 1) * b) for I in rows]) if rows else np.zeros(0, int)
    ci = np.concatenate([np.arange(J * b, (J + 1) * b) for J in cols]) if cols else np.zeros(0, int)
    return full[np.ix_(ri, ci)]


@pytest.mark.parametrize("n,b,P,Q", [(1024, 128, 2, 2), (1280, 128, 3, 2), (768, 256, 1, 3), (2560, 2560, 1, 1)])
def test_matgen_local_bit_exact(mxp, torch_cuda, n, b, P, Q):
    torch = torch_cuda
    from openmxp_b200 import grid as G
    p = mxp.panel_matgen(n, 42)
    full = to_np_colmajor(p.A, n, n, n)
    for pr in range(P):
        for pc in range(Q):
            ml, nl = G.local_extent(n, b, P, pr), G.local_extent(n, b, Q, pc)
            if ml == 0 or nl == 0:
                continue
            A = torch.full((ml * nl,), float("nan"), device="cuda")
            mxp.check(mxp.lib().mxp_matgen_local(n, b, 42, P, Q, pr, pc, p.d.data_ptr(), A.data_ptr(), ml,
                                                 torch.cuda.current_stream().cuda_stream))
            got = to_np_colmajor(A, ml, nl, ml)
            want = _local_blocks(full, n, b, P, Q, pr, pc)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (pr, pc)


@pytest.mark.parametrize("n,b,P,Q", [(2048, 256, 2, 2), (1536, 128, 3, 1), (1024, 512, 1, 2)])
def test_otf_gemv_local_sums_to_whole(mxp, torch_cuda, n, b, P, Q):
    torch = torch_cuda
    p = mxp.panel_matgen(n, 7)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    ws = mxp.Workspace(n, b, 0)
    whole = torch.zeros(n, dtype=torch.float64, device="cuda")
    mxp.otf_gemv(n, 7, p.d, 1.0, x, 0.0, whole, ws)
    parts = torch.zeros(n, dtype=torch.float64, device="cuda")
    for pr in range(P):
        for pc in range(Q):
            mxp.check(mxp.lib().mxp_otf_gemv_local(n, b, 7, P, Q, pr, pc, p.d.data_ptr(), 1.0, x.data_ptr(),
                                                   parts.data_ptr(), torch.cuda.current_stream().cuda_stream))
    scale = float((p.d.abs().max() + 0.5 * n) * x.abs().max())
    assert float((parts - whole).abs().max()) <= 1e-14 * scale


@pytest.mark.parametrize("m,k", [(2560, 2560), (777, 130), (64, 1)])
def test_block_gemv(mxp, torch_cuda, m, k):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(5)
    lda = m + 3
    A = torch.rand(lda * k, device="cuda", generator=g) - 0.5
    x = torch.rand(k, dtype=torch.float64, device="cuda", generator=g)
    y = torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    want = 0.5 * y - 2.0 * (A.view(k, lda)[:, :m].t().double() @ x)
    mxp.check(mxp.lib().mxp_block_gemv(m, k, -2.0, A.data_ptr(), lda, x.data_ptr(), 0.5, y.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream))
    assert float((y - want).abs().max()) <= 1e-13 * float(want.abs().max())


@pytest.mark.parametrize("form,trsm,lookahead", [(0, "strsm", True), (2, "strsm", True), (0, "split", True),
                                                 (2, "split", True), (2, "single", False)])
def test_one_process_grid_solver(mxp, orc, torch_cuda, form, trsm, lookahead):
    torch = torch_cuda
    from openmxp_b200 import grid as G
    n, b, seed = 2048, 256, 42
    be = G.CudaBackend(b, form)
    s = G.BlockCyclicSolver(G.ProcessGrid(1, 1), n, b, seed, be, form=form, trsm=trsm, lookahead=lookahead)
    s.factor()
    got = to_np_colmajor(s.A, n, n, n)
    # the single-GPU LU with the same steps: one panel per Schur pass, the
    # same panel solves, the FP8 panels from the separate cast
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form)
    ws.set_option(mxp.OPT_TRSM_TENSOR, 0 if trsm == "strsm" else 1)
    ws.set_option(mxp.OPT_TRSM_SINGLE, 1 if trsm == "single" else 0)
    ws.set_option(mxp.OPT_FP8_FUSED_CAST, 0)
    ws.set_option(mxp.OPT_MERGE_PANELS, 0)
    mxp.panel_lu(p, b, ws)
    want = to_np_colmajor(p.A, n, n, n)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    x, st = s.refine(maxit=20)
    assert st.converged and st.hpl_harness < 16.0
    A, d, _, rhs = orc.matgen(n, seed)
    xt = np.linalg.solve(orc.matgen_f64(n, seed, d), rhs)
    assert np.max(np.abs(x.cpu().numpy() - xt)) / np.max(np.abs(xt)) < 1e-10
    # and the oracle's restatement of the same algorithm, at the 1e-3 factor bar
    LU = A.copy(order="F")
    if trsm == "strsm":
        assert orc.panel_lu(LU, b, form) == 0
    else:
        from oracle import blocked as BO
        assert BO.panel_lu(LU, b, form, trsm=trsm) == 0
    assert rel_fro(got, LU) <= 1e-3
    be.close()
