"""The 2D block-cyclic driver (openmxp_b200/grid.py) across gloo ranks on the
CPU, with the oracle's kernels standing in for the GPU ones
(tests/grid_cpu_backend.py): grids 1x1, 1x2, 2x1, 2x2 and 3x1, block counts
that do and do not divide evenly over the grid.

Checks, with the depth-1 look-ahead on (the default) and off:
- STRSM panels: the gathered factors equal, bit for bit, the oracle's
  single-process blocked LU of the same matrix (orc_panel_lu: FP32 STRSM
  panels, FP16 or split BF16 Schur update; every element receives the same
  operations in the same order whatever the grid and schedule);
- panels by inverse (split BF16 and single BF16 products against the FP32
  triangular inverses broadcast from the diagonal owner): the factors of
  every grid equal the one-process run's bit for bit, and that run matches
  the numpy restatement of the same algorithm (oracle/blocked.py panel_lu,
  whose FP32 sums run in another order) to 1e-5 relative Frobenius;
- FP8 Schur updates with b = 128 (each E4M3 scale tile one whole block):
  factors bit-exact with the oracle's one-process FP8 LU on 2x2, 1x2, 3x1,
  and with the one-process run when the panels are one-BF16 products;
- the refinement reaches scaled residual < 16 with the same iteration count
  as on one process, and the solution matches an FP64 solve of the FP64
  system to 1e-10.
The local extents agree with the C ABI's mxp_local_extent."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run(P, Q, n, b, seed, form, rank=0, dist=None, trsm="strsm", lookahead=True):
    from openmxp_b200 import grid as G
    from tests.grid_cpu_backend import OracleBackend
    g = G.ProcessGrid(P, Q, rank=rank, dist=dist)
    s = G.BlockCyclicSolver(g, n, b, seed, OracleBackend(b, form), form=form, trsm=trsm, lookahead=lookahead)
    s.factor()
    F = s.gather_factors(0)
    x, st = s.refine(maxit=20)
    return (None if F is None else F.numpy().copy()), x.numpy().copy(), st


def _worker(rank, P, Q, port, n, b, seed, form, trsm, lookahead, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=P * Q, timeout=datetime.timedelta(seconds=120))
    try:
        F, x, st = _run(P, Q, n, b, seed, form, rank, dist, trsm, lookahead)
        q.put((rank, F, x, st.iterations, st.converged, st.hpl_harness))
    finally:
        dist.destroy_process_group()


def _spawn(P, Q, n, b, seed, form, trsm="strsm", lookahead=True):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, P, Q, port, n, b, seed, form, trsm, lookahead, q))
          for r in range(P * Q)]
    for p in ps:
        p.start()
    res = {}
    for _ in ps:
        r = q.get(timeout=300)
        res[r[0]] = r[1:]
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    return res


@pytest.fixture(scope="module")
def reference_lu():
    """The oracle's single-process blocked LU and FP64 solution, per case."""
    from oracle import oracle as O
    cache = {}

    def get(n, b, seed, form):
        key = (n, b, seed, form)
        if key not in cache:
            A, d, _, rhs = O.matgen(n, seed)
            LU = A.copy(order="F")
            assert O.panel_lu(LU, b, form) == 0
            xt = np.linalg.solve(O.matgen_f64(n, seed, d), rhs)
            cache[key] = (LU, xt)
        return cache[key]
    return get


@pytest.mark.parametrize("P,Q,n,b", [(1, 2, 512, 64), (2, 1, 512, 64), (2, 2, 512, 64), (2, 2, 448, 64),
                                     (3, 1, 448, 64)])
def test_grid_lu_and_refinement(reference_lu, P, Q, n, b):
    from oracle import oracle as O
    seed, form = 42, O.FORM_FP16
    res = _spawn(P, Q, n, b, seed, form)
    LU, xt = reference_lu(n, b, seed, form)
    F = res[0][0].reshape(n, n).T  # column-major gathered factors
    assert np.array_equal(F.view(np.uint32), np.asarray(LU, np.float32).view(np.uint32))
    _, x1, st1 = _run(1, 1, n, b, seed, form)
    for r, (_, x, its, conv, hpl) in res.items():
        assert conv and hpl < 16.0, (r, hpl)
        assert its == st1.iterations
        assert np.array_equal(x, res[0][1])  # every process holds the same solution
        assert np.max(np.abs(x - xt)) / np.max(np.abs(xt)) < 1e-10


def test_grid_split_bf16_form(reference_lu):
    from oracle import oracle as O
    n, b, seed, form = 384, 64, 7, O.FORM_BF16X2
    res = _spawn(2, 2, n, b, seed, form)
    LU, xt = reference_lu(n, b, seed, form)
    F = res[0][0].reshape(n, n).T
    assert np.array_equal(F.view(np.uint32), np.asarray(LU, np.float32).view(np.uint32))
    assert all(v[3] for v in res.values())


@pytest.mark.parametrize("P,Q,n", [(2, 2, 448), (1, 3, 512)])
def test_grid_without_lookahead(reference_lu, P, Q, n):
    """The plain schedule (whole trailing update, then the next panel) gives
    the same factors as the look-ahead one and as the oracle."""
    from oracle import oracle as O
    b, seed, form = 64, 42, O.FORM_FP16
    res = _spawn(P, Q, n, b, seed, form, lookahead=False)
    LU, xt = reference_lu(n, b, seed, form)
    F = res[0][0].reshape(n, n).T
    assert np.array_equal(F.view(np.uint32), np.asarray(LU, np.float32).view(np.uint32))
    assert all(v[3] and v[4] < 16.0 for v in res.values())


@pytest.fixture(scope="module")
def inverse_lu():
    """The one-process grid run with panels by inverse, per case."""
    cache = {}

    def get(n, b, seed, form, trsm):
        key = (n, b, seed, form, trsm)
        if key not in cache:
            cache[key] = _run(1, 1, n, b, seed, form, trsm=trsm)
        return cache[key]
    return get


@pytest.mark.parametrize("P,Q,n,trsm,lookahead", [(2, 2, 512, "split", True), (2, 2, 448, "split", False),
                                                  (3, 1, 448, "split", True), (1, 2, 512, "single", True)])
def test_grid_trsm_by_inverse(reference_lu, inverse_lu, P, Q, n, trsm, lookahead):
    from oracle import oracle as O
    b, seed, form = 64, 42, O.FORM_FP16
    F1, x1, st1 = inverse_lu(n, b, seed, form, trsm)
    res = _spawn(P, Q, n, b, seed, form, trsm=trsm, lookahead=lookahead)
    F = res[0][0]
    assert np.array_equal(F.view(np.uint32), F1.view(np.uint32))
    _, xt = reference_lu(n, b, seed, form)
    for r, (_, x, its, conv, hpl) in res.items():
        assert conv and hpl < 16.0, (r, hpl)
        assert its == st1.iterations
        assert np.array_equal(x, res[0][1])  # the refinement's sums over the grid differ from one process's
        assert np.max(np.abs(x - xt)) / np.max(np.abs(xt)) < 1e-10


@pytest.mark.parametrize("trsm", ["split", "single"])
def test_one_process_inverse_panels_match_blocked_oracle(inverse_lu, trsm):
    from oracle import blocked as BO
    from oracle import oracle as O
    n, b, seed, form = 512, 64, 42, O.FORM_FP16
    F1, _, _ = inverse_lu(n, b, seed, form, trsm)
    A, _, _, _ = O.matgen(n, seed)
    LU = A.copy(order="F")
    assert BO.panel_lu(LU, b, BO.FORM_FP16, trsm=trsm) == 0
    got = F1.reshape(n, n).T.astype(np.float64)
    want = np.asarray(LU, np.float64)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-5


@pytest.mark.parametrize("P,Q,lookahead,trsm", [(2, 2, True, "strsm"), (1, 2, False, "strsm"),
                                                (3, 1, True, "strsm"), (2, 2, True, "single")])
def test_grid_fp8_form(reference_lu, inverse_lu, P, Q, lookahead, trsm):
    """FP8 Schur updates (E4M3 operands, one power-of-two scale per 128 x 128
    tile): with b = 128 every scale tile is one whole block, so the factors
    equal the one-process oracle LU's bit for bit on any grid (STRSM panels),
    or the one-process grid run's (panels by one BF16 product, as the FP8
    form's TRSM runs)."""
    from oracle import oracle as O
    n, b, seed, form = 640, 128, 42, O.FORM_FP8
    res = _spawn(P, Q, n, b, seed, form, trsm=trsm, lookahead=lookahead)
    LU, xt = reference_lu(n, b, seed, form)
    F = res[0][0].reshape(n, n).T
    if trsm == "strsm":
        assert np.array_equal(F.view(np.uint32), np.asarray(LU, np.float32).view(np.uint32))
    else:
        F1, _, _ = inverse_lu(n, b, seed, form, trsm)
        assert np.array_equal(res[0][0].view(np.uint32), F1.view(np.uint32))
    for r, (_, x, its, conv, hpl) in res.items():
        assert conv and hpl < 16.0, (r, hpl)
        assert np.max(np.abs(x - xt)) / np.max(np.abs(xt)) < 1e-10


def test_single_process_grid_matches_oracle(reference_lu):
    from oracle import oracle as O
    n, b, seed = 320, 64, 11
    F, x, st = _run(1, 1, n, b, seed, O.FORM_FP16)
    LU, xt = reference_lu(n, b, seed, O.FORM_FP16)
    assert np.array_equal(F.reshape(n, n).T.view(np.uint32), np.asarray(LU, np.float32).view(np.uint32))
    assert st.converged and np.max(np.abs(x - xt)) / np.max(np.abs(xt)) < 1e-10


@pytest.mark.parametrize("n,b", [(512, 64), (448, 64), (122880, 2560), (2560, 2560)])
def test_local_extent_matches_abi(n, b):
    import ctypes as C

    import openmxp_b200 as mxp
    from openmxp_b200 import grid as G
    for nproc in (1, 2, 3, 4, 5, 8):
        tot = 0
        for me in range(nproc):
            ext = C.c_int64(-1)
            assert mxp.lib().mxp_local_extent(n, b, nproc, me, C.byref(ext)) == 0
            assert ext.value == G.local_extent(n, b, nproc, me)
            tot += ext.value
        assert tot == n


def test_blocks_upto():
    from openmxp_b200 import grid as G
    for nproc in (1, 2, 3, 4):
        for me in range(nproc):
            for k in range(-1, 20):
                assert G.blocks_upto(k, nproc, me) == sum(1 for I in range(k + 1) if I % nproc == me)


def test_grid_rejects_bad_shapes():
    from openmxp_b200 import grid as G
    with pytest.raises(ValueError):
        G.ProcessGrid(2, 2)  # more than one process without torch.distributed
    with pytest.raises(ValueError):
        G.local_extent(100, 64, 2, 0)
    from tests.grid_cpu_backend import OracleBackend
    with pytest.raises(ValueError):
        G.BlockCyclicSolver(G.ProcessGrid(1, 1), 128, 64, 1, OracleBackend(64, 0), trsm="lu")
