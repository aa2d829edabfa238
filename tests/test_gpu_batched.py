"""Batched form: every system of a batch factored and refined in one
persistent launch, checked system by system against the oracle (factors:
relative Frobenius <= 1e-3, the FP16-form bar) and an FP64 solve (forward
error), plus determinism of the replayed graph and the autotuner."""
import numpy as np
import pytest

from tests.gpu_util import rel_fro

pytestmark = pytest.mark.gpu


def _check_system(orc, bt, i, b, factors=True):
    n, seed = bt.n[i], bt.seeds[i]
    got = bt.matrix(i).cpu().numpy()
    if factors:
        A, _, _, _ = orc.matgen(n, seed)
        assert orc.panel_lu(A, b, 0) == 0
        assert rel_fro(got, A) <= 1e-3
        low = np.tril(np.ones((n, n), bool), -1)
        up = np.triu(np.ones((n, n), bool), 1)
        assert rel_fro(got[low], A[low]) <= 1e-3
        assert rel_fro(got[up], A[up]) <= 1e-3
    _, d, _, rhs = orc.matgen(n, seed, with_matrix=False)
    x64 = np.linalg.solve(orc.matgen_f64(n, seed, d), rhs)
    x = bt.vec(bt.x, i).cpu().numpy()
    assert np.max(np.abs(x - x64)) / np.max(np.abs(x64)) < 1e-10


@pytest.mark.parametrize("b,tile_n,stages", [(64, 256, 3), (128, 256, 3), (128, 128, 2), (256, 256, 2),
                                             (256, 128, 4)])
def test_batched_factors_and_solutions(mxp, orc, torch_cuda, b, tile_n, stages):
    sizes = [n for n in (256, 512, 768, 1024, 1280, 512, 2048) if n % b == 0]
    bt = mxp.Batch(sizes, [1000 + i for i in range(len(sizes))])
    bt.set_config(b, tile_n, stages)
    bt.matgen()
    st = bt.solve()
    assert (st["b"], st["tile_n"], st["stages"]) == (b, tile_n, stages)
    res = bt.results()
    for i in range(len(sizes)):
        assert res[i]["converged"] == 1 and res[i]["hpl_harness"] < 16.0 and res[i]["info"] == 0
        _check_system(orc, bt, i, b)
    bt.close()


def test_batched_ragged_blocks_and_small_orders(mxp, orc, torch_cuda):
    """Orders that are not multiples of the block size (a short last block)."""
    sizes = [128, 384, 640, 896, 1152]
    bt = mxp.Batch(sizes, [77 + i for i in range(len(sizes))])
    bt.set_config(256, 256, 3)
    bt.matgen()
    bt.solve()
    for i, r in enumerate(bt.results()):
        assert r["converged"] == 1 and r["hpl_harness"] < 16.0
        _check_system(orc, bt, i, 256, factors=False)
    bt.close()


def test_batched_replay_is_deterministic(mxp, torch_cuda):
    sizes = mxp.batch_sizes(40, 3)
    bt = mxp.Batch(sizes, [1000 + i for i in range(len(sizes))])
    bt.matgen()
    bt.solve()
    x1, r1 = bt.x.clone(), bt.results()
    bt.matgen()
    bt.solve()
    assert torch_cuda.equal(x1, bt.x)
    assert r1 == bt.results()
    assert all(r["converged"] == 1 for r in r1)
    bt.close()


def test_batched_autotune(mxp, torch_cuda):
    sizes = mxp.batch_sizes(96, 5)
    bt = mxp.Batch(sizes, [1000 + i for i in range(len(sizes))])
    bt.matgen()
    cfg = bt.autotune(sample=24)
    assert cfg["autotuned"] == 1 and cfg["b"] in (64, 128, 256) and cfg["tile_n"] in (128, 256)
    bt.matgen()
    st = bt.solve()
    assert (st["b"], st["tile_n"], st["stages"]) == (cfg["b"], cfg["tile_n"], cfg["stages"])
    assert all(r["converged"] == 1 for r in bt.results())
    bt.close()


def test_batched_rejects_bad_orders(mxp, torch_cuda):
    for bad in ([100], [8320], [256, 0]):
        with pytest.raises(mxp.MxpError) as e:
            mxp.Batch(bad, [1] * len(bad))
        assert e.value.status == mxp.INVALID_ARG
    bt = mxp.Batch([256], [1])
    with pytest.raises(mxp.MxpError):
        bt.set_config(96, 256, 4)
    bt.close()
