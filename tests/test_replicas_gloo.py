"""bench.py's multi-rank plumbing (replicas: one system per GPU, value =
all ranks' FLOPs / max-over-ranks time), run as 2 gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist = bench.init_dist("gloo")
    mx = bench.max_over_ranks(10.0 + rank, dist)
    sm = bench.sum_over_ranks(1.0 + rank, dist)
    bench.barrier(dist)
    q.put((rank, mx, sm))
    dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 11.0, 3.0), (1, 11.0, 3.0)]


def _ref_worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import io
    import contextlib
    import bench
    bench.CPU_SAMPLE.update(n=512, b=64)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        rc = bench.main(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"])
    q.put((rank, rc, out.getvalue()))


def test_reference_arm_rank0_only():
    """Under torchrun the reference arm runs on rank 0 only; others exit 0."""
    import json
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_ref_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(300)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1] == 0 and res[1][1] == 0
    line = json.loads(res[0][2].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert res[1][2].strip() == ""


def _part_worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import bench
    import openmxp_b200 as mxp
    dist = bench.init_dist("gloo")
    sizes = mxp.batch_sizes(2048, 3)
    part = mxp.batch_partition(sizes, world)
    mine = [i for i in range(len(sizes)) if part[i] == rank]
    work = torch.tensor([float(sum(sizes[i] ** 3 for i in mine))], dtype=torch.float64)
    got = [None] * world
    dist.all_gather_object(got, mine)
    loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(loads, work)
    q.put((rank, got, [float(t) for t in loads]))
    dist.destroy_process_group()


def test_batched_form_shards_systems_across_ranks():
    """The batched form's multi-GPU split: every rank computes the same
    partition on its own, the parts cover each system exactly once, and the
    n^3 work is balanced (no data exchange between ranks is needed)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_part_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1] == res[1][1]
    parts = res[0][1]
    flat = sorted(i for part in parts for i in part)
    assert flat == list(range(2048))
    loads = res[0][2]
    assert max(loads) / (sum(loads) / len(loads)) < 1.001
