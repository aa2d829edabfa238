"""Failure detection of the 2D block-cyclic driver across gloo ranks on the
CPU (the failure is made on the host, no GPU involved): one rank of a 2 x 2
grid raises in the middle of the LU, between two of its steps, and leaves.
The other ranks must not wait for it for ever: their next collective with the
missing rank ends with an error (the peer's connection closes, or the process
group's short timeout expires), each reports it, and every process exits.
The failing rank is chosen so that a rank of its process row and one of its
process column both notice it, and one rank shares no group with it: that
one learns of it at the first whole-grid collective (the refinement's
residual sum) or, if it never reaches one, by its own next collective with a
rank that has already left."""
import os
import socket
import sys
import time

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PG_TIMEOUT_S = 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, P, Q, port, fail_rank, fail_call, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from openmxp_b200 import grid as G
    from oracle import oracle as O
    from tests.grid_cpu_backend import OracleBackend

    class FailingBackend(OracleBackend):
        """Raises at the fail_call-th Schur update of rank fail_rank."""

        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.calls = 0

        def schur(self, *a, **k):
            self.calls += 1
            if rank == fail_rank and self.calls == fail_call:
                raise RuntimeError("injected failure")
            return super().schur(*a, **k)

    dist.init_process_group("gloo", rank=rank, world_size=P * Q,
                            timeout=datetime.timedelta(seconds=PG_TIMEOUT_S))
    t0 = time.monotonic()
    try:
        g = G.ProcessGrid(P, Q, rank=rank, dist=dist)
        s = G.BlockCyclicSolver(g, 512, 64, 42, FailingBackend(64, O.FORM_FP16), form=O.FORM_FP16)
        s.factor()
        s.refine(maxit=20)
        q.put((rank, "finished", "", time.monotonic() - t0))
    except Exception as e:  # the injected failure, or a collective that lost its peer
        q.put((rank, "error", type(e).__name__ + ": " + str(e)[:200], time.monotonic() - t0))
    finally:
        if rank == fail_rank:
            q.close()
            q.join_thread()  # the report is written before the process goes
            os._exit(1)  # leaves without taking part in any further collective
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_rank_failure_ends_every_rank():
    P, Q, fail_rank = 2, 2, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, P, Q, port, fail_rank, 3, q)) for r in range(P * Q)]
    for p in ps:
        p.start()
    res = {}
    try:
        for _ in ps:
            r = q.get(timeout=6 * PG_TIMEOUT_S + 60)
            res[r[0]] = r[1:]
    finally:
        for p in ps:
            p.join(30)
            if p.is_alive():
                p.kill()
                p.join(5)
    assert set(res) == set(range(P * Q)), res
    assert res[fail_rank][0] == "error" and "injected failure" in res[fail_rank][1]
    for r, (state, msg, secs) in res.items():
        assert state == "error", (r, state, msg)  # nobody finished a solve that lost a rank
        assert secs < 6 * PG_TIMEOUT_S, (r, secs)
    assert ps[fail_rank].exitcode == 1
