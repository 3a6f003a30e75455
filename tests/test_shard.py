"""Host-side logic of the multi-GPU path (design sharding), on CPU ranks with
the gloo backend: every design is solved exactly once, the assignment is the
same on every rank and balanced, and a rank that fails raises on the others
instead of hanging."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from coldplate_solver_b200 import geometry, shard


def small_designs():
    return [geometry.straight_channel(M=m, N=n, band=(2, m // 2)) for m, n in
            ((10, 12), (20, 30), (16, 40), (8, 9), (30, 31), (12, 64), (25, 25))]


def test_assignment_is_balanced_and_complete():
    ds = small_designs()
    for world in (1, 2, 3, 4):
        parts = shard.assign(ds, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(ds)))
        loads = [sum(ds[k].M * ds[k].N for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(d.M * d.N for d in ds)
    assert shard.assign(ds, 2) == shard.assign(list(ds), 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, fail_rank, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    ds = small_designs()

    def fake_solve(batch):  # stands in for the GPU batch solve (host logic only)
        if rank == fail_rank:
            raise RuntimeError("injected failure on this rank")
        return [{"cells": d.M * d.N, "rank": rank} for d in batch]
    try:
        res = shard.run_sharded(ds, fake_solve, rank, world)
        out_q.put((rank, "ok", [r["cells"] for r in res], sorted({r["rank"] for r in res})))
    except Exception as e:  # noqa: BLE001
        out_q.put((rank, "error", type(e).__name__, str(e)[:200]))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _run(world, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    out = {}
    while not q.empty():
        r = q.get()
        out[r[0]] = r[1:]
    return out


def test_two_gloo_ranks_gather_every_design_once():
    out = _run(2)
    ds = small_designs()
    expect = [d.M * d.N for d in ds]
    assert set(out) == {0, 1}
    for rank, (status, cells, ranks) in out.items():
        assert status == "ok", out
        assert cells == expect
        assert ranks == [0, 1]


def test_a_failing_rank_surfaces_as_an_error_not_a_hang():
    out = _run(2, fail_rank=1)
    assert out[1][0] == "error" and "injected" in out[1][2]
    # rank 0 either sees the collective fail or times out within the group timeout
    assert 0 not in out or out[0][0] == "error"
