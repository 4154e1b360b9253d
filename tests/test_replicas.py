"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy of the workload and the only collectives are the barrier and the
max-over-ranks of the timed region.  These helpers are exercised here with two
gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    torch, dist, ws, r, local = bench.dist_setup("gloo")
    assert (ws, r) == (world, rank)
    # each rank "timed" a different region; every rank must see the maximum
    local_ms = 100.0 + 10.0 * rank
    total = bench.max_over_ranks(dist, ws, local_ms)
    steps = 4
    value = total / (steps * ws)  # job-level ms per solve, as bench.run_ours reports it
    dist.barrier()
    q.put((rank, total, value))
    dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [110.0, 110.0]
    assert out[0][2] == pytest.approx(110.0 / 8)


def test_single_rank_needs_no_process_group():
    import bench
    torch, dist, ws, r, local = bench.dist_setup("gloo")
    assert ws == 1 and bench.max_over_ranks(dist, ws, 3.5) == 3.5
