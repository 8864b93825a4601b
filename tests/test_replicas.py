"""The replica plumbing of bench.py --gpus N on CPU: world size 2 over gloo.

Every rank times its own independent system; the reported time is the maximum over
ranks and the throughput counts the units of all ranks.  No GPU is used.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from bit_b200 import replicas
    dist = replicas.init("gloo", timeout_s=60)
    r, w, local = replicas.rank_info()
    replicas.barrier(dist)
    ms = replicas.max_over_ranks(10.0 * (r + 1), dist)   # rank r "took" 10 (r+1) ms
    seeds = [None] * w
    dist.all_gather_object(seeds, replicas.system_seed(r))
    out.put((r, w, local, ms, seeds))
    replicas.finish(dist)


def test_two_replicas_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, world, local, ms, seeds) in enumerate(res):
        assert (rank, world, local) == (r, 2, r)
        assert ms == 20.0                      # every rank reports the slowest rank's time
        assert len(set(seeds)) == 2            # each rank owns a different system


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from bit_b200 import replicas
    assert replicas.init("gloo") is None
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.rank_info() == (0, 1, 0)
