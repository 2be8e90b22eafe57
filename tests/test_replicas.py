"""Multi-rank host logic with two gloo ranks on CPU (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from torchcor_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx = replicas.reduce_max(1.5 + rank)
        sm = replicas.reduce_sum(10.0 * (rank + 1))
        mine = replicas.shard(list(range(13)), rank, world, weight=lambda i: (i * 7) % 5 + 1)
        q.put((rank, mx, sm, mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_timing_totals_and_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, mx0, sm0, s0), (r1, mx1, sm1, s1) = out
    assert mx0 == mx1 == 2.5 and sm0 == sm1 == 30.0
    assert sorted(s0 + s1) == list(range(13)) and not set(s0) & set(s1)
    w = lambda i: (i * 7) % 5 + 1  # noqa: E731
    assert abs(sum(map(w, s0)) - sum(map(w, s1))) <= max(map(w, range(13)))


def test_shard_single_process():
    assert replicas.shard(list("abc"), 0, 1) == list("abc")
    assert replicas.reduce_max(3.0) == 3.0 and replicas.reduce_sum(2.0) == 2.0
    with pytest.raises(ValueError):
        replicas.shard([1], 2, 2)
