"""Host-side multi-rank logic on CPU: two gloo ranks partition a batch with no overlap and no
data collective, and agree on the max-over-ranks timing."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from bridct_b200.dist import max_over_ranks, shard_range


def test_shard_range_covers_batch():
    for batch in (0, 1, 7, 262144, 262145):
        for world in (1, 2, 3, 8):
            spans = [shard_range(batch, r, world) for r in range(world)]
            assert spans[0][0] == 0
            for (a, n), (b, _) in zip(spans, spans[1:]):
                assert a + n == b
            assert sum(n for _, n in spans) == batch
            assert max(n for _, n in spans) - min(n for _, n in spans) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, count = shard_range(1000, rank, world)
        x = np.arange(1000, dtype=np.float64)[first:first + count]   # this rank's units only
        local_ms = 1.0 + rank                                        # stand-in device time
        q.put((rank, first, count, float(x.sum()), max_over_ranks(local_ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1:3] for r in res] == [(0, 500), (500, 500)]
    assert sum(r[3] for r in res) == sum(range(1000))
    assert all(r[4] == 2.0 for r in res)
