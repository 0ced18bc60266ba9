"""Host-side multi-rank logic on CPU: two gloo ranks partition a batch with no overlap and no
data collective, agree on the max-over-ranks timing, and, transforming their own shards (with the
oracle standing in for each rank's GPU), stitch back exactly the full-batch result.  The same
partition (bridct_b200.dist.shard / shard_range) feeds bench.py --gpus N and apply_sharded; ragged
batches split by elements (ragged_shard_range), as bench.py --workload ragged --gpus N does."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bridct_b200.dist import apply_sharded, gather_shards, max_over_ranks, shard, shard_range, stitch


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


def _transform_worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist

    from oracle import oracle as O

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        job = np.random.default_rng(5).uniform(-1, 1, (37, 16, 32)).astype(np.float32)  # every rank builds the job
        mine, first = shard(job, rank, world)                   # and transforms only its own arrays
        y_mine = O.sj_apply(np.ascontiguousarray(mine), 0)
        full = gather_shards(y_mine, first, job.shape[0])       # collection for checking only
        if rank == 0:
            q.put(("ok", bool(np.array_equal(full, O.sj_apply(job, 0))), int(mine.shape[0])))
        else:
            q.put(("ok", full is None, int(mine.shape[0])))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(("error", repr(e), -1))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_transform_their_shards_and_stitch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_transform_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [q.get(timeout=10) for _ in range(2)]
    assert all(r[0] == "ok" and r[1] is True for r in res), res
    assert sorted(r[2] for r in res) == [18, 19]


def test_apply_sharded_partition_logic_on_cpu():
    """apply_sharded's split and stitch, with the oracle as each device's transform."""
    import numpy as np

    from oracle import oracle as O

    x = np.random.default_rng(3).standard_normal((11, 8, 64)).astype(np.float32)
    seen = []

    def fake(piece, mode, dev):
        seen.append((dev, piece.shape[0]))
        return O.sj_apply(np.ascontiguousarray(piece), mode)

    y = apply_sharded(x, 1, devices=[0, 1, 2], transform=fake)
    assert seen == [(0, 4), (1, 4), (2, 3)]
    assert np.array_equal(y, O.sj_apply(x, 1))
    with pytest.raises(ValueError):
        stitch([(0, x[:3]), (4, x[4:])], 11)
    part, first = shard(x, 2, 3)
    assert first == 8 and part.shape[0] == 3


def test_ragged_shard_range_balances_elements():
    from bridct_b200.dist import ragged_shard_range

    rng = np.random.default_rng(9)
    sizes = [int(a * b) for a, b in zip(2 ** rng.integers(3, 11, 700), 2 ** rng.integers(3, 11, 700))]
    total = sum(sizes)
    for world in (1, 2, 3, 4, 8, 1000):
        spans = [ragged_shard_range(sizes, r, world) for r in range(world)]
        assert spans[0][0] == 0 and sum(c for _, c in spans) == len(sizes)
        for (a, n), (b, _) in zip(spans, spans[1:]):
            assert a + n == b                                                   # contiguous, in order
        for f, c in spans:
            assert abs(sum(sizes[f:f + c]) - total / world) <= max(sizes)       # within one array
    assert ragged_shard_range([], 0, 2) == (0, 0)
    with pytest.raises(ValueError):
        ragged_shard_range([64], 2, 2)


def _ragged_worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist

    from bridct_b200.dist import ragged_shard
    from oracle import oracle as O

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(12)
        items = [(int(2 ** rng.integers(3, 7)), int(2 ** rng.integers(3, 7)), int(rng.integers(0, 3)))
                 for _ in range(41)]
        x = rng.uniform(-1, 1, sum(h * w for h, w, _ in items)).astype(np.float32)
        mine, xs, first = ragged_shard(items, x, rank, world)     # a slice of the packed buffer
        out, pos = [], 0
        for h, w, m in mine:                                       # the oracle stands in for the GPU
            out.append(O.sj_apply(xs[pos:pos + h * w].reshape(1, h, w), m).ravel())
            pos += h * w
        y_mine = np.concatenate(out) if out else np.zeros(0, np.float32)
        parts = [None] * world
        dist.all_gather_object(parts, (first, len(mine), y_mine))
        if rank == 0:
            whole, pos = [], 0
            for h, w, m in items:
                whole.append(O.sj_apply(x[pos:pos + h * w].reshape(1, h, w), m).ravel())
                pos += h * w
            got = np.concatenate([p[2] for p in sorted(parts, key=lambda p: p[0])])
            q.put(("ok", bool(np.array_equal(got, np.concatenate(whole))), [p[1] for p in parts]))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(("error", repr(e), []))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_transform_balanced_ragged_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ragged_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    status, same, counts = q.get(timeout=10)
    assert status == "ok" and same, (status, same)
    assert sum(counts) == 41 and min(counts) > 0


def test_apply_ragged_sharded_partition_logic_on_cpu():
    """apply_ragged_sharded's element split and in-order stitch, with the oracle as each device's
    transform (per array)."""
    from bridct_b200.dist import apply_ragged_sharded
    from oracle import oracle as O

    rng = np.random.default_rng(21)
    items = [(int(2 ** rng.integers(3, 7)), int(2 ** rng.integers(3, 7)), int(rng.integers(0, 3))) for _ in range(29)]
    x = rng.uniform(-1, 1, sum(h * w for h, w, _ in items)).astype(np.float32)
    seen = []

    def fake(mine, piece, dev):
        seen.append((dev, len(mine)))
        out, pos = [], 0
        for h, w, m in mine:
            out.append(O.sj_apply(piece[pos:pos + h * w].reshape(1, h, w), m).ravel())
            pos += h * w
        return np.concatenate(out)

    y = apply_ragged_sharded(items, x, devices=[0, 1, 2], transform=fake)
    assert [d for d, _ in seen] == [0, 1, 2] and sum(n for _, n in seen) == 29
    pos, want = 0, []
    for h, w, m in items:
        want.append(O.sj_apply(x[pos:pos + h * w].reshape(1, h, w), m).ravel())
        pos += h * w
    assert np.array_equal(y, np.concatenate(want))
