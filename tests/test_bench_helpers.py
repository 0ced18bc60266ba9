"""bench.py's host-side helpers, on CPU: the multi-rank sharding of the job batch (every rank
gets exactly the workload's batch, the shards tile N copies of it), the launch counts it claims,
and the block-count rule of its timing."""
import numpy as np

import bench


def test_shard_of_tiles_n_copies_of_the_workload():
    x = np.arange(10 * 2 * 2, dtype=np.float32).reshape(10, 2, 2)
    mine, first = bench.shard_of(x, 0, 1)
    assert mine is x and first == 0
    for world in (2, 3, 8):
        parts = [bench.shard_of(x, r, world) for r in range(world)]
        assert all(p.shape == x.shape for p, _ in parts)                   # weak scaling: B arrays each
        assert [f for _, f in parts] == [r * 10 for r in range(world)]
        job = np.concatenate([p for p, _ in parts])
        assert np.array_equal(job, np.concatenate([x] * world))            # N copies, in order


def test_launches_per_step():
    assert bench.launches_per_step("sj", 8, 8, 262144, 0) == 1
    assert bench.launches_per_step("sj", 64, 64, 1024, 0) == 1
    assert bench.launches_per_step("sj", 1024, 1024, 1, 0) == 2
    assert bench.launches_per_step("sj", 1024, 32, 5, 1) == 1             # whole 32768-float arrays
    assert bench.launches_per_step("sj", 128, 256, 5, 0) == 2
    assert bench.launches_per_step("tc_bf16x3", 8, 8, 262144, 0) == 1
    assert bench.launches_per_step("tc_bf16x3", 64, 64, 1024, 0) == 1      # fused 64x64
    assert bench.launches_per_step("tc_tf32x3", 64, 64, 1024, 0) == 2
    assert bench.launches_per_step("tc_bf16x3", 256, 256, 2048, 0) == 2 * 1   # 512 MiB: one chunk
    assert bench.launches_per_step("tc_fp8", 256, 256, 2048, 0) == 12 * 2     # two 256 MB chunks


def test_block_count_and_spread():
    assert bench.block_count(0.5, 21) == 2000                 # about a second of blocks
    assert bench.block_count(100.0, 21) == 21                 # at least the requested blocks
    assert bench.block_count(1e-6, 21) == 4000                # capped
    s = bench.spread([3.0, 1.0, 2.0])
    assert s == {"blocks": 3, "min_ms": 1.0, "median_ms": 2.0, "max_ms": 3.0}


def test_parallelism_text():
    assert bench.parallelism(1, 262144, 0) == "single GPU"
    assert "dp4" in bench.parallelism(4, 262144, 262144) and "no collective" in bench.parallelism(4, 1, 1)


def test_ragged_share_cuts_n_copies_by_elements():
    rng = np.random.default_rng(7)
    items = [(int(2 ** rng.integers(3, 8)), int(2 ** rng.integers(3, 8)), int(rng.integers(0, 2)))
             for _ in range(60)]
    span = sum(h * w for h, w, _ in items)
    wl = {"items": items, "x": np.arange(span, dtype=np.float32), "desc": "mix"}
    for world in (2, 3, 5):
        shares = [bench.ragged_share(wl, r, world) for r in range(world)]
        assert sum((s["items"] for s in shares), []) == items * world          # contiguous runs, in order
        assert np.array_equal(np.concatenate([s["x"] for s in shares]), np.tile(wl["x"], world))
        for s in shares:
            assert s["x"].size == sum(h * w for h, w, _ in s["items"])
            assert abs(s["x"].size - span) <= max(h * w for h, w, _ in items)  # within one array of equal
