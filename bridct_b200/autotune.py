"""Autotuner for the batching form: picks the work-unit geometry of a ragged batch.

The persistent ragged kernel cuts a batch into units per shape class: whole arrays up to
`tile_floats` (both passes in one unit), column strips of `strip_floats` and row blocks of
`row_floats` for larger arrays, with `lookahead` larger arrays' strips queued ahead of their row
passes.  The best geometry depends on the batch's mix of shapes, so it is measured:

    from bridct_b200.autotune import tune
    result = tune(items, x)            # items: [(h, w, mode)], x: packed float32 CUDA tensor
    batch = RaggedBatch(items, tuning=result["best"])

The search is coordinate descent from the library default over the candidate values below (two
sweeps), each candidate timed with CUDA events around CUDA-graph replays of the persistent
launch on the caller's data.  Every candidate result is checked against the default geometry's
output before its time counts.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

CANDIDATES: Dict[str, Sequence[int]] = {
    "tile_floats": (1024, 2048, 4096, 8192, 16384),
    "strip_floats": (2048, 4096, 8192, 16384),
    "row_floats": (2048, 4096, 8192, 16384),
    "lookahead": (1, 2, 4, 8, 16, 32, 64),
}


def default_tuning() -> Dict[str, int]:
    from . import _lib

    t = _lib.RaggedTuning()
    _lib.lib().bridct_ragged_default_tuning(t)
    return {k: int(getattr(t, k)) for k in CANDIDATES}


def time_tuning(items, x, tuning: Dict[str, int], steps: int = 8, reference=None) -> Tuple[float, object]:
    """Milliseconds per persistent launch with `tuning` (graph replays); returns (ms, output)."""
    import torch

    from .ragged import RaggedBatch

    batch = RaggedBatch(items, tuning=tuning)
    y = torch.empty_like(x)
    stream = torch.cuda.Stream(device=x.device)
    with torch.cuda.stream(stream):
        for _ in range(3):
            batch.apply(x, y, stream=stream.cuda_stream)
    stream.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        for _ in range(steps):
            batch.apply(x, y, stream=stream.cuda_stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        g.replay()                      # warm the graph
        start.record(stream)
        g.replay()
        end.record(stream)
    end.synchronize()
    del g
    if batch.timed_out():
        raise RuntimeError(f"ragged launch reported a bounded-wait expiry with tuning {tuning}")
    if reference is not None:
        scale = float(reference.abs().max()) or 1.0
        if float((y - reference).abs().max()) > 1e-5 * scale:
            raise RuntimeError(f"ragged output with tuning {tuning} disagrees with the default geometry")
    return start.elapsed_time(end) / steps, y


def tune(items, x, candidates: Optional[Dict[str, Sequence[int]]] = None, sweeps: int = 2,
         steps: int = 8) -> Dict[str, object]:
    """Coordinate descent over `candidates`; returns {"best", "best_ms", "default_ms", "table"}."""
    candidates = candidates or CANDIDATES
    best = default_tuning()
    base_ms, reference = time_tuning(items, x, best, steps)
    table: List[Dict[str, object]] = [{"tuning": dict(best), "ms": base_ms}]
    seen = {tuple(sorted(best.items())): base_ms}
    best_ms = base_ms
    for _ in range(sweeps):
        improved = False
        for key, values in candidates.items():
            for v in values:
                trial = dict(best, **{key: int(v)})
                sig = tuple(sorted(trial.items()))
                if sig in seen:
                    continue
                ms, _ = time_tuning(items, x, trial, steps, reference)
                seen[sig] = ms
                table.append({"tuning": trial, "ms": ms})
                if ms < best_ms * 0.995:
                    best, best_ms, improved = trial, ms, True
        if not improved:
            break
    return {"best": best, "best_ms": best_ms, "default_ms": base_ms, "table": table}


def _time_graph(fn, x, steps: int) -> float:
    """Milliseconds per call of fn(stream) from a CUDA graph of `steps` calls (after a warm replay)."""
    import torch

    stream = torch.cuda.Stream(device=x.device)
    with torch.cuda.stream(stream):
        for _ in range(2):
            fn(stream.cuda_stream)
    stream.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        for _ in range(steps):
            fn(stream.cuda_stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        g.replay()
        start.record(stream)
        g.replay()
        end.record(stream)
    end.synchronize()
    del g
    return start.elapsed_time(end) / steps


def tune_classes(items, x, tuning: Optional[Dict[str, int]] = None, steps: int = 8,
                 streams: Sequence[int] = (1, 2, 4, 8)) -> Dict[str, object]:
    """Per-shape-class schedules of a ragged batch.

    Every shape class (height, width, mode) is timed alone in each schedule: in the persistent
    queue (a batch of that class's arrays only, at their own offsets), as its own fixed-shape
    launch, and for two-pass shapes with the few-array geometry; the fastest wins.  The chosen
    schedule is then timed on the whole batch for each side-stream count, next to the all-queue
    and all-launch schedules, a hybrid (whole-array classes in the queue, two-pass classes in
    their own launches), a merged schedule (two-pass classes in merged column and row passes) and
    size thresholds (classes under 1, 4, 16 or 64 MB in the queue, the rest in their own or merged
    launches), and the fastest whole-batch schedule is returned (its output checked against the
    all-queue result).  Returns {"schedule", "ms", "queue_ms", "launch_ms", "classes"}."""
    import torch

    from .ragged import RaggedBatch

    batch = RaggedBatch(items, tuning=tuning)
    y = torch.empty_like(x)
    ref = batch.apply(x)
    torch.cuda.synchronize()
    rows = []
    for i, c in enumerate(batch.classes()):
        idx = [k for k, it in enumerate(items) if (it[0], it[1], it[2]) == (c["h"], c["w"], c["mode"])]
        alone = RaggedBatch([items[k] for k in idx], offsets=[int(batch.offsets[k]) for k in idx], tuning=tuning)
        ms = {"queue": _time_graph(lambda s: alone.apply(x, y, stream=s), x, steps),
              "launch": _time_graph(lambda s: batch.apply_class(i, "launch", x, y, stream=s), x, steps)}
        if c["h"] * c["w"] > 16384:
            ms["launch_small"] = _time_graph(lambda s: batch.apply_class(i, "launch_small", x, y, stream=s), x, steps)
        best = min(ms, key=ms.get)
        rows.append({"class": c["key"], "arrays": c["arrays"], "ms": ms, "choice": best})
        del alone
    chosen = {r["class"]: r["choice"] for r in rows}
    every_launch = {r["class"]: min((k for k in r["ms"] if k != "queue"), key=r["ms"].get) for r in rows}
    # Timed alone, a class of a few small arrays is all launch latency whatever its schedule; run
    # together, the whole-array (tile) classes share one persistent launch beside the two-pass
    # classes' own launches.
    hybrid = {r["class"]: ("queue" if "launch_small" not in r["ms"] else every_launch[r["class"]]) for r in rows}
    # merged: the two-pass classes share one column-pass launch per column length and mode and one
    # row-pass launch per row length and mode (far fewer launches and tails); whole 32768-float
    # arrays keep their own launch, the rest the queue
    from .ragged import two_pass

    def merged_choice(r):
        h, w, m = (int(v) for v in r["class"].replace("/", "x").split("x"))
        if two_pass(h, w, m):
            return "merged"
        return "queue" if "launch_small" not in r["ms"] else every_launch[r["class"]]

    merged = {r["class"]: merged_choice(r) for r in rows}
    candidates = [("per_class", chosen), ("all_launch", every_launch), ("hybrid", hybrid), ("merged", merged)]
    # by size: classes of fewer than `thr` bytes share the persistent queue (one launch for all of
    # them, where alone each would be a launch-latency-bound launch of its own), larger classes keep
    # their own launches, or for two-pass shapes the merged passes
    def class_bytes(r):
        h, w, _ = (int(v) for v in r["class"].replace("/", "x").split("x"))
        return 8 * h * w * r["arrays"]

    for thr in (1 << 20, 4 << 20, 16 << 20, 64 << 20):
        big = [r for r in rows if class_bytes(r) >= thr]
        candidates.append((f"size{thr >> 20}MB", {r["class"]: every_launch[r["class"]] for r in big}))
        candidates.append((f"size{thr >> 20}MB_merged", {r["class"]: (merged[r["class"]] if merged[r["class"]] == "merged"
                                                                         else every_launch[r["class"]]) for r in big}))
    trials = []
    for name, classes in candidates:
        for n in streams:
            trials.append((name, {"classes": classes, "streams": int(n)}))
    results = [("all_queue", {"classes": {}, "streams": 1}, _time_graph(lambda s: batch.apply(x, y, stream=s), x, steps))]
    for name, sched in trials:
        b = RaggedBatch(items, tuning=tuning, schedule=sched)
        ms = _time_graph(lambda s: b.apply(x, y, stream=s), x, steps)
        torch.cuda.synchronize()
        scale = float(ref.abs().max()) or 1.0
        if float((y - ref).abs().max()) > 1e-5 * scale:
            raise RuntimeError(f"ragged schedule {name}/{sched['streams']} disagrees with the queue's output")
        results.append((name, sched, ms))
        del b
    name, sched, ms = min(results, key=lambda r: r[2])
    return {"schedule": sched, "kind": name, "ms": ms,
            "queue_ms": results[0][2],
            "trials": [{"kind": n, "streams": s["streams"], "ms": m} for n, s, m in results],
            "classes": rows}
