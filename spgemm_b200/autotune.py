"""Autotuner of the batched path.

Picks the tuning (include/spgemm_b200.h `spgemm_tuning`: the smallest row
that is merged by sorting, bin thresholds of the warp-per-row bins, warp
hash-table sizes, the long-row threshold, the mid-row bitmap width) that runs a given batch fastest on this GPU. Each
candidate is planned (spgemm_batch_plan) and then timed as replays of the
batch's CUDA graph (spgemm_batch_execute), so the choice reflects exactly
the work a serving loop repeats. The search is coordinate descent from the
default tuning over the candidate values below; results are cached in a JSON
file keyed by the GPU name and the batch's shape, so the search runs once per
batch shape and device.
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

# Parameters searched, in order, with their candidate values. Every value
# satisfies the ranges spgemm_set_tuning enforces.
SEARCH = [
    ("warp_table_max", [256, 512, 1024]),
    ("warp_p_max", [1024, 2048, 4096]),
    ("warp_cap_max", [128, 256, 512, 1024, 2048]),  # rows above: sorted (or mid / block)
    ("esc_p_min", [0, 4096]),                        # 4096: no sorted rows
    ("long_p", [2048, 4096]),
    ("mid_cols", [0, 1 << 16, 1 << 18]),
]

DEFAULT_CACHE = Path(os.environ.get("SPGEMM_B200_TUNE_CACHE",
                                    Path.home() / ".cache" / "spgemm_b200" / "batch_tuning.json"))


def batch_key(device_name: str, precision: int, shapes) -> str:
    """Cache key: GPU, precision and the batch's size profile (count, total
    rows, columns, nnz of A and B)."""
    rows = sum(s[0] for s in shapes)
    cols = sum(s[1] for s in shapes)
    nnz_a = sum(s[2] for s in shapes)
    nnz_b = sum(s[3] for s in shapes)
    return f"{device_name}|p{precision}|n{len(shapes)}|r{rows}|k{cols}|a{nnz_a}|b{nnz_b}"


def _time_batch(h, reps: int) -> float:
    h.batch_execute(graph=True)  # records the graph
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        h.batch_execute(graph=True)
        best = min(best, time.perf_counter() - t0)
    return best


def tune_batch(h, A_list, B_list, device_name: str = "gpu", reps: int = 3,
               cache: Path | None = DEFAULT_CACHE, log=None) -> dict:
    """Choose and set the fastest tuning for this batch on handle `h`, and
    leave the batch planned with it. A_list / B_list: device CM structs (as
    for Handle.batch_plan). Returns {"tuning": {...}, "ms": best, "tried": n,
    "cached": bool}."""
    shapes = [(a.num_rows, a.num_cols, a.nnz, b.nnz) for a, b in zip(A_list, B_list)]
    key = batch_key(device_name, h.precision, shapes)
    store = {}
    if cache is not None and Path(cache).exists():
        try:
            store = json.loads(Path(cache).read_text())
        except (OSError, ValueError):
            store = {}
    if key in store:
        h.set_tuning(**store[key]["tuning"])
        h.batch_plan(A_list, B_list)
        return {"tuning": store[key]["tuning"], "ms": store[key]["ms"], "tried": 0, "cached": True}

    best = h.tuning()
    h.batch_plan(A_list, B_list)
    best_s = _time_batch(h, reps)
    tried = 1
    for name, values in SEARCH:
        for v in values:
            if best[name] == v:
                continue
            cand = dict(best)
            cand[name] = v
            try:
                h.set_tuning(**cand)
                h.batch_plan(A_list, B_list)
                s = _time_batch(h, reps)
            except Exception as e:  # a candidate the engine rejects is skipped
                if log:
                    log(f"autotune: {name}={v} rejected: {e}")
                continue
            tried += 1
            if log:
                log(f"autotune: {name}={v} {s * 1e3:.3f} ms (best {best_s * 1e3:.3f})")
            if s < best_s:
                best, best_s = cand, s
    h.set_tuning(**best)
    h.batch_plan(A_list, B_list)
    chosen = {name: best[name] for name, _ in SEARCH}
    if cache is not None:
        try:
            Path(cache).parent.mkdir(parents=True, exist_ok=True)
            store[key] = {"tuning": chosen, "ms": best_s * 1e3}
            Path(cache).write_text(json.dumps(store, indent=1, sort_keys=True))
        except OSError:
            pass
    return {"tuning": chosen, "ms": best_s * 1e3, "tried": tried, "cached": False}
