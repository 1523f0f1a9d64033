"""Autotuner for the counting pipeline's launch shape.

Replaces the reference's brute-force sweep of 8 block sizes x 6
threads-per-intersection values (allParamTestGPURun, src/gpurun.cu:115-176,
grids in src/param.cu:2-6).  The knobs here never change a result (tested):

  group        threshold between the warp-per-item kernel and the block
               kernel: apexes with a forward list longer than 4*group go to
               the block kernel ("warp vs block");
  item_len     adjacency entries per warp work item (partition granularity);
  big_chunk    adjacency entries per block work item;
  big_hash_max longest forward list hashed in shared memory before the
               block kernel switches to in-place binary search ("hash vs
               search");
  labels       the degree-ordering policy: vertex ids ordered by (degree,
               id) (1) or degree ranks with rank-sorted forward lists and the
               block kernel's rank bitmap (2);
  region       warp-kernel hash slots per forward-list member (2 or 4):
               rows per table batch against collisions;
  rows         the group kernel's form with vertex-id labels: a warp per
               work item with per-row hash regions (1) or per-row merges of
               the id-ordered lists (2).

A graph's *degree profile* -- size, mean degree and skew buckets -- keys a
cache (in memory and, optionally, a JSON file), so each profile is tuned
once.  Each candidate is timed with CUDA events on the device (best of a few
runs after a warm-up).  search="grid" times every combination; "staged"
first picks labels x group x region x rows with the other knobs at the library's choice,
then item_len x big_chunk under that choice (for inputs whose single count
takes long, such as a whole batch).
"""
from __future__ import annotations

import itertools
import json
import math
import os
import threading

import torch

from . import api

DEFAULT_GRID = {
    "labels": (1, 2),
    "region": (2, 4),
    "rows": (1, 2),
    "group": (8, 16, 32),
    "item_len": (128, 256, 512, 1024),
    "big_chunk": (1024, 2048, 4096),
}
STAGES = (("labels", "group", "region", "rows"), ("item_len", "big_chunk"))

_lock = threading.Lock()
_memory: dict[str, dict] = {}


def degree_profile(off: torch.Tensor, nnz: int) -> str:
    """Bucketed (log2 n, log2 mean degree, log2 skew) of a CSR, as a key."""
    n = off.numel() - 1
    if n <= 0 or nnz <= 0:
        return "empty"
    deg = (off[1:] - off[:-1])
    dmax = int(deg.max().item())
    mean = nnz / n
    skew = dmax / max(mean, 1.0)
    return (f"n{int(math.log2(n))}-d{int(round(math.log2(max(mean, 1.0)) * 2))}"
            f"-s{int(math.log2(max(skew, 1.0)))}")


def load_cache(path: str | None) -> dict:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def save_cache(path: str | None, cache: dict) -> None:
    if not path:
        return
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def valid(tuning: dict) -> bool:
    """Per-row merges need vertex-id labels and use no hash regions, so
    (rows 2, labels 2) is rejected by the library and (rows 2, region 4)
    would time (rows 2, region 2) again."""
    if tuning.get("rows") == 2:
        return tuning.get("labels") != 2 and tuning.get("region", 2) == 2
    return True


def candidates(grid: dict | None = None):
    grid = grid or DEFAULT_GRID
    keys = sorted(grid)
    for vals in itertools.product(*(grid[k] for k in keys)):
        cand = dict(zip(keys, vals))
        if valid(cand):
            yield cand


def _search(time_fn, grid: dict, search: str):
    """(best ms, best tuning, candidates timed) over `grid` with time_fn."""
    if search == "grid":
        results = [(time_fn(c), c) for c in candidates(grid)]
        results.sort(key=lambda x: x[0])
        return results[0][0], results[0][1], len(results)
    if search != "staged":
        raise ValueError("search must be 'grid' or 'staged'")
    best: dict = {}
    best_ms, timed = math.inf, 0
    for stage in STAGES:
        sub = {k: grid[k] for k in stage if k in grid}
        if not sub:
            continue
        for cand in candidates(sub):
            tun = dict(best, **cand)
            if not valid(tun):
                continue
            ms = time_fn(tun)
            timed += 1
            if ms < best_ms:
                best_ms, stage_best = ms, tun
        best = dict(stage_best)
    return best_ms, best, timed


def time_tuning(counter: api.TriangleCounter, off, ind, tuning: dict, mode: str = "plain",
                reps: int = 3) -> float:
    """Best device time (ms) of one count with this tuning."""
    outputs = ("r",) if mode == "plain" else ()
    out = counter.count(off, ind, mode=mode, outputs=outputs, tuning=tuning)   # warm-up
    best = math.inf
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        counter.count(off, ind, mode=mode, out=out, tuning=tuning)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def autotune(off: torch.Tensor, ind: torch.Tensor, mode: str = "plain",
             cache_path: str | None = None, grid: dict | None = None,
             counter: api.TriangleCounter | None = None, reps: int = 3,
             force: bool = False, search: str = "grid") -> dict:
    """Best tuning for this graph's degree profile (cached per profile)."""
    key = f"{mode}:{degree_profile(off, ind.numel())}"
    with _lock:
        if not force and key in _memory:
            return dict(_memory[key]["tuning"])
        disk = load_cache(cache_path)
        if not force and key in disk:
            _memory[key] = disk[key]
            return dict(disk[key]["tuning"])
    counter = counter or api.TriangleCounter(off.device)
    best_ms, best, timed = _search(lambda c: time_tuning(counter, off, ind, c, mode, reps),
                                   grid or DEFAULT_GRID, search)
    entry = {"tuning": best, "ms": best_ms,
             "default_ms": time_tuning(counter, off, ind, {}, mode, reps),
             "candidates": timed}
    with _lock:
        _memory[key] = entry
        disk = load_cache(cache_path)
        disk[key] = entry
        save_cache(cache_path, disk)
    return dict(best)


def tuned_entry(off: torch.Tensor, nnz: int, mode: str = "plain") -> dict | None:
    """The cached entry (tuning, ms, default_ms) for this profile, if any."""
    return _memory.get(f"{mode}:{degree_profile(off, nnz)}")


def time_batch_tuning(counter: api.BatchCounter, batch: api.BatchCSR, out, tuning: dict,
                      reps: int = 2) -> float:
    """Best device time (ms) of one batched count with this tuning."""
    counter.count(batch, out=out, tuning=tuning)      # warm-up
    best = math.inf
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        counter.count(batch, out=out, tuning=tuning)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def autotune_batch(counter: api.BatchCounter, batch: api.BatchCSR, out=None,
                   cache_path: str | None = None, grid: dict | None = None, reps: int = 2,
                   force: bool = False, search: str = "staged") -> dict:
    """Best tuning for a batch (gtc_count_batch over the disjoint union),
    cached per degree profile of the union."""
    key = f"batch:{degree_profile(batch.off, batch.total_nnz)}"
    with _lock:
        if not force and key in _memory:
            return dict(_memory[key]["tuning"])
        disk = load_cache(cache_path)
        if not force and key in disk:
            _memory[key] = disk[key]
            return dict(disk[key]["tuning"])
    out = out if out is not None else counter.alloc_outputs(batch, ("graph_T",))
    best_ms, best, timed = _search(lambda c: time_batch_tuning(counter, batch, out, c, reps),
                                   grid or DEFAULT_GRID, search)
    entry = {"tuning": best, "ms": best_ms,
             "default_ms": time_batch_tuning(counter, batch, out, {}, reps),
             "candidates": timed}
    with _lock:
        _memory[key] = entry
        disk = load_cache(cache_path)
        disk[key] = entry
        save_cache(cache_path, disk)
    return dict(best)


def batch_entry(batch: api.BatchCSR) -> dict | None:
    """The cached batch entry (tuning, ms, default_ms) for this union, if any."""
    return _memory.get(f"batch:{degree_profile(batch.off, batch.total_nnz)}")
