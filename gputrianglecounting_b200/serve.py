"""Continuous-batching count server on one GPU.

Count requests arrive over time, each naming a graph whose CSR is already
resident in HBM.  The server keeps two FIFO queues -- small and large
requests (large: more than `large_nnz` adjacency entries) -- and a few
*slots* (a CUDA stream, a batch workspace and output buffers each).
Whenever a slot is free it admits queued small requests in arrival order
while their combined device footprint fits the slot's memory budget (and the
batch-size cap), packs their CSRs into the batched layout on the device
(gtc_batch_pack) and counts them in one pipeline run (gtc_count_batch).  A
large request runs alone, and large requests may hold at most all but one of
the slots, so small requests never queue behind them.  Requests that arrive while
batches run wait only for the next free slot, so admission and execution
overlap.  Each result (T and the per-vertex r) stays on the device; its
latency is the time from arrival to the host seeing the slot's completion
event.

The batching never changes a result: gtc_count_batch gives every graph
exactly what it gets alone (tested).

Device-memory exhaustion is handled on the host: a batch whose buffers cannot
be allocated goes back to the head of its queue, the slots' cached buffers are
released, and the admission cap halves (it doubles back after each completed
batch), so the batch is retried in smaller pieces; a request that cannot be
allocated even alone, with no other batch in flight, completes with
``error = "out of device memory"`` instead of stopping the loop.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api


@dataclass
class Request:
    rid: int
    graph_id: int
    arrival: float               # seconds, relative to the run start
    n: int = 0
    nnz: int = 0
    done: float = -1.0           # completion time (same clock)
    triangles: int = -1
    r: torch.Tensor | None = None   # per-vertex r on the device (kept if asked)
    error: str = ""                 # set when the request could not be served


def footprint_bytes(n: int, nnz: int, keep_vertex_results: bool = False) -> int:
    """Device bytes one request occupies inside a batch: the batch workspace
    the library sizes for the request alone (gtc_batch_workspace_size: union-id
    adjacency, forward lists, per-vertex records, accumulators and a ~66 KB
    size-independent part, which each request pays once and which covers the
    union's own and its rounding), plus its packed input (int64 offsets, int32
    ids, its vstart entry) and outputs (graph T; r when kept).  Summed over a batch this bounds
    the batch's real footprint from above."""
    share = api.batch_workspace_bytes(1, n, nnz)
    return share + 16 + 8 * (n + 1) + 4 * nnz + 8 + (8 * n if keep_vertex_results else 0)


def plan_batch(queue, budget: int, max_graphs: int, keep_vertex_results: bool = False) -> int:
    """Number of queued requests (a FIFO prefix) the next batch admits:
    as many as fit the memory budget and the cap, but always at least one
    (a single request larger than the budget runs alone)."""
    used, k = 0, 0
    for req in queue:
        need = footprint_bytes(req.n, req.nnz, keep_vertex_results)
        if k >= max_graphs or (k > 0 and used + need > budget):
            break
        used += need
        k += 1
    return k


def next_work(free_slot: bool, small_queue, large_queue, large_running: int,
              slots: int) -> str:
    """What a free slot takes next: "small" (a batch of small requests),
    "large" (one large request) or "" (nothing).  Small requests go first;
    large ones never take the last slot not already running a large one
    (with a single slot they simply wait for an empty small queue)."""
    if not free_slot:
        return ""
    if small_queue:
        return "small"
    if large_queue and large_running < max(1, slots - 1):
        return "large"
    return ""


def poisson_arrivals(rate: float, count: int, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson process with `rate` requests/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))


@dataclass
class _Slot:
    stream: torch.cuda.Stream
    counter: api.BatchCounter
    event: torch.cuda.Event | None = None
    requests: list = field(default_factory=list)
    out: api.BatchCounts | None = None
    batch: api.BatchCSR | None = None
    is_large: bool = False


def is_alloc_failure(exc: BaseException) -> bool:
    """A device allocation failed (torch's OOM, or the library's status)."""
    if isinstance(exc, torch.cuda.OutOfMemoryError):
        return True
    return isinstance(exc, api.GTCError) and exc.status == api._lib.GTC_ERR_OUT_OF_MEMORY


class CountServer:
    def __init__(self, graphs, device=None, slots: int = 3, budget_bytes: int = 6 << 30,
                 max_graphs: int = 512, keep_vertex_results: bool = False,
                 large_nnz: int = 16 << 20, tuning: dict | None = None):
        """graphs: device-resident CSRGraphs (int64 off, int32 ind) that
        requests refer to by index; tuning: launch shape for every batch
        (e.g. from autotune.autotune_batch), None = the library's choice."""
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.graphs = graphs
        self.budget = budget_bytes
        self.max_graphs = max_graphs
        self.cap = max_graphs                         # admission cap (halved on OOM)
        self.keep = keep_vertex_results
        self.slots = [self._new_slot() for _ in range(slots)]
        self.queue: deque[Request] = deque()          # small requests
        self.large: deque[Request] = deque()          # large requests
        self.large_nnz = large_nnz
        self.tuning = tuning
        self.batches = 0
        self.alloc_failures = 0
        self.hold = False                             # no launches until a batch completes

    # ---- device plumbing (one stream, counter and event per slot)
    def _new_slot(self) -> _Slot:
        return _Slot(torch.cuda.Stream(self.device), api.BatchCounter(self.device))

    def _record_event(self, slot: _Slot):
        ev = torch.cuda.Event()
        ev.record(slot.stream)
        return ev

    def _release_memory(self) -> None:
        for s in self.slots:
            if s.event is None:
                s.counter.release()
        torch.cuda.empty_cache()

    # ---- slots
    def _launch(self, slot: _Slot, reqs: list[Request]) -> bool:
        """Pack and count reqs on the slot; False if device memory ran out
        (nothing is left queued for them)."""
        gs = [self.graphs[r.graph_id] for r in reqs]
        try:
            with torch.cuda.stream(slot.stream):
                batch = slot.counter.pack(gs, stream=slot.stream)
                out = slot.counter.count(batch,
                                         outputs=("r", "graph_T") if self.keep else ("graph_T",),
                                         stream=slot.stream, tuning=self.tuning)
                ev = self._record_event(slot)
        except Exception as exc:                                       # noqa: BLE001
            if not is_alloc_failure(exc):
                raise
            return False
        slot.event, slot.requests, slot.out, slot.batch = ev, reqs, out, batch
        slot.is_large = len(reqs) == 1 and reqs[0].nnz > self.large_nnz
        self.batches += 1
        return True

    def _finish(self, slot: _Slot, now: float) -> list[Request]:
        T = slot.out.graph_T.cpu().numpy()
        vstart = slot.batch.vstart.cpu().numpy() if self.keep else None
        for i, req in enumerate(slot.requests):
            req.done = now
            req.triangles = int(T[i])
            if self.keep:
                req.r = slot.out.r[vstart[i]:vstart[i + 1]].clone()
        done = slot.requests
        slot.event, slot.requests, slot.out, slot.batch = None, [], None, None
        self.cap = min(self.max_graphs, self.cap * 2)
        self.hold = False
        return done

    def _on_alloc_failure(self, queue, reqs: list[Request], now: float) -> list[Request]:
        """Requeue a batch that could not be allocated; returns the requests
        that failed for good (a single request with nothing else in flight)."""
        self.alloc_failures += 1
        self._release_memory()
        busy = any(s.event is not None for s in self.slots)
        if len(reqs) == 1 and not busy:
            reqs[0].error = "out of device memory"
            reqs[0].done = now
            return reqs
        if len(reqs) > 1:
            self.cap = max(1, min(self.cap, len(reqs)) // 2)
        # with batches in flight, wait for one of them to free its memory
        self.hold = busy
        for r in reversed(reqs):
            queue.appendleft(r)
        return []

    # ---- the loop
    def run(self, requests: list[Request], timeout_s: float = 120.0) -> list[Request]:
        """Serve requests (sorted by arrival) in real time; returns them with
        completion times filled in."""
        for r in requests:
            g = self.graphs[r.graph_id]
            r.n, r.nnz = g.n, g.nnz
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        finished: list[Request] = []
        t0 = time.perf_counter()
        while len(finished) < len(requests):
            now = time.perf_counter() - t0
            if now > timeout_s:
                raise TimeoutError(f"serving did not finish in {timeout_s} s")
            while pending and pending[0].arrival <= now:
                req = pending.popleft()
                (self.large if req.nnz > self.large_nnz else self.queue).append(req)
            for slot in self.slots:
                if slot.event is not None and slot.event.query():
                    finished += self._finish(slot, time.perf_counter() - t0)
            for slot in self.slots:
                if self.hold:
                    break
                running_large = sum(1 for s in self.slots if s.event is not None and s.is_large)
                what = next_work(slot.event is None, self.queue, self.large, running_large,
                                 len(self.slots))
                if not what:
                    continue
                q = self.queue if what == "small" else self.large
                k = plan_batch(q, self.budget, self.cap, self.keep) if what == "small" else 1
                reqs = [q.popleft() for _ in range(k)]
                if not self._launch(slot, reqs):
                    finished += self._on_alloc_failure(q, reqs, time.perf_counter() - t0)
                    break                     # let running batches finish first
            if (not self.queue and not self.large and pending
                    and all(s.event is None for s in self.slots)):
                # idle until the next arrival
                wait = pending[0].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        return finished


def latency_stats(done: list[Request]) -> dict:
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    edges = sum(r.nnz // 2 for r in done)
    span = max(r.done for r in done) - min(r.arrival for r in done)
    return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "sustained_edges_per_s": edges / span if span > 0 else math.nan,
            "span_s": span}
