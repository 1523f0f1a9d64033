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


def footprint_bytes(n: int, nnz: int) -> int:
    """Device bytes one request occupies inside a batch: its share of the
    batch workspace (union-id adjacency, forward lists, per-vertex records,
    accumulators) plus packed input and outputs."""
    return 60 * n + 13 * nnz + 4096


def plan_batch(queue, budget: int, max_graphs: int) -> int:
    """Number of queued requests (a FIFO prefix) the next batch admits:
    as many as fit the memory budget and the cap, but always at least one
    (a single request larger than the budget runs alone)."""
    used, k = 0, 0
    for req in queue:
        need = footprint_bytes(req.n, req.nnz)
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
        self.keep = keep_vertex_results
        self.slots = [_Slot(torch.cuda.Stream(self.device), api.BatchCounter(self.device))
                      for _ in range(slots)]
        self.queue: deque[Request] = deque()          # small requests
        self.large: deque[Request] = deque()          # large requests
        self.large_nnz = large_nnz
        self.tuning = tuning
        self.batches = 0

    # ---- slots
    def _launch(self, slot: _Slot, reqs: list[Request]) -> None:
        gs = [self.graphs[r.graph_id] for r in reqs]
        with torch.cuda.stream(slot.stream):
            batch = slot.counter.pack(gs, stream=slot.stream)
            out = slot.counter.count(batch, outputs=("r", "graph_T") if self.keep else ("graph_T",),
                                     stream=slot.stream, tuning=self.tuning)
            ev = torch.cuda.Event()
            ev.record(slot.stream)
        slot.event, slot.requests, slot.out, slot.batch = ev, reqs, out, batch
        slot.is_large = len(reqs) == 1 and reqs[0].nnz > self.large_nnz
        self.batches += 1

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
        return done

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
                running_large = sum(1 for s in self.slots if s.event is not None and s.is_large)
                what = next_work(slot.event is None, self.queue, self.large, running_large,
                                 len(self.slots))
                if what == "small":
                    k = plan_batch(self.queue, self.budget, self.max_graphs)
                    self._launch(slot, [self.queue.popleft() for _ in range(k)])
                elif what == "large":
                    self._launch(slot, [self.large.popleft()])
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
