"""Serving loop: host-side admission logic (CPU) and, on the GPU, that every
request's result in the served mix equals the graph's result alone."""
from collections import namedtuple

import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import api, graphs as G, serve

R = namedtuple("R", "n nnz")


def test_plan_batch_fifo_budget_and_cap():
    q = [R(1000, 10_000)] * 10
    one = serve.footprint_bytes(1000, 10_000)
    assert serve.plan_batch(q, budget=3 * one, max_graphs=100) == 3
    assert serve.plan_batch(q, budget=100 * one, max_graphs=4) == 4
    # a request larger than the budget still runs (alone)
    assert serve.plan_batch([R(10**7, 10**9)] + q, budget=one, max_graphs=100) == 1
    assert serve.plan_batch([], budget=one, max_graphs=4) == 0


def test_poisson_arrivals_deterministic_and_rate():
    a = serve.poisson_arrivals(5000.0, 20000, seed=5)
    b = serve.poisson_arrivals(5000.0, 20000, seed=5)
    assert np.array_equal(a, b) and np.all(np.diff(a) > 0)
    assert abs(len(a) / a[-1] - 5000.0) / 5000.0 < 0.03


@pytest.mark.gpu
def test_served_results_equal_results_alone(cuda):
    specs = G.batched_specs(16, 21, 256, 4000)
    pool = [G.make_spec_graph(s, cuda) for s in specs] + [G.rmat(12, 16, 4).to(cuda)]
    tc = api.TriangleCounter(cuda)
    alone = []
    for g in pool:
        res = tc.count(g.off, g.ind, outputs=("r",))
        torch.cuda.synchronize()
        alone.append((res.triangles, res.r.clone()))
    rng = np.random.default_rng(3)
    arr = serve.poisson_arrivals(20000.0, 400, seed=3)
    reqs = [serve.Request(i, int(rng.integers(0, len(pool))), float(t)) for i, t in enumerate(arr)]
    server = serve.CountServer(pool, cuda, slots=2, budget_bytes=64 << 20, max_graphs=64,
                               keep_vertex_results=True)
    done = server.run(reqs, timeout_s=60)
    assert len(done) == len(reqs) and server.batches < len(reqs)   # requests were batched
    for r in done:
        T, rv = alone[r.graph_id]
        assert r.triangles == T
        assert torch.equal(r.r, rv)
    stats = serve.latency_stats(done)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0


def test_footprint_bounds_the_batch_workspace():
    """The admission footprint of a batch (sum over its requests) covers what
    the batch really allocates: the library's batch workspace for the union
    plus packed input and outputs."""
    from gputrianglecounting_b200 import api
    rng = np.random.default_rng(7)
    for _ in range(50):
        G_ = int(rng.integers(1, 200))
        ns = rng.integers(0, 300_000, G_)
        nnzs = ns * rng.integers(0, 40, G_)
        for keep in (False, True):
            admitted = sum(serve.footprint_bytes(int(n), int(e), keep) for n, e in zip(ns, nnzs))
            tn, te = int(ns.sum()), int(nnzs.sum())
            real = (api.batch_workspace_bytes(G_, tn, te) + 8 * (G_ + 1) + 8 * (tn + 1) + 4 * te
                    + 8 * G_ + (8 * tn if keep else 0))
            assert admitted >= real, (G_, keep, admitted, real)
            assert admitted <= 1.05 * real + api.batch_workspace_bytes(1, 0, 0) * G_


class _Done:
    def query(self):
        return True


class _FakeBatch:
    def __init__(self, gs):
        self.gs = gs
        self.vstart = torch.tensor(np.concatenate([[0], np.cumsum([g.n for g in gs])]))


class _FakeCounter:
    """Stands in for api.BatchCounter on the host: 'counts' a graph as T = n
    and raises torch's out-of-memory error when the batch's entries exceed
    the memory it pretends to have."""

    def __init__(self, server):
        self.server = server

    def pack(self, gs, stream=None):
        return _FakeBatch(gs)

    def count(self, batch, outputs=(), stream=None, tuning=None):
        nnz = sum(g.nnz for g in batch.gs)
        if nnz > self.server.fake_memory:
            raise torch.cuda.OutOfMemoryError("simulated: batch does not fit")
        return api.BatchCounts(r=None, t=None, lcc=None,
                               graph_T=torch.tensor([g.n for g in batch.gs]))

    def release(self):
        self.server.released += 1


class _HostServer(serve.CountServer):
    """The serving loop with its device plumbing replaced by host fakes."""

    def __init__(self, graphs, fake_memory, **kw):
        self.fake_memory = fake_memory
        self.released = 0
        super().__init__(graphs, device="cpu", **kw)

    def _new_slot(self):
        return serve._Slot(None, _FakeCounter(self))

    def _record_event(self, slot):
        return _Done()

    def _release_memory(self):
        for s in self.slots:
            s.counter.release()


def test_allocation_failure_splits_batches_and_fails_only_what_cannot_fit():
    """Simulated device-memory exhaustion: batches that do not fit are
    retried in halves, every request that fits alone is served with its
    result, and one that does not fit even alone completes with an error
    instead of stopping the loop."""
    graphs = [G.CSRGraph(np.zeros(n + 1, np.int64), np.zeros(e, np.int32))
              for n, e in [(10, 100)] * 12 + [(7, 5000)]]
    server = _HostServer(graphs, fake_memory=450, slots=2, budget_bytes=1 << 40,
                         max_graphs=64)
    reqs = [serve.Request(i, i % 12, 0.0) for i in range(24)] + [serve.Request(24, 12, 0.0)]
    done = server.run(reqs, timeout_s=10)
    assert len(done) == 25
    by_id = {r.rid: r for r in done}
    for i in range(24):
        assert by_id[i].error == "" and by_id[i].triangles == 10
    assert by_id[24].error == "out of device memory" and by_id[24].triangles == -1
    assert server.alloc_failures >= 2 and server.released > 0
    assert server.batches >= 6          # at most 4 requests of 100 entries fit per batch


def test_large_requests_never_take_the_last_slot():
    q_small, q_large = [R(10, 100)], [R(10**6, 10**8)]
    assert serve.next_work(True, q_small, q_large, 0, 3) == "small"
    assert serve.next_work(True, [], q_large, 1, 3) == "large"
    assert serve.next_work(True, [], q_large, 2, 3) == ""       # keep one slot for small ones
    assert serve.next_work(False, q_small, q_large, 0, 3) == ""
    assert serve.next_work(True, [], [], 0, 3) == ""
