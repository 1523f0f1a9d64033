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


def test_large_requests_never_take_the_last_slot():
    q_small, q_large = [R(10, 100)], [R(10**6, 10**8)]
    assert serve.next_work(True, q_small, q_large, 0, 3) == "small"
    assert serve.next_work(True, [], q_large, 1, 3) == "large"
    assert serve.next_work(True, [], q_large, 2, 3) == ""       # keep one slot for small ones
    assert serve.next_work(False, q_small, q_large, 0, 3) == ""
    assert serve.next_work(True, [], [], 0, 3) == ""
