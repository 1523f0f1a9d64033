"""Seeded generators and the host-side CSR checks.  CPU only."""
import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import graphs as G


@pytest.mark.parametrize("make", [
    lambda: G.erdos_renyi(3000, 16, 1),
    lambda: G.rmat(12, 16, 2),
    lambda: G.rgg2d(5000, 12, 3),
])
def test_generators_give_valid_simple_csr(make):
    g = make().numpy()
    assert g.off.dtype == np.int64 and g.ind.dtype == np.int32
    assert G.validate_csr_host(g.off, g.ind) is None


def test_generators_are_deterministic():
    a, b = G.rmat(11, 8, 9).numpy(), G.rmat(11, 8, 9).numpy()
    assert np.array_equal(a.off, b.off) and np.array_equal(a.ind, b.ind)
    c = G.rmat(11, 8, 10).numpy()
    assert not np.array_equal(a.ind, c.ind)


def test_er_mean_degree():
    g = G.erdos_renyi(16384, 16, 1)
    assert abs(g.nnz / g.n - 16) < 0.3


def test_rgg_mean_degree_and_locality():
    g = G.rgg2d(20000, 12, 3).numpy()
    assert abs(g.nnz / g.n - 12) < 1.0
    row = np.repeat(np.arange(g.n), np.diff(g.off))
    # Morton order keeps most neighbours close in id
    assert np.median(np.abs(g.ind.astype(np.int64) - row)) < 0.05 * g.n


def test_rmat_skew():
    g = G.rmat(14, 16, 2).numpy()
    deg = np.diff(g.off)
    assert deg.max() > 20 * deg.mean()


def test_rmat_partial_vertex_range():
    g = G.rmat(10, 8, 4, n=700).numpy()
    assert g.n == 700 and G.validate_csr_host(g.off, g.ind) is None


@pytest.mark.parametrize("defect,expect", [
    ("selfloop", "self-loop"), ("unsorted", "row not strictly ascending"),
    ("dup", "row not strictly ascending"), ("asym", "not symmetric"),
    ("range", "index out of range"), ("offsets", "offsets do not span the adjacency array"),
])
def test_host_validator_catches(defect, expect):
    g = G.complete(5).numpy()
    off, ind = g.off.copy(), g.ind.copy()
    if defect == "selfloop":
        ind[0] = 0
    elif defect == "unsorted":
        ind[0], ind[1] = ind[1], ind[0]
    elif defect == "dup":
        ind[1] = ind[0]
    elif defect == "asym":
        off = np.array([0, 1, 1], np.int64); ind = np.array([1], np.int32)
    elif defect == "range":
        ind[3] = 9
    elif defect == "offsets":
        off[-1] += 1
    assert G.validate_csr_host(off, ind) == expect


def test_to_device_roundtrip_cpu():
    g = G.cycle(6)
    h = g.to("cpu").numpy()
    assert np.array_equal(h.off, g.off) and torch.is_tensor(g.to("cpu").off)


def test_batched_specs_shape():
    specs = G.batched_specs(4096, 4)
    ns = np.array([s["n"] for s in specs])
    assert len(specs) == 4096 and ns.min() >= 256 and ns.max() <= 262_144
    assert sum(s["kind"] == "er" for s in specs) == 2048
    assert specs == G.batched_specs(4096, 4)
    er = [s["mean_degree"] for s in specs if s["kind"] == "er"]
    ef = [s["edge_factor"] for s in specs if s["kind"] == "rmat"]
    assert 8 <= min(er) and max(er) <= 32 and 8 <= min(ef) and max(ef) <= 16


def test_concat_and_slice_roundtrip():
    gs = [G.make_spec_graph(s) for s in G.batched_specs(10, 3, 256, 2000)]
    b = G.concat_graphs(gs, "cpu")
    assert b.num_graphs == 10 and b.total_n == sum(g.n for g in gs)
    for i, g in enumerate(gs):
        h = b.graph(i)
        assert np.array_equal(np.asarray(h.off), np.asarray(g.off))
        assert np.array_equal(np.asarray(h.ind), np.asarray(g.ind))
        assert G.validate_csr_host(np.asarray(h.off), np.asarray(h.ind)) is None
