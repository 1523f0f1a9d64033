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
