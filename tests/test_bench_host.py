"""Host-side pieces of bench.py that feed the reported line: the work model
behind the roofline, the int32 CSR the single-graph workloads use, and the
launch counts claimed as gpu_launches.  No GPU needed."""
import itertools

import numpy as np

import bench
from gputrianglecounting_b200 import graphs as G


def test_algorithmic_bytes_matches_definition():
    """B_alg = 4W + 4(n+1) + 4nnz + 16n with W = sum over undirected edges of
    min(d_u, d_v), checked against a direct loop on small graphs."""
    for g in (G.complete(6), G.wheel(9), G.rmat(8, 8, 3).numpy(), G.erdos_renyi(200, 6, 4).numpy()):
        off, ind = np.asarray(g.off, np.int64), np.asarray(g.ind, np.int64)
        n = off.size - 1
        deg = np.diff(off)
        w = 0
        for u in range(n):
            for v in ind[off[u]:off[u + 1]]:
                if u < v:
                    w += min(deg[u], deg[v])
        got = bench.algorithmic_bytes(g)
        assert got["W"] == w
        assert got["B_alg"] == 4 * w + 4 * (n + 1) + 4 * ind.size + 16 * n


def test_int32_offsets_keeps_the_graph():
    g = G.rmat(9, 8, 5).numpy()
    h = bench.int32_offsets(g)
    assert h.off.dtype == np.int32 and h.ind.dtype == np.int32
    assert np.array_equal(np.asarray(h.off, np.int64), np.asarray(g.off, np.int64))
    assert np.array_equal(h.ind, g.ind)
    assert bench.algorithmic_bytes(h) == bench.algorithmic_bytes(g)


def test_launch_counts_follow_the_library_plan():
    """5 launches per plain count with vertex-id labels (6 from 2^18 rows
    on, where long rows get their own placement launch), 11 with
    degree-rank labels; a batched step adds entry starts, globalize and
    per-graph T and drops the global-count kernel (and, with ranks, computes
    graph-major ranks in two more launches)."""
    assert bench.launches_per_count(1 << 22, 50 << 20) == 6           # RGG-like: ids
    assert bench.launches_per_count(1 << 16, 1 << 20) == 5            # small: ids
    assert bench.launches_per_count(1 << 20, 31 << 20) == 11          # R-MAT-like: ranks
    for n, nnz, lab in itertools.product((1 << 10, 1 << 20), (1 << 14, 1 << 25), (1, 2)):
        per = bench.launches_per_count(n, nnz, {"labels": lab})
        assert per == ((5 if n < (1 << 18) else 6) if lab == 1 else 11)
        assert bench.batch_launches(n, nnz, {"labels": lab}) == per + (2 if lab == 1 else 4)


def test_reference_timer_units_and_sampling():
    """The reference arm's timer: its units cover every row exactly once, a
    whole-graph step reproduces the reference's per-vertex r, and the k
    phases of the systematic light-unit sample cover every light unit
    exactly once (so the per-step estimates average to the full graph)."""
    from oracle import oracle as O
    g = bench.int32_offsets(G.rmat(11, 16, 3).numpy())
    rt = bench.ReferenceTimer(g, threads=2, step_s=1e-9)
    rows = np.sort(rt.unit_rows)
    assert np.array_equal(rows, np.arange(g.n))
    assert rt.unit_off[0] == 0 and rt.unit_off[-1] == g.n
    assert rt.n_heavy > 0                      # the hubs of an R-MAT graph
    rt.calibrate()
    assert not rt.whole and rt.k >= 1
    seen = np.concatenate([rt.light_units[p::rt.k] for p in range(rt.k)])
    assert np.array_equal(np.sort(seen), np.arange(rt.n_heavy, rt.unit_off.shape[0] - 1))
    st = rt.step(0)
    assert st["full_s"] > 0 and st["wall_s"] > 0
    whole = bench.ReferenceTimer(g, threads=2, step_s=1e9)
    whole.calibrate()
    assert whole.whole
    whole.step(0)
    r_ref, _, _, _ = O.per_vertex(g.off, g.ind)
    assert np.array_equal(whole.r, r_ref)
