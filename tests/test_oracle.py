"""The CPU oracle (oracle/tc_oracle.c) against the reference's own outputs
and against closed forms.  CPU only."""
import math

import numpy as np
import pytest

from gputrianglecounting_b200 import graphs as G
from oracle import oracle as O


def row_sums(off, vals):
    off = np.asarray(off, np.int64)
    c = np.concatenate([[0], np.cumsum(vals)])
    return c[off[1:]] - c[off[:-1]]


def test_golden_trine_matches_reference(golden_cases):
    for name, (off, ind, trine, total) in golden_cases.items():
        mine, mine_total = O.tri_ne(off, ind)
        assert np.array_equal(mine, trine), name
        assert mine_total == total, name
        r, t, lcc, s = O.per_vertex(off, ind)
        assert np.array_equal(r, row_sums(off, trine)), name
        assert s == total and np.array_equal(t * 2, r), name


def test_golden_invariants(golden_cases):
    for name, (off, ind, trine, total) in golden_cases.items():
        assert total % 6 == 0, name
        r, t, lcc, _ = O.per_vertex(off, ind)
        assert (r % 2 == 0).all()
        assert O.oriented_sum(off, ind) * 2 == total, name
        deg = np.diff(off)
        assert (t <= deg * (deg - 1) // 2).all(), name


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_random(seed):
    for g in (G.erdos_renyi(700, 12, seed), G.rmat(10, 12, seed), G.rgg2d(900, 10, seed)):
        g = g.numpy()
        ref, ref_total = O.ref_tri_ne(g.off, g.ind)
        mine, mine_total = O.tri_ne(g.off, g.ind)
        assert np.array_equal(ref, mine) and ref_total == mine_total
        rr, rs = O.ref_rows(g.off, g.ind)
        r, _, _, s = O.per_vertex(g.off, g.ind)
        assert np.array_equal(rr, r) and rs == s


@pytest.mark.parametrize("n", [3, 4, 5, 9, 17])
def test_complete_graph(n):
    g = G.complete(n)
    r, t, lcc, s = O.per_vertex(g.off, g.ind)
    assert (t == math.comb(n - 1, 2)).all()
    assert s == 6 * math.comb(n, 3)
    assert (lcc == 1.0).all()


@pytest.mark.parametrize("n", [3, 4, 5, 12])
def test_cycles(n):
    g = G.cycle(n)
    r, t, lcc, s = O.per_vertex(g.off, g.ind)
    assert s == (6 if n == 3 else 0)
    assert (t == (1 if n == 3 else 0)).all()


def test_star_and_wheel():
    r, t, lcc, s = O.per_vertex(G.star(30).off, G.star(30).ind)
    assert s == 0 and (lcc == 0).all()
    w = G.wheel(11)          # hub + 10-cycle: 10 triangles
    r, t, lcc, s = O.per_vertex(w.off, w.ind)
    assert s == 60 and t[0] == 10 and (t[1:] == 2).all()
    assert lcc[0] == 20 / (10 * 9) and (lcc[1:] == 4 / 6).all()


def test_disjoint_union_is_additive():
    a, b = G.complete(6), G.wheel(9)
    u = G.disjoint_union(a, b)
    ra, _, _, sa = O.per_vertex(a.off, a.ind)
    rb, _, _, sb = O.per_vertex(b.off, b.ind)
    ru, _, _, su = O.per_vertex(u.off, u.ind)
    assert su == sa + sb and np.array_equal(ru, np.concatenate([ra, rb]))


def test_empty_and_isolated():
    g = G.from_edge_list(8, [])
    r, t, lcc, s = O.per_vertex(g.off, g.ind)
    assert s == 0 and (r == 0).all() and (lcc == 0).all()


def test_lcc_formula_exact():
    g = G.rmat(9, 8, 5).numpy()
    r, t, lcc, _ = O.per_vertex(g.off, g.ind)
    assert np.array_equal(lcc.view(np.int64), O.lcc_formula(r, np.diff(g.off)).view(np.int64))


def test_subset_matches_rows():
    g = G.rmat(9, 8, 6).numpy()
    r, _, _, _ = O.per_vertex(g.off, g.ind)
    v = np.array([0, 5, 5, 17, g.n - 1], np.int32)
    assert np.array_equal(O.subset(g.off, g.ind, v), r[v])


def test_planted_mistake_is_caught():
    """A corrupted oracle input (one triangle edge removed on one side only
    would be invalid; instead drop a whole edge) changes the count -- the
    comparison is sensitive."""
    g = G.complete(5)
    r0, _, _, s0 = O.per_vertex(g.off, g.ind)
    h = G.from_edge_list(5, [(i, j) for i in range(5) for j in range(i + 1, 5) if (i, j) != (0, 1)])
    r1, _, _, s1 = O.per_vertex(h.off, h.ind)
    assert s1 != s0 and not np.array_equal(r0, r1)
