"""Input formats against the reference's own converter and reader (compiled
from its sources into oracle/_ref).  CPU only."""
import os

import numpy as np
import pytest

from gputrianglecounting_b200 import formats, graphs as G
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_formats_available(),
                               reason="reference formats not built (make -C oracle ref)")


def write_metis(path, g, comment=True, extra=None):
    g = g.numpy()
    with open(path, "w") as f:
        if comment:
            f.write("% generated for a format test\n")
        f.write(f"{g.n} {g.nnz // 2}\n")
        for v in range(g.n):
            nb = list(g.ind[g.off[v]:g.off[v + 1]] + 1)
            if extra and v in extra:
                nb += extra[v]
            f.write(" ".join(map(str, nb)) + "\n")


@needs_ref
@pytest.mark.parametrize("make", [lambda: G.rmat(9, 8, 3), lambda: G.wheel(12),
                                  lambda: G.disjoint_union(G.complete(5), G.from_edge_list(4, []))])
def test_writer_matches_reference_converter_bytes(tmp_path, make):
    g = make().numpy()
    metis = str(tmp_path / "g.graph")
    write_metis(metis, g, comment=True)
    ref_info = str(tmp_path / "ref.info")
    O.ref_metis_to_info(metis, ref_info)
    mine = formats.read_metis(metis)[0]
    assert np.array_equal(mine.off, g.off) and np.array_equal(mine.ind, g.ind)
    my_info = str(tmp_path / "mine.info")
    formats.write_info(my_info, mine)
    assert open(my_info).read() == open(ref_info).read()


@needs_ref
def test_reader_matches_reference_reader(tmp_path):
    g = G.rmat(10, 8, 5).numpy()
    base = str(tmp_path / "graph")
    formats.write_info(base + ".info", g)
    off, ind = O.ref_read_info(base, g.n, g.nnz)
    mine = formats.read_info_base(base)
    assert np.array_equal(off, mine.off) and np.array_equal(ind, mine.ind)
    assert np.array_equal(mine.off, g.off) and np.array_equal(mine.ind, g.ind)


def test_metis_cleanup_comments_loops_duplicates(tmp_path):
    g = G.wheel(8).numpy()
    path = str(tmp_path / "w.graph")
    # vertex 0 lists itself and a duplicate of neighbour 2 (1-based ids)
    write_metis(path, g, comment=True, extra={0: [1, 2]})
    h, stats = formats.read_metis(path)
    assert stats == {"self_loops": 1, "duplicates": 1, "header_m": g.nnz // 2}
    assert np.array_equal(h.off, g.off) and np.array_equal(h.ind, g.ind)


def test_format_errors(tmp_path):
    p = str(tmp_path / "bad.graph")
    open(p, "w").write("3 2 1\n2\n1\n\n")
    with pytest.raises(formats.FormatError, match="weighted"):
        formats.read_metis(p)
    open(p, "w").write("3 1\n2\n\n\n")           # 1 -> 2 without 2 -> 1
    with pytest.raises(formats.FormatError, match="symmetric"):
        formats.read_metis(p)
    q = str(tmp_path / "bad.info")
    open(q, "w").write("4\t3\n0\t1\t2\n1\t0")
    with pytest.raises(formats.FormatError):
        formats.read_info(q)


def test_roundtrip_and_count_input(tmp_path):
    from oracle import oracle as Or
    g = G.erdos_renyi(500, 10, 7).numpy()
    path = str(tmp_path / "er.info")
    formats.write_info(path, g)
    h = formats.read_info(path)
    r1, _, _, s1 = Or.per_vertex(g.off, g.ind)
    r2, _, _, s2 = Or.per_vertex(h.off, h.ind)
    assert s1 == s2 and np.array_equal(r1, r2)
