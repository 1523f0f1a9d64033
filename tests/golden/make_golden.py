"""Generate tests/golden/reference_cases.npz from the reference itself.

Runs the reference's own count_all_trianglesCPU (src/clusteringCount.cpp:50-70),
compiled unchanged from its sources by `make -C oracle ref`, on small seeded
graphs and stores, per case: the CSR (off, ind), the reference's per-edge
triNE and its total.  The reference ships no golden vectors or fixtures, so
these outputs of the reference are the pinned values the oracle and the CUDA
path are checked against.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gputrianglecounting_b200 import graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    yield "er_n300_d8_s11", G.erdos_renyi(300, 8, 11)
    yield "er_n2000_d16_s1", G.erdos_renyi(2000, 16, 1)
    yield "rmat_s9_ef8_s12", G.rmat(9, 8, 12)
    yield "rmat_s11_ef16_s2", G.rmat(11, 16, 2)
    yield "rgg_n1500_d12_s13", G.rgg2d(1500, 12, 13)
    yield "complete_12", G.complete(12)
    yield "wheel_17", G.wheel(17)
    yield "star_40", G.star(40)
    yield "cycle_3", G.cycle(3)
    yield "cycle_10", G.cycle(10)
    yield "union_k5_c4_w8", G.disjoint_union(G.complete(5), G.cycle(4), G.wheel(8))
    yield "isolated_10", G.from_edge_list(10, [])
    yield "single_edge_plus_isolated", G.from_edge_list(6, [(1, 4)])
    yield "isolated_then_k4", G.disjoint_union(G.from_edge_list(100, []), G.complete(4))


def main():
    out = {}
    for name, g in cases():
        g = g.numpy()
        err = G.validate_csr_host(g.off, g.ind)
        assert err is None, (name, err)
        tri, total = O.ref_tri_ne(g.off, g.ind)
        out[f"{name}__off"] = g.off.astype(np.int64)
        out[f"{name}__ind"] = g.ind.astype(np.int32)
        out[f"{name}__trine"] = tri.astype(np.int64)
        out[f"{name}__total"] = np.array([total], np.int64)
        print(f"{name:28s} n={g.n:6d} nnz={g.nnz:8d} total={total}")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
