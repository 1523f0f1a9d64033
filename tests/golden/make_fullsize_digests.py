"""Generate tests/golden/fullsize_digests.json from the reference itself.

The two large single-graph workloads -- R-MAT scale 20 (edge factor 16,
(0.57, 0.19, 0.19, 0.05), seed 2) and the 2D random geometric graph
(n = 4,194,304, mean degree 12, Morton order, seed 3) -- are generated on the
host by gputrianglecounting_b200.graphs, exactly as the tests generate them.
For every vertex the reference's own count_all_trianglesCPU (vertex-list
overload, src/clusteringCount.cpp:125-155, compiled unchanged by
`make -C oracle ref`) gives triNE, whose row sum is r(v), the value the
reference kernel stores in out[v] (src/clusteringCount.cu:314-359).  The
arrays are too large to commit, so the file holds SHA-256 digests of the
little-endian bytes of

  * the CSR itself (int64 offsets, int32 ids), to pin the generated graph;
  * r (int64), t = r / 2 (int64) and lcc = r / (d (d - 1)) (float64, 0 for
    d < 2, one IEEE division of exactly converted integers),

plus n, nnz and T = sum(r) / 6.  The C restatement (oracle/tc_oracle.c) is
checked against the same arrays before anything is written.

    make -C oracle oracle ref && python tests/golden/make_fullsize_digests.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gputrianglecounting_b200 import graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fullsize_digests.json")


def sha256(a: np.ndarray, dtype: str) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


WORKLOADS = {
    "rmat20": ("R-MAT scale 20, edge factor 16, (0.57,0.19,0.19,0.05), seed 2",
               lambda: G.rmat(20, 16, 2)),
    "rgg4m": ("2D RGG n=4194304, mean degree 12, Morton order, seed 3",
              lambda: G.rgg2d(1 << 22, 12, 3)),
}


def digests(off, ind, r) -> dict:
    deg = np.diff(off.astype(np.int64))
    lcc = O.lcc_formula(r, deg)
    return {"r_sha256": sha256(r, "<i8"), "t_sha256": sha256(r // 2, "<i8"),
            "lcc_sha256": sha256(lcc, "<f8")}


def main():
    out = {}
    for name, (label, make) in WORKLOADS.items():
        t0 = time.time()
        g = make().numpy()
        n = g.n
        r, total = O.ref_all_rows_i32(g.off.astype(np.int32), g.ind)
        assert total == int(r.sum()) and total % 6 == 0 and not (r % 2).any()
        r_or, t_or, lcc_or, total_or = O.per_vertex(g.off, g.ind)
        assert np.array_equal(r_or, r) and total_or == total, name
        d = digests(g.off, g.ind, r)
        assert d["lcc_sha256"] == sha256(lcc_or, "<f8"), name
        out[name] = {
            "graph": label,
            "n": n, "nnz": g.nnz, "T": total // 6,
            "off_sha256": sha256(g.off, "<i8"), "ind_sha256": sha256(g.ind, "<i4"),
            **d,
        }
        print(f"{name}: n={n} nnz={g.nnz} T={total // 6} ({time.time() - t0:.1f} s)", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
