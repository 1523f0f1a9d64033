"""Graph file formats of the reference's input path.

* `.info` -- the CSR text file the reference's host path reads
  (readGraph, src/graphRead.cpp:2-26): the numbers "<n+1> <nnz>", then the
  n+1 offsets, then the nnz neighbour ids, whitespace separated.  The
  reference's converter writes it as one header line "<n+1>\\t<nnz>", the
  offsets tab-separated on one line and the ids tab-separated on the next
  (writeGraph, src/csrdatacreate.cpp:86-114); write_info produces the same
  bytes.
* METIS / DIMACS10 adjacency text -- optional '%' comment lines, a header
  "n m" (m undirected edges), then one line per vertex listing its 1-based
  neighbours (readGraph, src/csrdatacreate.cpp:3-47).  Only the unweighted
  format is accepted, as in the reference (its parser reads "n m" only).
  Unlike the reference's converter, read_metis removes self-loops and
  duplicate neighbours (the counting contract needs a simple graph) and
  reports how many it removed; rows are sorted ascending as in the reference.
"""
from __future__ import annotations

import os

import numpy as np

from .graphs import CSRGraph, validate_csr_host


class FormatError(ValueError):
    pass


def _ints(text: str) -> np.ndarray:
    if not text.strip():
        return np.zeros(0, np.int64)
    return np.array(text.split(), dtype=np.int64)


def read_info(path: str) -> CSRGraph:
    """Read a `.info` CSR file (give the full path, suffix included)."""
    with open(path) as f:
        vals = _ints(f.read())
    if vals.size < 2:
        raise FormatError(f"{path}: missing '<n+1> <nnz>' header")
    n1, nnz = int(vals[0]), int(vals[1])
    if n1 < 1 or nnz < 0 or vals.size != 2 + n1 + nnz:
        raise FormatError(f"{path}: expected {n1} offsets and {nnz} ids, "
                          f"found {vals.size - 2} numbers")
    off = vals[2:2 + n1].astype(np.int64)
    ind = vals[2 + n1:].astype(np.int64)
    if ind.size and (ind.min() < 0 or ind.max() >= n1 - 1 or ind.max() > np.iinfo(np.int32).max):
        raise FormatError(f"{path}: neighbour id out of range")
    return CSRGraph(off, ind.astype(np.int32), os.path.basename(path))


def read_info_base(base: str) -> CSRGraph:
    """Reference calling convention: the caller names the graph, the reader
    appends ".info" (src/graphRead.cpp:6-7)."""
    return read_info(base + ".info")


def write_info(path: str, graph: CSRGraph) -> None:
    g = graph.numpy()
    off = np.asarray(g.off, np.int64)
    ind = np.asarray(g.ind, np.int64)
    with open(path, "w") as f:
        f.write(f"{off.size}\t{ind.size}\n")
        f.write("\t".join(map(str, off.tolist())))
        f.write("\n")
        f.write("\t".join(map(str, ind.tolist())))


def read_metis(path: str, require_symmetric: bool = True) -> tuple[CSRGraph, dict]:
    """METIS adjacency file -> simple symmetric CSR (0-based, rows sorted).

    Returns the graph and {"self_loops": k, "duplicates": k} removed.
    """
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines) and lines[i].startswith("%"):
        i += 1
    if i >= len(lines):
        raise FormatError(f"{path}: no header")
    head = lines[i].split()
    if len(head) < 2:
        raise FormatError(f"{path}: header must be 'n m'")
    if len(head) > 2 and head[2] not in ("0", "000"):
        raise FormatError(f"{path}: weighted METIS format '{head[2]}' is not supported")
    n, m = int(head[0]), int(head[1])
    rows = lines[i + 1:i + 1 + n]
    rows += [""] * (n - len(rows))
    srcs, dsts = [], []
    for v, line in enumerate(rows):
        nb = _ints(line)
        if nb.size:
            if nb.min() < 1 or nb.max() > n:
                raise FormatError(f"{path}: vertex {v + 1} lists a neighbour outside 1..{n}")
            srcs.append(np.full(nb.size, v, np.int64))
            dsts.append(nb - 1)
    src = np.concatenate(srcs) if srcs else np.zeros(0, np.int64)
    dst = np.concatenate(dsts) if dsts else np.zeros(0, np.int64)
    loops = int((src == dst).sum())
    keep = src != dst
    src, dst = src[keep], dst[keep]
    key = src * n + dst
    uniq = np.unique(key)
    dups = int(key.size - uniq.size)
    row = uniq // n
    col = (uniq - row * n).astype(np.int32)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(row, minlength=n), out=off[1:])
    g = CSRGraph(off, col, os.path.basename(path))
    if require_symmetric:
        why = validate_csr_host(off, col)
        if why is not None:
            raise FormatError(f"{path}: {why} (header says m = {m})")
    return g, {"self_loops": loops, "duplicates": dups, "header_m": m}


def metis_to_info(metis_path: str, info_path: str) -> dict:
    g, stats = read_metis(metis_path)
    write_info(info_path, g)
    return stats
