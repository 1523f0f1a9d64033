"""Seeded synthetic graph generators and CSR helpers.

The reference reads DIMACS10 graphs from `.info` text files
(src/graphRead.cpp:2-26); those files are not available, so the workloads are
synthetic graphs with the shapes the benchmark names: Erdos-Renyi G(n, p),
R-MAT (a, b, c, d) and a 2D random geometric graph in Morton order.  Every
generator returns a *simple symmetric CSR*: int64 offsets of length n+1, int32
adjacency sorted ascending within each row, no self-loops, no duplicates.

All generators are written with torch tensor ops so the same code runs on the
host or on a GPU; a given (seed, device type) always yields the same graph.
This module is input plumbing only; no counting happens here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class CSRGraph:
    """A simple symmetric CSR graph (host numpy or device torch arrays)."""

    off: "np.ndarray | torch.Tensor"   # int64 [n+1]
    ind: "np.ndarray | torch.Tensor"   # int32 [nnz]
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.off.shape[0]) - 1

    @property
    def nnz(self) -> int:
        return int(self.ind.shape[0])

    @property
    def m(self) -> int:
        """Undirected edge count (nnz / 2 for a symmetric graph)."""
        return self.nnz // 2

    def numpy(self) -> "CSRGraph":
        if isinstance(self.off, np.ndarray):
            return self
        return CSRGraph(self.off.cpu().numpy(), self.ind.cpu().numpy(), self.name)

    def to(self, device) -> "CSRGraph":
        off = torch.as_tensor(self.off).to(device)
        ind = torch.as_tensor(self.ind).to(device)
        return CSRGraph(off, ind, self.name)


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def csr_from_pairs(src: torch.Tensor, dst: torch.Tensor, n: int,
                   name: str = "") -> CSRGraph:
    """Symmetric simple CSR from an undirected pair list.

    Self-loops are dropped, both directions are added, duplicates removed,
    and each row is sorted ascending (the layout the reference's converter
    produces, src/csrdatacreate.cpp:43-45, plus dedupe and loop removal).
    """
    src = src.to(torch.int64)
    dst = dst.to(torch.int64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    keys = torch.cat([src * n + dst, dst * n + src])
    keys = torch.unique(keys, sorted=True)
    row = torch.div(keys, n, rounding_mode="floor")
    col = (keys - row * n).to(torch.int32)
    counts = torch.bincount(row, minlength=n)
    off = torch.zeros(n + 1, dtype=torch.int64, device=keys.device)
    off[1:] = torch.cumsum(counts, 0)
    return CSRGraph(off, col.contiguous(), name)


def erdos_renyi(n: int, mean_degree: float, seed: int, device="cpu") -> CSRGraph:
    """Exact G(n, p) with p = mean_degree / (n - 1).

    The upper-triangle pair index space (n(n-1)/2 pairs, row-major) is walked
    with geometric skips (Batagelj & Brandes, 2005), so each pair is present
    independently with probability p.
    """
    device = torch.device(device)
    p = float(mean_degree) / (n - 1)
    total = n * (n - 1) // 2
    g = _gen(seed, device)
    expect = total * p
    chunk = int(expect + 8 * math.sqrt(expect + 1) + 64)
    log_q = math.log1p(-p)
    pos_parts = []
    last = torch.tensor(-1, dtype=torch.int64, device=device)
    while True:
        u = torch.rand(chunk, generator=g, dtype=torch.float64, device=device)
        # skip >= 1 : number of trials to the next success
        skip = torch.floor(torch.log1p(-u) / log_q).to(torch.int64) + 1
        pos = last + torch.cumsum(skip, 0)
        inside = pos < total
        pos_parts.append(pos[inside])
        if not bool(inside.all()):
            break
        last = pos[-1]
    pos = torch.cat(pos_parts)
    # row i starts at S(i) = i*n - i*(i+1)/2 in the row-major upper triangle
    i_all = torch.arange(n, dtype=torch.int64, device=device)
    starts = i_all * n - i_all * (i_all + 1) // 2
    row = torch.searchsorted(starts, pos, right=True) - 1
    col = pos - starts[row] + row + 1
    return csr_from_pairs(row, col, n, name=f"er_n{n}_d{mean_degree:g}_s{seed}")


def rmat_pairs(scale: int, n_edges: int, abcd, g: torch.Generator, device,
               chunk: int = 1 << 24):
    """R-MAT edge samples: one quadrant draw per level (Chakrabarti et al. 2004)."""
    a, b, c, _ = abcd
    t1, t2, t3 = a, a + b, a + b + c
    srcs, dsts = [], []
    done = 0
    while done < n_edges:
        k = min(chunk, n_edges - done)
        u = torch.zeros(k, dtype=torch.int64, device=device)
        v = torch.zeros(k, dtype=torch.int64, device=device)
        for _ in range(scale):
            r = torch.rand(k, generator=g, dtype=torch.float32, device=device)
            ubit = (r >= t2).to(torch.int64)
            vbit = ((r >= t1) & (r < t2)) | (r >= t3)
            u = u * 2 + ubit
            v = v * 2 + vbit.to(torch.int64)
        srcs.append(u)
        dsts.append(v)
        done += k
    return torch.cat(srcs), torch.cat(dsts)


def rmat(scale: int, edge_factor: int, seed: int, device="cpu",
         abcd=(0.57, 0.19, 0.19, 0.05), n: int | None = None) -> CSRGraph:
    """R-MAT graph: 2^scale vertices, edge_factor * 2^scale samples.

    Duplicates and self-loops are removed and the result symmetrised.  With
    `n` < 2^scale, samples with an endpoint >= n are dropped (used for the
    batched workload's non power-of-two sizes).
    """
    device = torch.device(device)
    nv = n if n is not None else (1 << scale)
    g = _gen(seed, device)
    src, dst = rmat_pairs(scale, edge_factor * nv, abcd, g, device)
    if nv != (1 << scale):
        keep = (src < nv) & (dst < nv)
        src, dst = src[keep], dst[keep]
    return csr_from_pairs(src, dst, nv, name=f"rmat_s{scale}_ef{edge_factor}_s{seed}")


def _morton2(x: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """Interleave the low 21 bits of x and y (x in even bits)."""
    def spread(v):
        v = v & 0x1FFFFF
        v = (v | (v << 32)) & 0x1F00000000FFFF
        v = (v | (v << 16)) & 0x1F0000FF0000FF
        v = (v | (v << 8)) & 0x100F00F00F00F00F
        v = (v | (v << 4)) & 0x10C30C30C30C30C3
        v = (v | (v << 2)) & 0x1249249249249249
        return v
    return spread(x) | (spread(y) << 1)


def rgg2d(n: int, mean_degree: float, seed: int, device="cpu",
          chunk: int = 1 << 21) -> CSRGraph:
    """2D random geometric graph in the unit square, Morton-relabelled.

    Radius r = sqrt(mean_degree / (pi n)); u ~ v iff |p_u - p_v|^2 < r^2.
    Vertex ids follow the Morton (Z-order) code of each point on a 2^20 grid,
    so neighbours are close in id.
    """
    device = torch.device(device)
    g = _gen(seed, device)
    pts = torch.rand((n, 2), generator=g, dtype=torch.float64, device=device)
    r = math.sqrt(mean_degree / (math.pi * n))
    q = (pts * (1 << 20)).to(torch.int64).clamp_(0, (1 << 20) - 1)
    code = _morton2(q[:, 0], q[:, 1])
    order = torch.argsort(code, stable=True)
    pts = pts[order].contiguous()                    # id = Morton rank
    cells = max(1, int(math.floor(1.0 / r)))
    cw = 1.0 / cells
    cx = (pts[:, 0] / cw).to(torch.int64).clamp_(0, cells - 1)
    cy = (pts[:, 1] / cw).to(torch.int64).clamp_(0, cells - 1)
    cid = cx * cells + cy
    by_cell = torch.argsort(cid, stable=True)
    cell_sorted = cid[by_cell]
    cell_start = torch.searchsorted(cell_sorted, torch.arange(cells * cells + 1, device=device))
    cnt = cell_start[1:] - cell_start[:-1]
    r2 = r * r
    srcs, dsts = [], []
    # half-neighbourhood: same cell (pairs i<j) and four forward cells
    offsets = [(0, 0), (1, -1), (1, 0), (1, 1), (0, 1)]
    for s in range(0, n, chunk):
        ids = torch.arange(s, min(n, s + chunk), device=device)
        px, py = cx[ids], cy[ids]
        for dx, dy in offsets:
            nx, ny = px + dx, py + dy
            ok = (nx >= 0) & (nx < cells) & (ny >= 0) & (ny < cells)
            a = ids[ok]
            tc = nx[ok] * cells + ny[ok]
            k = cnt[tc]
            if k.numel() == 0:
                continue
            rep_a = torch.repeat_interleave(a, k)
            base = torch.repeat_interleave(cell_start[tc], k)
            first = torch.cumsum(k, 0) - k
            within = torch.arange(int(k.sum()), device=device) - torch.repeat_interleave(first, k)
            b = by_cell[base + within]
            if dx == 0 and dy == 0:
                sel = rep_a < b
                rep_a, b = rep_a[sel], b[sel]
            d = pts[rep_a] - pts[b]
            close = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) < r2
            srcs.append(rep_a[close])
            dsts.append(b[close])
    src = torch.cat(srcs) if srcs else torch.zeros(0, dtype=torch.int64, device=device)
    dst = torch.cat(dsts) if dsts else torch.zeros(0, dtype=torch.int64, device=device)
    return csr_from_pairs(src, dst, n, name=f"rgg2d_n{n}_d{mean_degree:g}_s{seed}")


# ---------------------------------------------------------------- small cases

def from_edge_list(n: int, edges) -> CSRGraph:
    """CSR (host numpy) from an explicit undirected edge list."""
    if len(edges) == 0:
        off = np.zeros(n + 1, dtype=np.int64)
        return CSRGraph(off, np.zeros(0, dtype=np.int32))
    e = torch.as_tensor(np.asarray(edges, dtype=np.int64).reshape(-1, 2))
    return csr_from_pairs(e[:, 0], e[:, 1], n).numpy()


def complete(n: int) -> CSRGraph:
    return from_edge_list(n, [(i, j) for i in range(n) for j in range(i + 1, n)])


def cycle(n: int) -> CSRGraph:
    return from_edge_list(n, [(i, (i + 1) % n) for i in range(n)])


def star(n: int) -> CSRGraph:
    return from_edge_list(n, [(0, i) for i in range(1, n)])


def wheel(n: int) -> CSRGraph:
    """Hub 0 joined to a cycle on 1..n-1."""
    k = n - 1
    rim = [(1 + i, 1 + (i + 1) % k) for i in range(k)]
    return from_edge_list(n, [(0, i) for i in range(1, n)] + rim)


def disjoint_union(*graphs: CSRGraph) -> CSRGraph:
    offs, inds, base_v, base_e = [np.zeros(1, np.int64)], [], 0, 0
    for gph in graphs:
        gph = gph.numpy()
        offs.append(gph.off[1:] + base_e)
        inds.append(gph.ind + base_v)
        base_v += gph.n
        base_e += gph.nnz
    return CSRGraph(np.concatenate(offs), np.concatenate(inds).astype(np.int32)
                    if inds else np.zeros(0, np.int32))


# ------------------------------------------------------------- host checks

def validate_csr_host(off: np.ndarray, ind: np.ndarray) -> str | None:
    """Host-side check of the input contract; returns None or a reason."""
    off = np.asarray(off)
    ind = np.asarray(ind)
    n = off.shape[0] - 1
    if n < 0:
        return "offsets empty"
    if off[0] != 0 or off[-1] != ind.shape[0]:
        return "offsets do not span the adjacency array"
    deg = np.diff(off)
    if (deg < 0).any():
        return "offsets decrease"
    if ind.shape[0] == 0:
        return None
    if ind.min() < 0 or ind.max() >= n:
        return "index out of range"
    row = np.repeat(np.arange(n, dtype=np.int64), deg)
    if (row == ind).any():
        return "self-loop"
    same_row = row[1:] == row[:-1]
    if (ind[1:][same_row] <= ind[:-1][same_row]).any():
        return "row not strictly ascending"
    fwd = row * n + ind
    rev = np.sort(ind.astype(np.int64) * n + row)
    if not np.array_equal(fwd, rev):
        return "not symmetric"
    return None


def forward_stats(gph: CSRGraph) -> dict:
    """Degree-ordered work statistics of a graph (host, numpy)."""
    gph = gph.numpy()
    off, ind = gph.off, gph.ind.astype(np.int64)
    n = gph.n
    deg = np.diff(off)
    row = np.repeat(np.arange(n, dtype=np.int64), deg)
    fwd = (deg[ind] > deg[row]) | ((deg[ind] == deg[row]) & (ind > row))
    dplus = np.bincount(row[fwd], minlength=n)
    mins_und = np.minimum(deg[row], deg[ind])[row < ind]
    fr, fc = row[fwd], ind[fwd]
    return {
        "n": n, "nnz": int(gph.nnz), "m": int(gph.nnz // 2),
        "max_deg": int(deg.max()) if n else 0,
        "max_fwd_deg": int(dplus.max()) if n else 0,
        "W_min_undirected": int(mins_und.sum()),
        "W_fwd_min": int(np.minimum(dplus[fr], dplus[fc]).sum()),
        "W_fwd_merge": int((dplus[fr] + dplus[fc]).sum()),
        "probe_vtx_centric": int(dplus[fc].sum()),
    }


# ------------------------------------------------------------------ batches

def batched_specs(num_graphs: int = 4096, seed: int = 4, n_lo: int = 256,
                  n_hi: int = 262_144) -> list[dict]:
    """Parameters of the batched workload: vertex counts log-uniform in
    [n_lo, n_hi]; half the graphs Erdos-Renyi with mean degree uniform in
    [8, 32], half R-MAT (0.57, 0.19, 0.19, 0.05) with edge factor uniform in
    [8, 16]; one derived seed per graph."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), num_graphs)).astype(np.int64)
    kinds = np.array(["er"] * (num_graphs // 2) + ["rmat"] * (num_graphs - num_graphs // 2))
    rng.shuffle(kinds)
    er_deg = rng.uniform(8.0, 32.0, num_graphs)
    ef = rng.uniform(8.0, 16.0, num_graphs)
    specs = []
    for g in range(num_graphs):
        s = {"kind": str(kinds[g]), "n": int(max(n[g], 2)), "seed": int(seed) * 1_000_003 + g}
        if s["kind"] == "er":
            s["mean_degree"] = float(er_deg[g])
        else:
            s["edge_factor"] = float(ef[g])
        specs.append(s)
    return specs


def make_spec_graph(spec: dict, device="cpu") -> CSRGraph:
    n = spec["n"]
    if spec["kind"] == "er":
        return erdos_renyi(n, min(spec["mean_degree"], n - 1), spec["seed"], device)
    device = torch.device(device)
    scale = max(1, int(math.ceil(math.log2(n))))
    g = _gen(spec["seed"], device)
    src, dst = rmat_pairs(scale, int(round(spec["edge_factor"] * n)), (0.57, 0.19, 0.19, 0.05),
                          g, device)
    keep = (src < n) & (dst < n)
    return csr_from_pairs(src[keep], dst[keep], n, name=f"rmat_n{n}_s{spec['seed']}")


def concat_graphs(graphs: list[CSRGraph], device=None):
    """(vstart, off, ind) of the concatenated layout with graph-local ids."""
    from .api import BatchCSR
    device = torch.device(device) if device is not None else graphs[0].off.device
    ns = torch.tensor([0] + [g.n for g in graphs], dtype=torch.int64)
    es = torch.tensor([0] + [g.nnz for g in graphs], dtype=torch.int64)
    vstart = torch.cumsum(ns, 0).to(device)
    ebase = torch.cumsum(es, 0)
    offs = [torch.as_tensor(g.off)[:-1].to(device) + int(ebase[i]) for i, g in enumerate(graphs)]
    offs.append(torch.tensor([int(ebase[-1])], dtype=torch.int64, device=device))
    off = torch.cat(offs)
    ind = torch.cat([torch.as_tensor(g.ind).to(device) for g in graphs]) if graphs else \
        torch.zeros(0, dtype=torch.int32, device=device)
    return BatchCSR(vstart, off, ind)


def batched(num_graphs: int = 4096, seed: int = 4, device="cpu", n_lo: int = 256,
            n_hi: int = 262_144):
    """The batched workload as one BatchCSR (built graph by graph on `device`)."""
    specs = batched_specs(num_graphs, seed, n_lo, n_hi)
    graphs = [make_spec_graph(s, device) for s in specs]
    return concat_graphs(graphs, device), specs
