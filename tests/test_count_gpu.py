"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference's own outputs.  Integer outputs must be bit-exact; the local
clustering coefficient must be bit-identical to the host formula (tolerance
0: one correctly rounded division of exactly converted integers)."""
import math

import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import api, graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_SHAPES = [{}, {"group": 4}, {"group": 8}, {"group": 16, "region": 2}, {"group": 32, "region": 2},
           {"group": 8, "item_len": 64, "big_chunk": 128},
           {"group": 4, "big_hash_max": 8},     # block kernel's in-place search path
           {"group": 32, "item_len": 32, "big_chunk": 32, "big_hash_max": 16}]
# every launch shape with vertex-id labels (1) and degree-rank labels (2),
# the group kernel's merge form (rows 2, vertex ids implied) under the shapes
# that set the group, plus the library's own choice
TUNINGS = ([None] + [dict(t, labels=lab) for t in _SHAPES for lab in (1, 2)]
           + [dict(t, rows=2) for t in _SHAPES if "group" in t])


def _dev(off, ind, dev, off_dtype=torch.int64):
    return (torch.as_tensor(np.asarray(off)).to(dev, off_dtype),
            torch.as_tensor(np.asarray(ind, np.int32)).to(dev))


def _check(off, ind, res, r_ref=None):
    if r_ref is None:
        r_ref, t_ref, lcc_ref, total = O.per_vertex(off, ind)
    else:
        total = int(r_ref.sum())
        t_ref = r_ref // 2
        lcc_ref = O.lcc_formula(r_ref, np.diff(off))
    torch.cuda.synchronize()
    assert np.array_equal(res.r.cpu().numpy(), r_ref)
    assert np.array_equal(res.t.cpu().numpy(), t_ref)
    assert np.array_equal(res.lcc.cpu().numpy().view(np.int64), lcc_ref.view(np.int64))
    g = res.global_counts.cpu().numpy()
    assert g[2] == total and g[0] * 6 == total and g[1] * 2 == total


def test_golden_reference_cases(cuda, golden_cases):
    counter = api.TriangleCounter(cuda)
    for name, (off, ind, trine, total) in golden_cases.items():
        csum = np.concatenate([[0], np.cumsum(trine)])
        r_ref = csum[off[1:]] - csum[off[:-1]]
        for off_dtype in (torch.int64, torch.int32):
            d_off, d_ind = _dev(off, ind, cuda, off_dtype)
            for tun in TUNINGS:
                res = counter.count(d_off, d_ind, tuning=tun)
                _check(off, ind, res, r_ref)


@pytest.mark.parametrize("make", [
    lambda: G.erdos_renyi(16384, 16, 1),         # the ER config itself
    lambda: G.rmat(14, 16, 2),
    lambda: G.rmat(16, 16, 3),
    lambda: G.rgg2d(60000, 12, 3),
    lambda: G.erdos_renyi(3000, 60, 4),
])
def test_random_graphs_vs_oracle(cuda, make):
    g = make().numpy()
    r_ref, t_ref, lcc_ref, total = O.per_vertex(g.off, g.ind)
    counter = api.TriangleCounter(cuda)
    d_off, d_ind = _dev(g.off, g.ind, cuda)
    for tun in TUNINGS:
        res = counter.count(d_off, d_ind, tuning=tun)
        _check(g.off, g.ind, res, r_ref)
    res = counter.count(d_off, d_ind, mode="oriented")
    torch.cuda.synchronize()
    assert res.r is None and res.oriented_sum == O.oriented_sum(g.off, g.ind)
    assert res.total == total


def test_dense_graph_block_kernel_paths(cuda):
    """K_n exercises the block kernel (forward lists up to n-1) with both the
    shared table and the in-place search; closed form t = C(n-1, 2)."""
    n = 1500
    off = np.arange(n + 1, dtype=np.int64) * (n - 1)
    ind = np.concatenate([np.delete(np.arange(n, dtype=np.int32), i) for i in range(n)])
    d_off, d_ind = _dev(off, ind, cuda)
    counter = api.TriangleCounter(cuda)
    for tun in (None, {"big_hash_max": 64}, {"group": 4, "big_chunk": 100},
                {"labels": 1}, {"labels": 2}, {"labels": 2, "group": 4, "big_chunk": 100}):
        res = counter.count(d_off, d_ind, tuning=tun)
        torch.cuda.synchronize()
        assert (res.t.cpu().numpy() == math.comb(n - 1, 2)).all()
        assert res.triangles == math.comb(n, 3)
        assert (res.lcc.cpu().numpy() == 1.0).all()


def test_rank_labels_large_range(cuda):
    """Degree-rank labels on a graph with more than 131072 vertices ranked
    above some block-kernel apexes, so the block kernel also takes its hash
    table and in-place search paths with rank keys."""
    g = G.rgg2d(1 << 20, 14, 7).numpy()
    r_ref, t_ref, lcc_ref, total = O.per_vertex(g.off, g.ind)
    counter = api.TriangleCounter(cuda)
    d_off, d_ind = _dev(g.off, g.ind, cuda)
    for tun in ({"labels": 2, "group": 4}, {"labels": 2, "group": 4, "big_hash_max": 8},
                {"labels": 2, "group": 4, "big_chunk": 32}):
        _check(g.off, g.ind, counter.count(d_off, d_ind, tuning=tun), r_ref)


def test_rows_split_across_many_tiles(cuda):
    """Rows longer than one 2048-item placement tile get their forward lists
    assembled from parts placed in any order.  K_5000: every row spans three
    or four tiles and every forward list is long (the lowest-ranked vertex's
    holds 4,999 members), so the list sort, the rank counters and the
    vertex-id search path all see multi-part lists; t(v) = C(n-1, 2).  Wheel:
    a 20,000-entry hub row whose forward list is empty, checked against the
    oracle."""
    n = 5000
    off = np.arange(n + 1, dtype=np.int64) * (n - 1)
    ind = np.concatenate([np.delete(np.arange(n, dtype=np.int32), i) for i in range(n)])
    d_off, d_ind = _dev(off, ind, cuda)
    counter = api.TriangleCounter(cuda)
    for tun in (None, {"labels": 1}, {"labels": 2}, {"labels": 1, "big_hash_max": 4},
                {"labels": 2, "group": 4}):
        res = counter.count(d_off, d_ind, tuning=tun)
        torch.cuda.synchronize()
        assert (res.t.cpu().numpy() == math.comb(n - 1, 2)).all(), tun
        assert res.triangles == math.comb(n, 3)
    g = G.wheel(20001)
    for off_dtype in (torch.int64, torch.int32):
        d_off, d_ind = _dev(g.off, g.ind, cuda, off_dtype)
        for tun in (None, {"labels": 1}, {"labels": 2}, {"labels": 1, "big_hash_max": 4}):
            _check(g.off, g.ind, counter.count(d_off, d_ind, tuning=tun))


def test_edge_cases(cuda):
    counter = api.TriangleCounter(cuda)
    for g in (G.from_edge_list(1, []), G.from_edge_list(9, []), G.from_edge_list(4, [(0, 3)]),
              G.cycle(3), G.star(70), G.wheel(200)):
        d_off, d_ind = _dev(g.off, g.ind, cuda)
        _check(g.off, g.ind, counter.count(d_off, d_ind))
    # n = 0
    d_off = torch.zeros(1, dtype=torch.int64, device=cuda)
    d_ind = torch.zeros(0, dtype=torch.int32, device=cuda)
    res = counter.count(d_off, d_ind)
    torch.cuda.synchronize()
    assert res.r.numel() == 0 and res.triangles == 0


def test_deterministic_and_stream(cuda):
    g = G.rmat(13, 16, 8).to(cuda)
    counter = api.TriangleCounter(cuda)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        a = counter.count(g.off, g.ind, stream=s)
    s.synchronize()
    b = counter.count(g.off, g.ind)
    torch.cuda.synchronize()
    assert torch.equal(a.r, b.r) and torch.equal(a.lcc, b.lcc)


def test_subset(cuda):
    g = G.rmat(12, 16, 5).numpy()
    r_ref, _, _, _ = O.per_vertex(g.off, g.ind)
    rng = np.random.default_rng(0)
    v = np.concatenate([[0, 1, g.n - 1], rng.integers(0, g.n, 500)]).astype(np.int32)
    for off_dtype in (torch.int64, torch.int32):
        d_off, d_ind = _dev(g.off, g.ind, cuda, off_dtype)
        out = api.count_subset(d_off, d_ind, torch.as_tensor(v).to(cuda))
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), r_ref[v])


def _placement_boundary_graph():
    """2^18 + 7 vertices (the thread-per-row build's size): a ring with
    chords (degree 4, many triangles) plus centres of degree 31-34, 62-66,
    127-130 and 5,000 joined to runs of consecutive ring vertices (so each
    centre closes a triangle with every consecutive pair), and fan vertices
    with 31-33, 63-65 and 127-129 forward neighbours in a hub clique.  Rows
    straddle the 64-entry limit of the thread-per-row build, and forward
    lists straddle the group kernels' caps (32, 64, 128), in both
    labelings."""
    n = (1 << 18) + 7
    i = torch.arange(n, dtype=torch.int64)
    src = [i, i]
    dst = [(i + 1) % n, (i + 2) % n]
    # each centre is also a ring vertex (degree 4): d + 4 = 31-34, 62-66, ...
    degs = [27, 28, 29, 30, 58, 59, 60, 61, 62, 123, 124, 125, 126, 4996]
    for k, d in enumerate(degs):
        c = 20 + k
        start = 1000 + k * 9000
        nb = torch.arange(start, start + d, dtype=torch.int64)
        src.append(torch.full((d,), c, dtype=torch.int64))
        dst.append(nb)
    # a 200-vertex clique of hubs, and "fan" vertices joined to k of the hubs
    # (all of higher degree), so that their forward lists hold exactly k
    # members around the caps, each closing C(k, 2) triangles
    hubs = torch.arange(200_000, 200_200, dtype=torch.int64)
    hi, hj = torch.triu_indices(200, 200, offset=1)
    src.append(hubs[hi])
    dst.append(hubs[hj])
    for k, f in enumerate([31, 32, 33, 63, 64, 65, 127, 128, 129]):
        fan = 150_000 + 10 * k
        src.append(torch.full((f,), fan, dtype=torch.int64))
        dst.append(hubs[(torch.arange(f) * 7 + k) % 200])
    return G.csr_from_pairs(torch.cat(src), torch.cat(dst), n).numpy()


@pytest.mark.parametrize("tun", [None, {"labels": 1, "rows": 1}, {"labels": 1, "rows": 2},
                                 {"labels": 1, "rows": 2, "group": 16},
                                 {"labels": 1, "rows": 2, "group": 32}, {"labels": 2},
                                 {"labels": 2, "group": 8}])
def test_placement_and_cap_boundaries(tun, cuda):
    g = _placement_boundary_graph()
    deg = np.diff(g.off)
    assert {63, 64, 65, 5000} <= set(deg.tolist())
    r_ref, t_ref, lcc_ref, total = O.per_vertex(g.off, g.ind)
    for off_dtype in (torch.int32, torch.int64):
        d_off, d_ind = _dev(g.off, g.ind, cuda, off_dtype)
        res = api.TriangleCounter(cuda).count(d_off, d_ind, tuning=tun)
        torch.cuda.synchronize()
        assert np.array_equal(res.r.cpu().numpy(), r_ref), (tun, off_dtype)
        assert np.array_equal(res.lcc.cpu().numpy().view(np.int64), lcc_ref.view(np.int64))
        assert res.total == total


def _wide_hub_graph():
    """Two hubs of degree 2,600: hub 0's neighbours spread over 2^21 + 7
    ids (beyond the hub kernel's bitmap span, so its rows are binary
    searched), hub 1's packed into 2,600 consecutive ids (bitmap); the
    neighbours are joined in a path, so both hubs close many triangles, and
    hub 0's neighbours share a few with hub 1."""
    n = (1 << 21) + 7
    spread = np.unique(np.linspace(2, n - 1, 2600).astype(np.int64))
    packed = np.arange(10, 10 + 2600, dtype=np.int64)
    edges = [(0, int(x)) for x in spread] + [(1, int(x)) for x in packed]
    edges += [(int(a), int(b)) for a, b in zip(spread[:-1], spread[1:])]
    edges += [(int(a), int(b)) for a, b in zip(packed[:-1:2], packed[1::2])]
    edges += [(0, 1)]
    return G.from_edge_list(n, sorted({(min(a, b), max(a, b)) for a, b in edges if a != b}))


@pytest.mark.parametrize("which", ["rmat", "wide"])
def test_subset_hub_rows(which, cuda):
    """Listed rows longer than the hash table (the hub kernel, a whole GPU
    per hub), listed several times and spread over several 1,024-vertex
    scan chunks, beside ordinary rows; the int32 vertex-list shim as well."""
    if which == "rmat":
        g = G.rmat(16, 16, 7).numpy()
    else:
        g = _wide_hub_graph()
    deg = np.diff(g.off)
    hubs = np.nonzero(deg > 2048)[0]
    assert hubs.size >= 2
    rng = np.random.default_rng(3)
    v = np.concatenate([hubs, rng.integers(0, g.n, 3000), hubs[::-1], [hubs[0]] * 3])
    v = v[rng.permutation(v.size)].astype(np.int32)
    ref = O.subset(g.off, g.ind, v)
    assert ref[np.isin(v, hubs)].min() > 0
    for off_dtype in (torch.int64, torch.int32):
        d_off, d_ind = _dev(g.off, g.ind, cuda, off_dtype)
        out = api.count_subset(d_off, d_ind, torch.as_tensor(v).to(cuda))
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref), off_dtype
    d_off = torch.as_tensor(g.off).to(cuda, torch.int32)
    d_ind = torch.as_tensor(g.ind).to(cuda, torch.int32)
    d_v = torch.as_tensor(v).to(cuda)
    vout = torch.full((v.size,), -1, dtype=torch.int32, device=cuda)
    api.kernelCall(4, 128, v.size, d_off, d_ind, vout, 1, 128, 0, vertex=d_v)
    torch.cuda.synchronize()
    assert np.array_equal(vout.cpu().numpy().astype(np.int64), ref)


@pytest.mark.parametrize("which", ["rmat", "er"])
def test_compat_kernelCall(which, cuda):
    """The reference's kernelCall argument list (src/gpurun.cu:31-37).  The
    R-MAT graph has a low mean degree but a high skew (the shims switch it to
    degree-rank labels); the ER graph keeps vertex-id labels."""
    g = (G.rmat(12, 12, 6) if which == "rmat" else G.erdos_renyi(3000, 10, 4)).numpy()
    r_ref, _, _, _ = O.per_vertex(g.off, g.ind)
    for dt in (torch.int64, torch.int32):
        d_off = torch.as_tensor(g.off).to(cuda, dt)
        d_ind = torch.as_tensor(g.ind).to(cuda, dt)
        out = torch.full((g.n,), -1, dtype=dt, device=cuda)
        for bs, tpi in ((256, 1), (32, 32), (96, 4), (1024, 2)):
            out.fill_(-1)
            api.kernelCall(g.n, bs, g.n, d_off, d_ind, out, tpi, bs // tpi, int(math.log2(tpi)))
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy().astype(np.int64), r_ref)
        # vertex-list overload
        v = torch.as_tensor(np.arange(0, g.n, 7)).to(cuda, dt)
        vout = torch.zeros(v.numel(), dtype=dt, device=cuda)
        api.kernelCall(4, 128, v.numel(), d_off, d_ind, vout, 1, 128, 0, vertex=v)
        torch.cuda.synchronize()
        assert np.array_equal(vout.cpu().numpy().astype(np.int64), r_ref[::7])
        # unsupported block size: nothing launched, error reported
        out.fill_(-1)
        with pytest.raises(api.GTCError):
            api.kernelCall(g.n, 100, g.n, d_off, d_ind, out, 1, 100, 0)
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == -1).all()


@pytest.mark.parametrize("defect,reason", [
    ("ok", 0), ("offsets", 1), ("range", 2), ("selfloop", 3), ("unsorted", 4), ("asym", 5),
    ("asym_lower", 5), ("ok_rmat", 0)])
def test_validate_csr(cuda, defect, reason):
    g = G.complete(6).numpy()
    off, ind = g.off.copy(), g.ind.copy()
    if defect == "offsets":
        off[3] = off[4] + 1
    elif defect == "range":
        ind[2] = 60
    elif defect == "selfloop":
        ind[0] = 0
    elif defect == "unsorted":
        ind[0], ind[1] = ind[1], ind[0]
    elif defect == "asym":
        off = np.array([0, 1, 2, 3], np.int64); ind = np.array([1, 2, 0], np.int32)
    elif defect == "asym_lower":
        # every entry (a, x) with a < x has its reverse; the extra (2, 0) has
        # none, which only the count of such entries reveals
        off = np.array([0, 1, 2, 3], np.int64); ind = np.array([1, 0, 0], np.int32)
    elif defect == "ok_rmat":
        h = G.rmat(14, 16, 9).numpy()
        off, ind = np.asarray(h.off, np.int64), np.asarray(h.ind, np.int32)
    for off_dtype in (torch.int64, torch.int32):
        d_off, d_ind = _dev(off, ind, cuda, off_dtype)
        assert api.validate_csr(d_off, d_ind)[0] == reason


@pytest.mark.skipif(not O.ref_gpu_available(), reason="reference GPU kernel not built")
def test_reference_gpu_kernel_parity(cuda):
    """Second oracle: the reference's own kernel (tpi = 1) on the same input."""
    lib = O.ref_gpu_lib()
    for g in (G.rmat(13, 16, 2), G.erdos_renyi(16384, 16, 1), G.rgg2d(30000, 12, 3)):
        gd = g.to(cuda)
        off64 = gd.off.to(torch.int64)
        pad = 8
        ind64 = torch.zeros(g.nnz + 2 * pad, dtype=torch.int64, device=cuda)
        ind64[pad:pad + g.nnz] = gd.ind.to(torch.int64)
        ref_out = torch.zeros(g.n, dtype=torch.int64, device=cuda)
        torch.cuda.synchronize()
        assert lib.ref_gpu_count_i64(1024, 256, g.n, off64.data_ptr(),
                                     ind64[pad:].data_ptr(), ref_out.data_ptr()) == 0
        res = api.count_triangles(gd.off, gd.ind)
        torch.cuda.synchronize()
        assert torch.equal(res.r, ref_out)


def test_out_of_range_ids_are_reported_not_dereferenced(cuda):
    """A neighbour id outside [0, n) is never dereferenced: the kernels skip
    it and gtc_count_status reports GTC_ERR_INVALID_CSR.  The bad ids sit in
    the largest row (a block-kernel apex) and in a low-degree row (warp
    kernel), under both labelings; a valid count on the same workspace then
    reports OK again (each count clears the status word)."""
    g = G.rmat(12, 16, 3).numpy()
    counter = api.TriangleCounter(cuda)
    d_off, d_ind = _dev(g.off, g.ind, cuda)
    counter.count(d_off, d_ind)
    counter.check_status()
    deg = np.diff(g.off)
    hub = int(np.argmax(deg))
    low = int(np.argmin(np.where(deg >= 2, deg, 1 << 30)))
    for bad in (g.n, g.n + 12345, -1, -(1 << 31), (1 << 31) - 1):
        ind = g.ind.copy()
        ind[g.off[hub] + deg[hub] // 2] = bad
        ind[g.off[low] + 1] = bad
        bad_ind = torch.from_numpy(ind).to(cuda)
        for tun in (None, {"labels": 1}, {"labels": 2}, {"group": 4, "big_hash_max": 8}):
            counter.count(d_off, bad_ind, tuning=tun)
            with pytest.raises(api.GTCError) as e:
                counter.check_status()
            assert e.value.status == 2
        counter.count(d_off, bad_ind, mode="oriented")
        with pytest.raises(api.GTCError):
            counter.check_status()
    res = counter.count(d_off, d_ind)
    counter.check_status()
    _check(g.off, g.ind, res)


def test_compat_wide_id_is_reported(cuda):
    """kernelCall<int64_t> with an id that does not fit the graph (2^32 + 3
    would wrap to 3 if narrowed blindly) reports GTC_ERR_INVALID_CSR through
    gtc_compat_last_status instead of counting a wrapped id."""
    g = G.wheel(30).numpy()
    off = torch.from_numpy(g.off).to(cuda)
    ind = torch.from_numpy(g.ind.astype(np.int64)).to(cuda)
    out = torch.zeros(g.n, dtype=torch.int64, device=cuda)
    api.kernelCall(1, 256, g.n, off, ind, out, 1, 256, 0)
    torch.cuda.synchronize()
    r_ref, _, _, _ = O.per_vertex(g.off, g.ind)
    assert np.array_equal(out.cpu().numpy(), r_ref)
    ind[4] = (1 << 32) + 3
    with pytest.raises(api.GTCError) as e:
        api.kernelCall(1, 256, g.n, off, ind, out, 1, 256, 0)
    assert e.value.status == 2
