"""Batched counting: every graph of a batch gets exactly what it gets alone
(oracle and single-graph gtc_count), in the concatenated layout, after
packing separate graphs, and under CUDA-graph replay."""
import math

import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import api, graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mixed_graphs():
    gs = [G.make_spec_graph(s) for s in G.batched_specs(24, 9, 256, 3000)]
    gs += [G.complete(30), G.from_edge_list(1, []), G.from_edge_list(5, []), G.wheel(40),
           G.CSRGraph(np.zeros(1, np.int64), np.zeros(0, np.int32), "n0"), G.rmat(12, 16, 3)]
    return [g.numpy() for g in gs]


def _check_against_oracle(graphs, batch, res):
    r = res.r.cpu().numpy()
    lcc = res.lcc.cpu().numpy()
    gT = res.graph_T.cpu().numpy()
    vstart = batch.vstart.cpu().numpy()
    for i, g in enumerate(graphs):
        r_ref, _, lcc_ref, total = O.per_vertex(g.off, g.ind)
        sl = slice(vstart[i], vstart[i + 1])
        assert np.array_equal(r[sl], r_ref), i
        assert np.array_equal(lcc[sl].view(np.int64), lcc_ref.view(np.int64)), i
        assert gT[i] * 6 == total, i


def test_batch_matches_oracle_and_single_graph(cuda):
    graphs = _mixed_graphs()
    batch = G.concat_graphs(graphs, cuda)
    bc = api.BatchCounter(cuda)
    for tun in (None, {"group": 4}, {"group": 32, "item_len": 64, "big_chunk": 64},
                {"labels": 2}, {"labels": 2, "group": 4, "big_chunk": 64},
                {"labels": 1, "group": 4, "big_hash_max": 8}, {"rows": 2, "group": 16}):
        res = bc.count(batch, outputs=("r", "lcc", "graph_T"), tuning=tun)
        torch.cuda.synchronize()
        _check_against_oracle(graphs, batch, res)
    # adjacency at an address that is not 16-byte aligned: the id
    # globalization takes its scalar path, with the same result
    shifted = torch.empty(batch.ind.numel() + 1, dtype=torch.int32, device=cuda)
    shifted[1:] = batch.ind
    unaligned = api.BatchCSR(batch.vstart, batch.off, shifted[1:])
    assert unaligned.ind.data_ptr() % 16 != 0
    res = bc.count(unaligned, outputs=("r", "lcc", "graph_T"))
    torch.cuda.synchronize()
    _check_against_oracle(graphs, batch, res)
    # against single-graph gtc_count on each graph
    tc = api.TriangleCounter(cuda)
    res = bc.count(batch, outputs=("r", "graph_T"))
    torch.cuda.synchronize()
    for i, g in enumerate(graphs):
        if g.n == 0:
            continue
        d = g.to(cuda)
        one = tc.count(d.off, d.ind, outputs=("r",))
        torch.cuda.synchronize()
        v0, v1 = int(batch.vstart[i]), int(batch.vstart[i + 1])
        assert torch.equal(one.r, res.r[v0:v1])
        assert one.triangles == int(res.graph_T[i])


def test_pack_equals_concat(cuda):
    graphs = _mixed_graphs()
    dev_graphs = [g.to(cuda) for g in graphs]
    bc = api.BatchCounter(cuda)
    packed = bc.pack(dev_graphs)
    ref = G.concat_graphs(graphs, cuda)
    torch.cuda.synchronize()
    assert torch.equal(packed.vstart, ref.vstart)
    assert torch.equal(packed.off, ref.off)
    assert torch.equal(packed.ind, ref.ind)
    res = bc.count(packed)
    torch.cuda.synchronize()
    _check_against_oracle(graphs, packed, res)


def test_batch_cuda_graph_replay(cuda):
    graphs = _mixed_graphs()
    batch = G.concat_graphs(graphs, cuda)
    bc = api.BatchCounter(cuda)
    out = bc.alloc_outputs(batch, ("r", "lcc", "graph_T"))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        bc.count(batch, out=out, stream=s)          # warm-up outside capture
    s.synchronize()
    want = out.graph_T.clone(), out.r.clone()
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gr, stream=s):
        bc.count(batch, out=out, stream=s)
    for _ in range(3):
        out.graph_T.fill_(-1)
        out.r.fill_(-1)
        gr.replay()
        torch.cuda.synchronize()
        assert torch.equal(out.graph_T, want[0]) and torch.equal(out.r, want[1])
    del gr


def test_batched_workload_sample(cuda):
    """The 4,096-graph workload's generator on the device, a bounded slice:
    the first 48 graphs, checked graph by graph against the oracle."""
    specs = G.batched_specs(4096, 4)[:48]
    graphs = [G.make_spec_graph(s, cuda) for s in specs]
    batch = G.concat_graphs(graphs, cuda)
    res = api.BatchCounter(cuda).count(batch)
    torch.cuda.synchronize()
    _check_against_oracle([g.numpy() for g in graphs], batch, res)


def test_batch_local_id_out_of_range_is_reported(cuda):
    """A graph-local id outside its graph's [0, n_g) is turned into an
    out-of-range id (never another graph's vertex) and reported."""
    graphs = _mixed_graphs()[:8]
    batch = G.concat_graphs(graphs, cuda)
    bc = api.BatchCounter(cuda)
    bc.count(batch)
    bc.check_status()
    bad = batch.ind.clone()
    v0 = int(batch.vstart[3])
    n3 = int(batch.vstart[4]) - v0
    bad[int(batch.off[v0]) + 1] = n3          # valid id in graph 4, not in graph 3
    bc.count(api.BatchCSR(batch.vstart, batch.off, bad))
    with pytest.raises(api.GTCError) as e:
        bc.check_status()
    assert e.value.status == 2


def test_full_batched_workload_per_vertex_equals_single_graph(cuda):
    """All 4,096 graphs of the batched workload: every per-vertex r and lcc
    of the one-launch batch equals the graph counted alone by gtc_count, and
    every per-graph T matches (the first 48 graphs are also checked against
    the oracle in test_batched_workload_sample)."""
    specs = G.batched_specs(4096, 4)
    graphs = [G.make_spec_graph(s, cuda) for s in specs]
    batch = G.concat_graphs(graphs, cuda)
    bc = api.BatchCounter(cuda)
    tc = api.TriangleCounter(cuda)
    r_one = torch.empty(batch.total_n, dtype=torch.int64, device=cuda)
    lcc_one = torch.empty(batch.total_n, dtype=torch.float64, device=cuda)
    T_one = torch.empty(len(graphs), 3, dtype=torch.int64, device=cuda)
    vstart = batch.vstart.cpu().numpy()
    for i, g in enumerate(graphs):
        sl = slice(int(vstart[i]), int(vstart[i + 1]))
        tc.count(g.off, g.ind, out=api.TriangleCounts(r=r_one[sl], t=None, lcc=lcc_one[sl],
                                                      global_counts=T_one[i]))
    torch.cuda.synchronize()
    # vertex-id labels (the library's choice for this mean degree) and
    # graph-major degree ranks
    for tun in (None, {"labels": 2, "group": 16}):
        res = bc.count(batch, outputs=("r", "lcc", "graph_T"), tuning=tun)
        bc.check_status()
        assert torch.equal(res.r, r_one), tun
        assert torch.equal(res.lcc.view(torch.int64), lcc_one.view(torch.int64)), tun
        assert torch.equal(res.graph_T, T_one[:, 0]), tun
