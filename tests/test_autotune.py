"""Autotuner: profile keys, cache round trip (CPU) and tuning on the GPU."""
import json

import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import api, autotune, graphs as G


def test_profile_buckets_and_cache_roundtrip(tmp_path):
    g = G.rmat(10, 8, 1)
    off = torch.as_tensor(g.off)
    key = autotune.degree_profile(off, g.nnz)
    assert key.startswith("n10-")
    assert autotune.degree_profile(torch.zeros(1, dtype=torch.int64), 0) == "empty"
    h = G.erdos_renyi(1 << 10, 16, 2)
    assert autotune.degree_profile(torch.as_tensor(h.off), h.nnz) != key   # skew differs
    path = str(tmp_path / "tune.json")
    autotune.save_cache(path, {"plain:x": {"tuning": {"group": 8}, "ms": 1.0}})
    assert autotune.load_cache(path)["plain:x"]["tuning"] == {"group": 8}
    # 2 x 2 x 2 x 3 x 4 x 3 combinations less the 72 with merges under rank
    # labels and the 36 with merges and 4 hash slots per member
    assert len(list(autotune.candidates())) == 180
    assert not autotune.valid({"rows": 2, "labels": 2})
    assert not autotune.valid({"rows": 2, "labels": 1, "region": 4})
    assert autotune.valid({"rows": 2, "labels": 1, "region": 2}) and autotune.valid({"rows": 1})


def test_staged_search_host_only():
    """Staged search: labels x group x region x rows first (other knobs at the
    library's choice), then item_len x big_chunk under the winner."""
    cost = lambda t: (abs(t.get("group", 32) - 16) + (0 if t.get("labels") == 2 else 5)
                      + abs(t.get("item_len", 512) - 256) / 100 + t.get("big_chunk", 2048) / 1e4)
    ms, best, timed = autotune._search(cost, autotune.DEFAULT_GRID, "staged")
    assert best == {"labels": 2, "group": 16, "region": 2, "rows": 1, "item_len": 256,
                    "big_chunk": 1024}
    # stage 1: 3 groups x (ids: 2 regions x hash + merge; ranks: 2 regions)
    assert timed == 3 * (3 + 2) + 4 * 3
    ms_g, best_g, timed_g = autotune._search(cost, autotune.DEFAULT_GRID, "grid")
    assert best_g == best and timed_g == 180
    with pytest.raises(ValueError):
        autotune._search(cost, autotune.DEFAULT_GRID, "random")


@pytest.mark.gpu
def test_autotune_picks_a_valid_tuning_with_identical_results(cuda, tmp_path):
    g = G.rmat(13, 16, 7).to(cuda)
    path = str(tmp_path / "tune.json")
    grid = {"labels": (1, 2), "group": (8, 32), "item_len": (256, 512), "big_chunk": (1024,)}
    best = autotune.autotune(g.off, g.ind, cache_path=path, grid=grid, reps=1)
    assert best["group"] in (8, 32) and best["item_len"] in (256, 512)
    assert best["labels"] in (1, 2)
    assert json.load(open(path))   # persisted
    assert autotune.autotune(g.off, g.ind, cache_path=path, grid=grid) == best   # cached
    tc = api.TriangleCounter(cuda)
    a = tc.count(g.off, g.ind, tuning=best)
    b = tc.count(g.off, g.ind)
    torch.cuda.synchronize()
    assert torch.equal(a.r, b.r) and torch.equal(a.lcc, b.lcc)


@pytest.mark.gpu
def test_autotune_batch_staged(cuda, tmp_path):
    graphs = [G.make_spec_graph(s, cuda) for s in G.batched_specs(24, 9, n_hi=16384)]
    batch = G.concat_graphs(graphs, cuda)
    bc = api.BatchCounter(cuda)
    grid = {"labels": (1, 2), "group": (8, 32), "item_len": (256,), "big_chunk": (1024, 2048)}
    best = autotune.autotune_batch(bc, batch, cache_path=str(tmp_path / "b.json"), grid=grid)
    assert best["labels"] in (1, 2) and best["group"] in (8, 32)
    assert autotune.batch_entry(batch)["candidates"] == 4 + 2
    a = bc.count(batch, tuning=best)
    b = bc.count(batch)
    torch.cuda.synchronize()
    assert torch.equal(a.graph_T, b.graph_T) and torch.equal(a.r, b.r)
