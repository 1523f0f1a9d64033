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
    assert len(list(autotune.candidates())) == 36


@pytest.mark.gpu
def test_autotune_picks_a_valid_tuning_with_identical_results(cuda, tmp_path):
    g = G.rmat(13, 16, 7).to(cuda)
    path = str(tmp_path / "tune.json")
    grid = {"group": (8, 32), "item_len": (256, 512), "big_chunk": (1024,)}
    best = autotune.autotune(g.off, g.ind, cache_path=path, grid=grid, reps=1)
    assert best["group"] in (8, 32) and best["item_len"] in (256, 512)
    assert json.load(open(path))   # persisted
    assert autotune.autotune(g.off, g.ind, cache_path=path, grid=grid) == best   # cached
    tc = api.TriangleCounter(cuda)
    a = tc.count(g.off, g.ind, tuning=best)
    b = tc.count(g.off, g.ind)
    torch.cuda.synchronize()
    assert torch.equal(a.r, b.r) and torch.equal(a.lcc, b.lcc)
