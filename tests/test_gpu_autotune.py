"""Autotuner: picks a configuration at least as fast as the default, keeps
results identical to the oracle, and round-trips through its cache file."""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_keeps_parity_and_caches(cuda_ok, tmp_path):
    scale = 16
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=5)
    ref = O.pagerank(n, f, t, True)
    cache = str(tmp_path / "tune.txt")
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        r = dg.autotune(batch=True, cache_path=cache)
        assert r["candidates"] > 10 and not r["from_cache"]
        assert r["best_ms"] <= r["default_ms"] * 1.0000001
        assert r["capw"] + r["shortmax"] <= 512 and r["batch_tile_width"] in (32, 64, 128)
        x, _ = dg.solve(ig.Options())
        assert np.abs(x - ref).max() <= 1e-10
        X, iters, st = dg.ppr_batch([np.array([1, 2], np.uint32), np.array([7], np.uint32)])
        assert st["tile_width"] == r["batch_tile_width"]
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        r2 = dg.autotune(batch=True, cache_path=cache)
        assert r2["from_cache"] and (r2["capw"], r2["shortmax"], r2["split"]) == (r["capw"], r["shortmax"], r["split"])
        x, _ = dg.solve(ig.Options())
        assert np.abs(x - ref).max() <= 1e-10
