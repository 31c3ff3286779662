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
        # the segmented passes' hot prefixes (a degree-sorted unweighted graph)
        assert r["seg_hot"] in (24576, 32768, 40960) and r["seg_hot64"] in (4096, 8192, 12288)
        assert 0 < r["seg_best_ms"] <= r["seg_default_ms"]
        xr, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
        assert st.error_bound <= 1e-10
        x, _ = dg.solve(ig.Options())
        assert np.abs(x - ref).max() <= 1e-10
        X, iters, st = dg.ppr_batch([np.array([1, 2], np.uint32), np.array([7], np.uint32)])
        assert st["tile_width"] == r["batch_tile_width"]
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        r2 = dg.autotune(batch=True, cache_path=cache)
        assert r2["from_cache"] and (r2["capw"], r2["shortmax"], r2["split"]) == (r["capw"], r["shortmax"], r["split"])
        assert (r2["seg_hot"], r2["seg_hot64"]) == (r["seg_hot"], r["seg_hot64"])
        x, _ = dg.solve(ig.Options())
        assert np.abs(x - ref).max() <= 1e-10
