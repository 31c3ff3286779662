"""Batched personalized PageRank (FP32 SpMM, per-column freeze; Chebyshev
steps on undirected graphs) against the oracle's FP64 personalized_pagerank
on every column.

Tolerance: each column stops at a successive L1 change < 1e-8, so its
error is <= 1e-8 * d/(1-d) ~ 5.7e-8 from the stop rule plus FP32 rounding
(about 1e-7 of the vector's L1 mass); the test allows L1 <= 1e-6 per column.
"""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu
TOL_COL = 1e-8
L1_COL = 1e-6


def seed_sets(n, K, rng, max_seeds=60):
    out = []
    for _ in range(K):
        c = int(np.clip(np.floor(np.exp(rng.random() * np.log(max_seeds))), 1, max_seeds))
        out.append(rng.choice(n, size=c, replace=False).astype(np.uint32))
    out[0] = np.array([3, 3, 7], np.uint32)  # duplicates add weight, like _vs
    return out


def reset_of(n, seeds):
    r = np.zeros(n)
    for v in seeds:
        r[v] += 1.0 / len(seeds)
    return r


@pytest.mark.parametrize("vec", [1, 2, 4])
def test_batch_matches_oracle_sbm(cuda_ok, vec):
    sizes = [1250] * 16
    n = sum(sizes)
    pin, pout = 16 / 1249, 4 / (15 * 1250)
    pref = [[pin if i == j else pout for j in range(16)] for i in range(16)]
    f, t = O.sbm_game(pref, sizes, False, False, False, 9)
    rng = np.random.default_rng(17)
    K = 40  # not a multiple of the tile width: exercises a partial tile
    seeds = seed_sets(n, K, rng)
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        X, iters, st = dg.ppr_batch(seeds, 0.85, TOL_COL, 1000, vec)
    assert st["tile_width"] == 32 * vec and X.shape == (n, K)
    for k in range(K):
        ref = O.personalized_pagerank(n, f, t, False, reset_of(n, seeds[k]), 0.85)
        err = np.abs(X[:, k].astype(np.float64) - ref).sum()
        assert err <= L1_COL, (k, err, iters[k])
        assert abs(X[:, k].sum() - 1) < 1e-5
    assert iters.min() >= 5 and iters.max() < 1000


def test_chebyshev_steps_on_undirected_graphs(cuda_ok):
    # With batch_cheb = 1, undirected graphs take Chebyshev steps between the
    # reference's stop tests; batch_cheb = 0 (the default) gives the plain
    # power steps.  Both meet the oracle on every column, the Chebyshev
    # columns in fewer iterations, and directed graphs never take them.
    blocks, bs = 32, 1500
    n = blocks * bs
    pin, pout = 16 / (bs - 1), 4 / ((blocks - 1) * bs)
    pref = [[pin if i == j else pout for j in range(blocks)] for i in range(blocks)]
    f, t = O.sbm_game(pref, [bs] * blocks, False, False, False, 12)
    rng = np.random.default_rng(23)
    seeds = seed_sets(n, 48, rng, max_seeds=300)
    out = {}
    try:
        for cheb in (1, 0):
            ig.set_tuning("batch_cheb", cheb)
            with ig.DeviceGraph.from_host(n, f, t, False) as dg:
                out[cheb] = dg.ppr_batch(seeds, 0.85, TOL_COL, 1000)
    finally:
        ig.reset_tuning()
    assert out[1][2]["chebyshev"] and not out[0][2]["chebyshev"]
    for k in range(len(seeds)):
        ref = O.personalized_pagerank(n, f, t, False, reset_of(n, seeds[k]), 0.85)
        for cheb in (1, 0):
            err = np.abs(out[cheb][0][:, k].astype(np.float64) - ref).sum()
            assert err <= L1_COL, (cheb, k, err)
    it_cheb, it_plain = out[1][1].astype(np.int64), out[0][1].astype(np.int64)
    print({"chebyshev_column_iterations": int(it_cheb.sum()), "plain_column_iterations": int(it_plain.sum())})
    assert it_cheb.sum() < 0.8 * it_plain.sum(), (it_cheb.sum(), it_plain.sum())
    ff, tt = O.erdos_renyi_gnm(3000, 20_000, True, False, 4)
    ig.set_tuning("batch_cheb", 1)
    try:
        with ig.DeviceGraph.from_host(3000, ff, tt, True) as dg:
            _, _, st = dg.ppr_batch([np.array([1, 2], np.uint32)], 0.85, TOL_COL, 1000)
    finally:
        ig.reset_tuning()
    assert not st["chebyshev"]


def test_batch_relabelled_directed_with_dangling(cuda_ok):
    n = 12_000
    f, t = O.barabasi_game_bag(n, 4, False, True, 2)  # directed BA: vertex 0 dangling, skewed degrees
    rng = np.random.default_rng(3)
    seeds = seed_sets(n, 33, rng)
    ig.set_tuning("relabel", 1)
    try:
        with ig.DeviceGraph.from_host(n, f, t, True) as dg:
            assert dg.relabelled
            X, iters, st = dg.ppr_batch(seeds, 0.85, TOL_COL, 1000)
    finally:
        ig.reset_tuning()
    for k in range(len(seeds)):
        ref = O.personalized_pagerank(n, f, t, True, reset_of(n, seeds[k]), 0.85)
        assert np.abs(X[:, k].astype(np.float64) - ref).sum() <= L1_COL, k


def test_batch_columns_freeze_independently(cuda_ok):
    # a column whose reset sits on an isolated vertex converges at once; the
    # others keep iterating, and the frozen column keeps its value
    n = 5000
    f, t = O.erdos_renyi_gnm(n - 1, 30_000, False, False, 5)
    seeds = [np.array([n - 1], np.uint32), np.array([0, 1, 2], np.uint32)]
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        X, iters, _ = dg.ppr_batch(seeds, 0.85, TOL_COL, 1000)
    assert iters[0] <= 2 < iters[1]
    assert abs(X[n - 1, 0] - 1.0) < 1e-6
    ref = O.personalized_pagerank(n, f, t, False, reset_of(n, seeds[1]), 0.85)
    assert np.abs(X[:, 1] - ref).sum() <= L1_COL


def test_batch_validation(cuda_ok):
    f, t = O.erdos_renyi_gnm(100, 300, True, False, 1)
    with ig.DeviceGraph.from_host(100, f, t, True) as dg:
        with pytest.raises(ig.InvalidArgument, match="reset_vids must not be empty"):
            dg.ppr_batch([np.array([1], np.uint32), np.array([], np.uint32)])
        with pytest.raises(ig.InvalidArgument, match=r"reset vertex 100 out of range \(vcount = 100\)"):
            dg.ppr_batch([np.array([100], np.uint32)])
        with pytest.raises(ig.InvalidArgument, match="damping"):
            dg.ppr_batch([np.array([1], np.uint32)], damping=1.0)


def test_barrier_timeout_is_reported_and_the_context_survives(cuda_ok):
    # Failure detection without a fault: the test hook makes every grid
    # barrier of the persistent batched kernel wait for one arrival that never
    # comes.  The barrier's bounded wait (about 1.5 s) expires, the kernel
    # records PRG_ERR_TIMEOUT and every block returns; the host raises, and
    # the next call on the same graph and context succeeds.
    n = 3000
    f, t = O.barabasi_game_bag(n, 3, False, False, 5)
    seeds = [np.array([1, 2, 3], np.uint32)]
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        ig.set_tuning("batch_barrier_extra", 1)
        try:
            with pytest.raises(ig.DeviceTimeout, match="grid barrier timed out"):
                dg.ppr_batch(seeds, 0.85, TOL_COL, 1000, 1)
        finally:
            ig.reset_tuning()
        X, iters, st = dg.ppr_batch(seeds, 0.85, TOL_COL, 1000, 1)
    ref = O.personalized_pagerank(n, f, t, False, reset_of(n, seeds[0]), 0.85)
    assert np.abs(X[:, 0].astype(np.float64) - ref).sum() <= L1_COL
