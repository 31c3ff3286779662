"""Parity at the configurations' full sizes, on the reference's own seeded
generators (the other GPU files cover the same semantics on smaller graphs):

* configuration 2: undirected Barabasi-Albert, n = 1,000,000, 8 edges per new
  vertex (barabasi_game_bag, outpref), weights f32-valued in [0.5, 2.0]:
  FP64 drop-in pagerank_weighted max-abs <= 1e-10 against the restatement,
  FP32-refined and FP64-Krylov L1 <= 1e-10 against the tight oracle;
* configuration 4: SBM with n = 2,000,000 in 64 blocks (p_in = 16/31249,
  p_out = 4/(63*31250)), K = 256 log-uniform seed sets: the whole batch on
  the GPU; all 256 columns certified within L1 1e-6 of the restatement by
  an FP64 residual pass, and a sample of columns compared with
  personalized_pagerank_vs of the restatement directly (L1 <= 1e-6 per
  column, the batched tolerance)."""
import math

import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu


def test_config2_weighted_barabasi_full_size(cuda_ok):
    n = 1_000_000
    f, t = O.barabasi_game_bag(n, 8, True, False, 20241203)
    assert len(f) == 7_999_992
    w = O.uniform_weights(len(f), 20241204)
    g = ig.Graph.from_edge_arrays(n, f, t, False)
    got = ig.pagerank_weighted(g, w)
    ref = O.pagerank_weighted(n, f, t, False, w)
    assert float(np.max(np.abs(got - ref))) <= 1e-10
    tight, _, _ = O.pagerank_tight(n, f, t, False, weights=w, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, False, weights=w) as dg:
        for prec in (ig.PRECISION_FP32_REFINED, ig.PRECISION_FP64_KRYLOV):
            x, st = dg.solve(ig.Options(precision=prec))
            assert np.abs(x - tight).sum() <= 1e-10, (prec, np.abs(x - tight).sum())
            assert st.error_bound <= 1e-10


def test_config4_batched_sbm_full_size(cuda_ok):
    blocks, bs = 64, 31_250
    n = blocks * bs
    pin, pout = 16 / (bs - 1), 4 / ((blocks - 1) * bs)
    pref = [[pin if i == j else pout for j in range(blocks)] for i in range(blocks)]
    f, t = O.sbm_game(pref, [bs] * blocks, False, False, False, 4)
    rng = np.random.default_rng(2024)
    K = 256
    seeds = []
    for _ in range(K):
        c = int(min(1000, max(1, math.floor(math.exp(rng.random() * math.log(1000.0))))))
        seeds.append(rng.choice(n, c, replace=False).astype(np.uint32))
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        X, iters, st = dg.ppr_batch(seeds, 0.85, 1e-8, 1000)
    assert X.shape == (n, K) and iters.max() < 1000
    # every column, certified: ||G(x) - x||_1 in FP64 bounds ||x - x*||_1 by
    # res / (1 - d), and the restatement (stop at a change < 1e-10) is within
    # d/(1-d) * 1e-10 of x*, so the L1 distance to it is at most the sum
    res = O.ppr_residuals(n, f, t, False, seeds, X)
    bound = res / 0.15 + 0.85 / 0.15 * 1e-10
    print({"cfg4_max_certified_l1": float(bound.max()), "column_iterations": int(st["column_iterations"]),
           "ms": st["ms"]})
    assert bound.max() <= 1e-6, (int(bound.argmax()), float(bound.max()))
    for k in (0, 1, 77, 255):
        r = np.zeros(n)
        for v in seeds[k]:
            r[v] += 1.0 / len(seeds[k])
        ref = O.personalized_pagerank(n, f, t, False, r, 0.85)
        assert np.abs(X[:, k].astype(np.float64) - ref).sum() <= 1e-6, k
