"""GPU eigenvector centrality and HITS (prg_eigenvector_centrality,
prg_hub_and_authority_scores) against the CPU restatements of the reference's
power iterations (eigenvector.rs:286-372, hits.rs:122-230).

The GPU sums each row in CSR order and the reference in ascending neighbour
order, so the iterates differ by rounding and a stop may come one iteration
apart; both stop at an L1 change below 1e-14 (eigenvector) / 1e-12 (HITS), so
the vectors agree to well under 1e-10 max-abs and the eigenvalues to 1e-10
relative."""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def G(n, pairs, directed):
    a = np.array(pairs, np.uint32).reshape(-1, 2)
    return ig.Graph.from_edge_arrays(n, a[:, 0], a[:, 1], directed)


def edges(g):
    f, t = g.edge_arrays()
    return f, t


def test_reference_unit_cases(cuda_ok):
    # eigenvector.rs:770-829
    assert len(ig.eigenvector_centrality(ig.Graph.with_vertices(0))) == 0
    assert list(ig.eigenvector_centrality(ig.Graph.with_vertices(1))) == [1.0]
    assert np.allclose(ig.eigenvector_centrality(ig.Graph.with_vertices(3)), 1.0, atol=1e-9)
    assert np.allclose(ig.eigenvector_centrality(G(3, [(0, 1), (1, 2), (2, 0)], False)), 1.0, atol=1e-9)
    x = ig.eigenvector_centrality(G(4, [(0, 1), (0, 2), (0, 3)], False))
    assert np.allclose(x, [1.0] + [1 / np.sqrt(3)] * 3, atol=1e-9)
    k4 = [(u, v) for u in range(4) for v in range(u + 1, 4)]
    assert np.allclose(ig.eigenvector_centrality(G(4, k4, False)), 1.0, atol=1e-9)
    with pytest.raises(ig.Unsupported, match="directed eigenvector_centrality"):
        ig.eigenvector_centrality(G(3, [(0, 1)], True))
    # hits.rs:627-730
    s = ig.hub_and_authority_scores(G(3, [], True))
    assert np.all(s.hub == 1) and np.all(s.authority == 1) and s.eigenvalue == 0.0
    assert abs(ig.hub_and_authority_scores(G(2, [(0, 1)], True)).eigenvalue - 1.0) < 1e-6
    s = ig.hub_and_authority_scores(G(4, [(0, 2), (0, 3), (1, 2), (1, 3)], True))
    assert np.allclose(s.hub, [1, 1, 0, 0], atol=1e-9) and np.allclose(s.authority, [0, 0, 1, 1], atol=1e-9)
    assert abs(s.eigenvalue - 4.0) < 1e-6
    s = ig.hub_and_authority_scores(G(3, [(0, 2), (1, 2)], True))
    assert abs(s.hub[2]) < 1e-9 and abs(s.authority[2] - 1) < 1e-9
    s = ig.hub_and_authority_scores(G(1, [(0, 0)], False))  # one vertex, one loop: lambda = 2
    assert list(s.hub) == [1.0] and s.eigenvalue == 4.0


def _compare_eig(n, f, t):
    g = ig.Graph.from_edge_arrays(n, f, t, False)
    x, lam = ig.eigenvector_centrality(g, with_eigenvalue=True)
    gf, gt = edges(g)
    ref, rlam, _ = O.eigenvector_centrality(n, gf, gt)
    assert np.max(np.abs(x - ref)) <= TOL, np.max(np.abs(x - ref))
    assert abs(lam - rlam) <= TOL * abs(rlam)
    return g


@pytest.mark.parametrize("kind", ["er", "ba", "rmat", "loops"])
def test_eigenvector_matches_restatement(cuda_ok, kind):
    if kind == "er":
        n = 20_000
        f, t = O.erdos_renyi_gnm(n, 100_000, False, False, 3)
    elif kind == "ba":
        n = 30_000
        f, t = O.barabasi_game_bag(n, 4, False, False, 8)
    elif kind == "rmat":
        n = 1 << 15
        f, t = O.rmat(15, 8 * n, seed=4)
    else:
        rng = np.random.default_rng(2)
        n = 5000
        f = rng.integers(0, n, 30_000).astype(np.uint32)
        t = rng.integers(0, n, 30_000).astype(np.uint32)
        f[:200] = t[:200] = 7  # loops, counted twice
    _compare_eig(n, f, t)


@pytest.mark.parametrize("kind", ["rmat", "ba"])
def test_hits_directed_matches_restatement(cuda_ok, kind):
    if kind == "rmat":
        n = 1 << 15
        f, t = O.rmat(15, 8 * n, seed=6)
    else:
        n = 20_000
        f, t = O.barabasi_game_bag(n, 3, False, True, 9)
    g = ig.Graph.from_edge_arrays(n, f, t, True)
    s = ig.hub_and_authority_scores(g)
    h, a, lam, _ = O.hub_and_authority_scores(n, f, t, True)
    assert np.max(np.abs(s.hub - h)) <= TOL and np.max(np.abs(s.authority - a)) <= TOL
    assert abs(s.eigenvalue - lam) <= TOL * abs(lam)
    assert s.hub.max() == 1.0 and s.authority.max() == 1.0 and s.hub.min() >= 0.0


def test_hits_undirected_delegates(cuda_ok):
    n = 10_000
    f, t = O.erdos_renyi_gnm(n, 40_000, False, False, 12)
    g = ig.Graph.from_edge_arrays(n, f, t, False)
    s = ig.hub_and_authority_scores(g)
    x, lam = ig.eigenvector_centrality(g, with_eigenvalue=True)
    assert np.array_equal(s.hub, x) and np.array_equal(s.authority, x)
    assert abs(s.eigenvalue - lam * lam) <= 1e-12 * lam * lam


def test_weighted_reference_unit_cases(cuda_ok):
    # eigenvector.rs:830-878
    star = G(5, [(0, v) for v in range(1, 5)], False)
    x, lam = ig.eigenvector_centrality_weighted(star, np.ones(4), with_eigenvalue=True)
    assert np.allclose(x, [1.0, 0.5, 0.5, 0.5, 0.5], atol=1e-9) and abs(lam - 2.0) < 1e-6
    k5 = G(5, [(u, v) for u in range(5) for v in range(u + 1, 5)], False)
    x, lam = ig.eigenvector_centrality_weighted(k5, np.ones(10), with_eigenvalue=True)
    assert np.allclose(x, 1.0, atol=1e-9) and abs(lam - 4.0) < 1e-6
    x, lam = ig.eigenvector_centrality_weighted(ig.Graph.with_vertices(4), [], with_eigenvalue=True)
    assert np.all(x == 1.0) and lam == 0.0
    path = G(3, [(0, 1), (1, 2)], False)
    x, lam = ig.eigenvector_centrality_weighted(path, [0.0, 0.0], with_eigenvalue=True)
    assert np.all(x == 1.0) and lam == 0.0
    with pytest.raises(ig.InvalidArgument, match=r"weights vector length \(1\) not equal to number of edges \(2\)"):
        ig.eigenvector_centrality_weighted(path, [1.0])
    with pytest.raises(ig.Unsupported, match="directed eigenvector_centrality_weighted"):
        ig.eigenvector_centrality_weighted(G(3, [(0, 1)], True), [1.0])
    # negative weights: the signed pivot (closed form: eigenvector [1, -sqrt 2, 1]
    # of W = -A for the path, pivot on vertex 1)
    x, lam = ig.eigenvector_centrality_weighted(path, [-1.0, -1.0], with_eigenvalue=True)
    assert np.allclose(x, [-1 / np.sqrt(2), 1.0, -1 / np.sqrt(2)], atol=1e-9) and abs(lam - np.sqrt(2)) < 1e-9
    s = ig.hub_and_authority_scores_weighted(path, [-1.0, -1.0])
    assert np.allclose(s.hub, x, atol=1e-9) and abs(s.eigenvalue - 2.0) < 1e-9
    # hits.rs:763-880
    s = ig.hub_and_authority_scores_weighted(G(0, [], True), [])
    assert len(s.hub) == 0 and s.eigenvalue == 0.0
    s = ig.hub_and_authority_scores_weighted(G(3, [], True), [])
    assert np.all(s.hub == 1.0) and np.all(s.authority == 1.0) and s.eigenvalue == 0.0
    dpath = G(3, [(0, 1), (1, 2)], True)
    s = ig.hub_and_authority_scores_weighted(dpath, [0.0, 0.0])
    assert np.all(s.hub == 1.0) and np.all(s.authority == 1.0) and s.eigenvalue == 0.0
    with pytest.raises(ig.InvalidArgument, match="weights length 1 does not match edge count 2"):
        ig.hub_and_authority_scores_weighted(dpath, [1.0])
    g = G(5, [(0, 1), (0, 2), (1, 3), (2, 3), (3, 4), (1, 4)], True)
    sw, su = ig.hub_and_authority_scores_weighted(g, np.ones(6)), ig.hub_and_authority_scores(g)
    assert np.allclose(sw.hub, su.hub, atol=1e-9) and np.allclose(sw.authority, su.authority, atol=1e-9)
    assert abs(sw.eigenvalue - su.eigenvalue) < 1e-9
    s = ig.hub_and_authority_scores_weighted(G(4, [(0, 2), (0, 3), (1, 2), (1, 3)], True), [1.0, 4.0, 2.0, 3.0])
    assert abs(s.hub[2]) < 1e-9 and abs(s.hub[3]) < 1e-9 and abs(s.authority[0]) < 1e-9
    assert abs(s.authority[1]) < 1e-9 and s.authority[3] > s.authority[2]
    u = G(4, [(0, 1), (1, 2), (2, 3), (0, 3)], False)
    sw, su = ig.hub_and_authority_scores_weighted(u, np.ones(4)), ig.hub_and_authority_scores(u)
    assert np.allclose(sw.hub, su.hub, atol=1e-9) and abs(sw.eigenvalue - su.eigenvalue) < 1e-9


def _weighted_graph(kind, directed):
    if kind == "er":
        n = 20_000
        f, t = O.erdos_renyi_gnm(n, 100_000, directed, False, 31)
    elif kind == "ba":
        n = 30_000
        f, t = O.barabasi_game_bag(n, 4, False, directed, 32)
    elif kind == "rmat":
        n = 1 << 15
        f, t = O.rmat(15, 8 * n, seed=33)
    else:
        rng = np.random.default_rng(34)
        n = 5000
        f = rng.integers(0, n, 30_000).astype(np.uint32)
        t = rng.integers(0, n, 30_000).astype(np.uint32)
        f[:200] = t[:200] = 7  # loops
    g = ig.Graph.from_edge_arrays(n, f, t, directed)
    gf, gt = edges(g)
    w = O.uniform_weights(len(gf), 35, 0.0, 3.0)
    w[::97] = 0.0  # zero-weight edges stay in the graph
    return n, g, gf, gt, w


@pytest.mark.parametrize("kind", ["er", "ba", "rmat", "loops"])
def test_eigenvector_weighted_matches_restatement(cuda_ok, kind):
    n, g, gf, gt, w = _weighted_graph(kind, False)
    x, lam = ig.eigenvector_centrality_weighted(g, w, with_eigenvalue=True)
    ref, rlam, _ = O.eigenvector_centrality_weighted(n, gf, gt, w)
    assert np.max(np.abs(x - ref)) <= TOL, np.max(np.abs(x - ref))
    assert abs(lam - rlam) <= TOL * abs(rlam)
    s = ig.hub_and_authority_scores_weighted(g, w)
    assert np.array_equal(s.hub, x) and np.array_equal(s.authority, x)
    assert abs(s.eigenvalue - lam * lam) <= 1e-12 * lam * lam


@pytest.mark.parametrize("kind", ["er", "ba", "rmat"])
def test_hits_weighted_directed_matches_restatement(cuda_ok, kind):
    n, g, gf, gt, w = _weighted_graph(kind, True)
    s = ig.hub_and_authority_scores_weighted(g, w)
    h, a, lam, _ = O.hub_and_authority_scores_weighted(n, gf, gt, w, True)
    assert np.max(np.abs(s.hub - h)) <= TOL and np.max(np.abs(s.authority - a)) <= TOL
    assert abs(s.eigenvalue - lam) <= TOL * abs(lam)
    assert s.hub.max() == 1.0 and s.authority.max() == 1.0 and s.hub.min() >= 0.0


def test_directed_reference_unit_cases(cuda_ok):
    # eigenvector.rs:880-1052, through the GPU entry point
    full = ig.eigenvector_centrality_full
    k5 = G(5, [(u, v) for u in range(5) for v in range(5) if u != v], True)
    s = ig.eigenvector_centrality_directed(k5, ig.EIG_OUT)
    assert np.allclose(s.vector, 1.0, atol=1e-9) and abs(s.eigenvalue - 4.0) < 1e-6
    k10 = G(10, [(u, v) for u in range(10) for v in range(10) if u != v], True)
    s = ig.eigenvector_centrality_directed(k10, ig.EIG_OUT)
    assert np.allclose(s.vector, 1.0, atol=1e-9) and abs(s.eigenvalue - 9.0) < 1e-9
    out_star, in_star = G(5, [(0, v) for v in range(1, 5)], True), G(5, [(v, 0) for v in range(1, 5)], True)
    s = ig.eigenvector_centrality_directed(out_star, ig.EIG_OUT)
    assert list(s.vector) == [0.0, 1.0, 1.0, 1.0, 1.0] and s.eigenvalue == 0.0
    s = ig.eigenvector_centrality_directed(in_star, ig.EIG_IN)
    assert list(s.vector) == [0.0, 1.0, 1.0, 1.0, 1.0] and s.eigenvalue == 0.0
    s = ig.eigenvector_centrality_directed(in_star, ig.EIG_OUT)
    assert list(s.vector) == [1.0, 0.0, 0.0, 0.0, 0.0] and s.eigenvalue == 0.0
    chord = G(4, [(0, 1), (1, 2), (2, 3), (3, 0), (1, 3)], True)
    s = ig.eigenvector_centrality_directed(chord, ig.EIG_OUT)
    assert abs(s.eigenvalue - 1.220744) < 1e-4
    assert np.allclose(s.vector, [0.819173, 0.671044, 0.549700, 1.0], atol=1e-3)
    s = ig.eigenvector_centrality_directed(G(5, [], True), ig.EIG_OUT)
    assert np.all(s.vector == 1.0) and s.eigenvalue == 0.0
    cyc = G(50, [(i, (i + 1) % 50) for i in range(50)], True)
    s = ig.eigenvector_centrality_directed(cyc, ig.EIG_OUT)
    assert abs(s.eigenvalue - 1.0) < 1e-9 and s.vector.max() - s.vector.min() < 1e-9
    tri = G(3, [(0, 1), (1, 2), (2, 0)], False)
    a, b = full(tri, ig.EIG_OUT), full(tri, ig.EIG_ALL)
    assert np.allclose(a.vector, 1.0, atol=1e-9) and np.array_equal(a.vector, b.vector)
    r = ig.eigenvector_centrality_directed_weighted(G(3, [(0, 1), (1, 2), (2, 0)], True), ig.EIG_ALL, [1.0] * 3)
    assert len(r.vector) == 3
    with pytest.raises(ig.InvalidArgument, match=r"weights vector length \(1\) not equal to number of edges \(3\)"):
        ig.eigenvector_centrality_directed_weighted(G(3, [(0, 1), (1, 2), (2, 0)], True), ig.EIG_OUT, [1.0])
    # hits.rs:871-883: negative weights are taken, nothing is clipped, and the
    # hub vector still reaches |1|
    s = ig.hub_and_authority_scores_weighted(G(3, [(0, 1), (1, 2), (2, 0)], True), [1.0, -1.0, 1.0])
    assert np.all(np.isfinite(s.hub)) and np.all(np.isfinite(s.authority))
    assert abs(np.abs(s.hub).max() - 1.0) < 1e-6
    # directed 2-cycle with weights -1 (Out): the seed is the lambda = -1 eigenvector
    s = ig.eigenvector_centrality_directed_weighted(G(2, [(0, 1), (1, 0)], True), ig.EIG_OUT, [-1.0, -1.0])
    assert list(s.vector) == [1.0, 1.0] and s.eigenvalue == -1.0


def _directed_case(kind):
    if kind == "rmat":
        n = 1 << 13
        f, t = O.rmat(13, 8 * n, seed=51)
    elif kind == "er":
        n = 6000
        f, t = O.erdos_renyi_gnm(n, 24_000, True, False, 52)
    elif kind == "dag":  # edges from lower to higher ids: a DAG with many sinks and sources
        rng = np.random.default_rng(53)
        n = 20_000
        a = rng.integers(0, n, 80_000)
        b = rng.integers(0, n, 80_000)
        keep = a != b
        f = np.minimum(a, b)[keep].astype(np.uint32)
        t = np.maximum(a, b)[keep].astype(np.uint32)
    else:  # cycles through a hub plus loops
        rng = np.random.default_rng(54)
        n = 4000
        f = rng.integers(0, n, 16_000).astype(np.uint32)
        t = rng.integers(0, n, 16_000).astype(np.uint32)
        f[:100] = t[:100] = 9
    return n, f, t


@pytest.mark.parametrize("kind", ["rmat", "er", "dag", "loops"])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("weighted", [False, True])
def test_directed_matches_restatement(cuda_ok, kind, mode, weighted):
    n, f, t = _directed_case(kind)
    g = ig.Graph.from_edge_arrays(n, f, t, True)
    gf, gt = g.edge_arrays()
    w = None
    if weighted:
        w = O.uniform_weights(len(gf), 55, 0.0, 2.0)
        w[::11] = 0.0
    s = ig.eigenvector_centrality_full(g, mode, w)
    ref, lam, _ = O.eigenvector_centrality_full(n, gf, gt, True, mode, weights=w)
    assert np.max(np.abs(s.vector - ref)) <= TOL, np.max(np.abs(s.vector - ref))
    assert abs(s.eigenvalue - lam) <= TOL * max(abs(lam), 1.0)
    if kind == "dag" and mode != 2:
        assert s.eigenvalue == 0.0 and set(np.unique(s.vector)) <= {0.0, 1.0}


def _mixed_weights(m, seed):
    # mostly positive, 5 % small negative weights: the dominant eigenvector is
    # well separated, so the signed iterations converge well inside the cap
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.2, 2.0, m)
    neg = rng.random(m) < 0.05
    w[neg] = -rng.uniform(0.05, 0.5, int(neg.sum()))
    return w


@pytest.mark.parametrize("kind", ["er", "ba", "rmat"])
def test_negative_weights_match_restatement(cuda_ok, kind):
    if kind == "er":
        n = 20_000
        f, t = O.erdos_renyi_gnm(n, 100_000, False, False, 61)
    elif kind == "ba":  # degree-skewed: relabelled, so pivot ties go through the caller ids
        n = 30_000
        f, t = O.barabasi_game_bag(n, 4, False, False, 62)
    else:
        n = 1 << 13
        f, t = O.rmat(13, 8 * n, seed=63)
    g = ig.Graph.from_edge_arrays(n, f, t, False)
    gf, gt = g.edge_arrays()
    w = _mixed_weights(len(gf), 64)
    x, lam = ig.eigenvector_centrality_weighted(g, w, with_eigenvalue=True)
    ref, rlam, it = O.eigenvector_centrality_weighted(n, gf, gt, w)
    assert it < 5000 and x.min() < 0.0  # signed: nothing clamped
    assert np.max(np.abs(x - ref)) <= TOL and abs(lam - rlam) <= TOL * abs(rlam)
    s = ig.hub_and_authority_scores_weighted(g, w)
    h, _, hlam, _ = O.hub_and_authority_scores_weighted(n, gf, gt, w, False)
    assert np.max(np.abs(s.hub - h)) <= TOL and abs(s.eigenvalue - hlam) <= TOL * abs(hlam)
    gd = ig.Graph.from_edge_arrays(n, f, t, True)
    df, dt = gd.edge_arrays()
    wd = _mixed_weights(len(df), 65)
    s = ig.hub_and_authority_scores_weighted(gd, wd)
    h, a, hlam, it = O.hub_and_authority_scores_weighted(n, df, dt, wd, True)
    assert it < 5000
    assert np.max(np.abs(s.hub - h)) <= TOL and np.max(np.abs(s.authority - a)) <= TOL
    assert abs(s.eigenvalue - hlam) <= TOL * abs(hlam)
    if kind == "rmat":  # the directed shifted iterations converge on this graph
        for mode in (ig.EIG_OUT, ig.EIG_IN, ig.EIG_ALL):
            r = ig.eigenvector_centrality_full(gd, mode, wd)
            ref, rlam, it = O.eigenvector_centrality_full(n, df, dt, True, mode, weights=wd)
            assert it < 5000
            assert np.max(np.abs(r.vector - ref)) <= TOL, (mode, np.max(np.abs(r.vector - ref)))
            assert abs(r.eigenvalue - rlam) <= TOL * abs(rlam)


@pytest.mark.parametrize("kind", ["er", "ba", "rmat", "loops"])
def test_row_block_product_matches_restatement(cuda_ok, kind):
    # the same checks with the adjacency product as the row-block pass
    # (tuning seg_eig64 = 0; the tile-segmented pass is the default for
    # unweighted graphs): undirected eigenvector centrality, directed HITS,
    # and the directed modes, unweighted
    ig.set_tuning("seg_eig64", 0)
    try:
        test_eigenvector_matches_restatement(cuda_ok, kind)
        if kind in ("rmat", "ba"):
            test_hits_directed_matches_restatement(cuda_ok, kind)
        if kind in ("rmat", "er", "loops"):
            for mode in (0, 1, 2):
                test_directed_matches_restatement(cuda_ok, kind, mode, False)
    finally:
        ig.reset_tuning()
