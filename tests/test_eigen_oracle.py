"""The CPU restatements of eigenvector_centrality and hub_and_authority_scores
(unweighted; oracle/prg_oracle.c) pinned to the reference's own unit tests
(src/algorithms/properties/eigenvector.rs:770-829, hits.rs:627-760)."""
import numpy as np

import oracle as O


def E(pairs):
    a = np.array(pairs, np.uint32).reshape(-1, 2)
    return a[:, 0].copy(), a[:, 1].copy()


def test_eigenvector_reference_cases():
    assert len(O.eigenvector_centrality(0, *E([]))[0]) == 0
    assert list(O.eigenvector_centrality(1, *E([]))[0]) == [1.0]
    assert np.allclose(O.eigenvector_centrality(3, *E([]))[0], 1.0, atol=1e-9)
    assert np.allclose(O.eigenvector_centrality(3, *E([(0, 1), (1, 2), (2, 0)]))[0], 1.0, atol=1e-9)
    x, lam, _ = O.eigenvector_centrality(4, *E([(0, 1), (0, 2), (0, 3)]))
    assert np.allclose(x, [1.0] + [1 / np.sqrt(3)] * 3, atol=1e-9)
    assert abs(lam - np.sqrt(3)) < 1e-9
    k4 = [(u, v) for u in range(4) for v in range(u + 1, 4)]
    assert np.allclose(O.eigenvector_centrality(4, *E(k4))[0], 1.0, atol=1e-9)


def test_hits_reference_cases():
    h, a, lam, _ = O.hub_and_authority_scores(3, *E([]), True)
    assert np.all(h == 1.0) and np.all(a == 1.0) and lam == 0.0
    h, a, lam, _ = O.hub_and_authority_scores(2, *E([(0, 1)]), True)
    assert abs(lam - 1.0) < 1e-6
    h, a, lam, _ = O.hub_and_authority_scores(4, *E([(0, 2), (0, 3), (1, 2), (1, 3)]), True)
    assert np.allclose(h, [1, 1, 0, 0], atol=1e-9) and np.allclose(a, [0, 0, 1, 1], atol=1e-9)
    assert abs(lam - 4.0) < 1e-6
    h, a, lam, _ = O.hub_and_authority_scores(3, *E([(0, 1), (1, 2), (2, 0)]), True)
    assert np.allclose(h, 1.0, atol=1e-9) and abs(lam - 1.0) < 1e-6
    h, a, _, _ = O.hub_and_authority_scores(3, *E([(0, 2), (1, 2)]), True)  # sink
    assert abs(h[2]) < 1e-9 and abs(a[2] - 1) < 1e-9 and abs(a[0]) < 1e-9 and abs(a[1]) < 1e-9
    h, a, _, _ = O.hub_and_authority_scores(3, *E([(0, 1), (0, 2)]), True)  # source
    assert abs(a[0]) < 1e-9 and abs(h[0] - 1) < 1e-9
    # undirected: hub = authority = eigenvector centrality, eigenvalue = lambda^2
    ec, lam1, _ = O.eigenvector_centrality(4, *E([(0, 1), (0, 2), (0, 3)]))
    h, a, lam, _ = O.hub_and_authority_scores(4, *E([(0, 1), (0, 2), (0, 3)]), False)
    assert np.array_equal(h, ec) and np.array_equal(a, ec) and abs(lam - lam1 ** 2) < 1e-12
    # h proportional to A a after convergence (hits.rs doc example)
    f, t = E([(0, 1), (0, 3), (1, 2), (1, 3), (2, 0), (2, 4), (3, 2), (4, 0), (4, 1)])
    h, a, _, _ = O.hub_and_authority_scores(5, f, t, True)
    ha = np.zeros(5)
    np.add.at(ha, f, a[t])
    assert np.allclose(ha / ha.max(), h, atol=1e-6)


def test_eigenvector_weighted_reference_cases():
    # eigenvector.rs:830-878
    x, lam, _ = O.eigenvector_centrality_weighted(5, *E([(0, v) for v in range(1, 5)]), np.ones(4))
    assert np.allclose(x, [1.0, 0.5, 0.5, 0.5, 0.5], atol=1e-9) and abs(lam - 2.0) < 1e-6
    k5 = [(u, v) for u in range(5) for v in range(u + 1, 5)]
    x, lam, _ = O.eigenvector_centrality_weighted(5, *E(k5), np.ones(10))
    assert np.allclose(x, 1.0, atol=1e-9) and abs(lam - 4.0) < 1e-6
    x, lam, _ = O.eigenvector_centrality_weighted(4, *E([]), np.zeros(0))
    assert np.all(x == 1.0) and lam == 0.0
    x, lam, _ = O.eigenvector_centrality_weighted(3, *E([(0, 1), (1, 2)]), np.zeros(2))
    assert np.all(x == 1.0) and lam == 0.0
    # unit weights give the unweighted centrality (a different seed, same fixed point)
    f, t = E([(0, 1), (1, 2), (2, 3), (3, 0), (0, 2), (4, 0)])
    xw, lw, _ = O.eigenvector_centrality_weighted(5, f, t, np.ones(6))
    xu, lu, _ = O.eigenvector_centrality(5, f, t)
    assert np.allclose(xw, xu, atol=1e-9) and abs(lw - lu) < 1e-9


def test_hits_weighted_reference_cases():
    # hits.rs:763-880
    h, a, lam, _ = O.hub_and_authority_scores_weighted(0, *E([]), np.zeros(0), True)
    assert len(h) == 0 and len(a) == 0 and lam == 0.0
    h, a, lam, _ = O.hub_and_authority_scores_weighted(3, *E([]), np.zeros(0), True)
    assert np.all(h == 1.0) and np.all(a == 1.0) and lam == 0.0
    h, a, lam, _ = O.hub_and_authority_scores_weighted(3, *E([(0, 1), (1, 2)]), np.zeros(2), True)
    assert np.all(h == 1.0) and np.all(a == 1.0) and lam == 0.0
    f, t = E([(0, 1), (0, 2), (1, 3), (2, 3), (3, 4), (1, 4)])
    hw, aw, lw, _ = O.hub_and_authority_scores_weighted(5, f, t, np.ones(6), True)
    hu, au, lu, _ = O.hub_and_authority_scores(5, f, t, True)
    assert np.allclose(hw, hu, atol=1e-6) and np.allclose(aw, au, atol=1e-6) and abs(lw - lu) < 1e-6
    h, a, _, _ = O.hub_and_authority_scores_weighted(4, *E([(0, 2), (0, 3), (1, 2), (1, 3)]),
                                                     np.array([1.0, 4.0, 2.0, 3.0]), True)
    assert abs(h[2]) < 1e-9 and abs(h[3]) < 1e-9 and abs(a[0]) < 1e-9 and abs(a[1]) < 1e-9
    assert a[3] > a[2]
    # hub proportional to W authority after convergence
    f, t = E([(0, 1), (0, 2), (1, 3), (2, 3), (3, 4), (4, 0)])
    w = np.array([1.5, 0.5, 2.0, 1.0, 0.75, 1.25])
    h, a, _, _ = O.hub_and_authority_scores_weighted(5, f, t, w, True)
    wa = np.zeros(5)
    np.add.at(wa, f, w * a[t])
    assert np.allclose(wa / np.abs(wa).max(), h, atol=1e-6)
    # undirected: the weighted eigenvector and its eigenvalue squared
    f, t = E([(0, 1), (1, 2), (2, 3), (0, 3)])
    h, a, lam, _ = O.hub_and_authority_scores_weighted(4, f, t, np.ones(4), False)
    hu, au, lu, _ = O.hub_and_authority_scores(4, f, t, False)
    assert np.allclose(h, hu, atol=1e-6) and np.array_equal(h, a) and abs(lam - lu) < 1e-6


def test_eigenvector_directed_reference_cases():
    # eigenvector.rs:880-1052 (directed) and :960-985 (dispatch)
    full = O.eigenvector_centrality_full
    k5 = [(u, v) for u in range(5) for v in range(5) if u != v]
    x, lam, _ = full(5, *E(k5), True, O.EIG_OUT)
    assert np.allclose(x, 1.0, atol=1e-9) and abs(lam - 4.0) < 1e-6
    k10 = [(u, v) for u in range(10) for v in range(10) if u != v]
    x, lam, _ = full(10, *E(k10), True, O.EIG_OUT)
    assert np.allclose(x, 1.0, atol=1e-9) and abs(lam - 9.0) < 1e-9
    x, lam, _ = full(5, *E([(0, v) for v in range(1, 5)]), True, O.EIG_OUT)  # DAG: sinks
    assert list(x) == [0.0, 1.0, 1.0, 1.0, 1.0] and lam == 0.0
    x, lam, _ = full(5, *E([(v, 0) for v in range(1, 5)]), True, O.EIG_IN)  # DAG, In: sources
    assert list(x) == [0.0, 1.0, 1.0, 1.0, 1.0] and lam == 0.0
    x, lam, _ = full(5, *E([(v, 0) for v in range(1, 5)]), True, O.EIG_OUT)
    assert list(x) == [1.0, 0.0, 0.0, 0.0, 0.0] and lam == 0.0
    x, lam, _ = full(4, *E([(0, 1), (1, 2), (2, 3), (3, 0), (1, 3)]), True, O.EIG_OUT)
    assert abs(lam - 1.220744) < 1e-4 and np.allclose(x, [0.819173, 0.671044, 0.549700, 1.0], atol=1e-3)
    x, lam, _ = full(5, *E([]), True, O.EIG_OUT)
    assert np.all(x == 1.0) and lam == 0.0
    x, lam, _ = full(50, *E([(i, (i + 1) % 50) for i in range(50)]), True, O.EIG_OUT)
    assert abs(lam - 1.0) < 1e-9 and x.max() - x.min() < 1e-9
    # undirected input takes the symmetric path whatever the mode
    tri = E([(0, 1), (1, 2), (2, 0)])
    a = full(3, *tri, False, O.EIG_OUT)
    b = full(3, *tri, False, O.EIG_ALL)
    assert np.allclose(a[0], 1.0, atol=1e-9) and np.array_equal(a[0], b[0]) and a[1] == b[1]
    # In mode on G is Out mode on the reversed graph
    rng = np.random.default_rng(4)
    f = rng.integers(0, 300, 3000).astype(np.uint32)
    t = rng.integers(0, 300, 3000).astype(np.uint32)
    xi, li, _ = full(300, f, t, True, O.EIG_IN)
    xo, lo, _ = full(300, t, f, True, O.EIG_OUT)
    assert np.array_equal(xi, xo) and li == lo
    # unit weights are the unweighted iteration
    xw, lw, _ = full(300, f, t, True, O.EIG_OUT, weights=np.ones(3000))
    xu, lu, _ = full(300, f, t, True, O.EIG_OUT)
    assert np.array_equal(xw, xu) and lw == lu


def test_negative_weight_rules():
    # hits.rs:871-883: with negative weights nothing is clipped and the hub
    # vector still reaches |1|
    h, a, lam, _ = O.hub_and_authority_scores_weighted(3, *E([(0, 1), (1, 2), (2, 0)]), np.array([1.0, -1.0, 1.0]),
                                                       True)
    assert np.all(np.isfinite(h)) and np.all(np.isfinite(a)) and abs(np.abs(h).max() - 1.0) < 1e-6
    # undirected path 0-1-2 with weights -1: the largest eigenvalue of W + I
    # is 1 + sqrt 2, eigenvector [1, -sqrt 2, 1]; the signed pivot is vertex 1
    x, lam, _ = O.eigenvector_centrality_weighted(3, *E([(0, 1), (1, 2)]), np.array([-1.0, -1.0]))
    assert np.allclose(x, [-1 / np.sqrt(2), 1.0, -1 / np.sqrt(2)], atol=1e-9) and abs(lam - np.sqrt(2)) < 1e-9
    # the same graph through HITS: hub = authority = x, eigenvalue lambda^2
    h, a, lam2, _ = O.hub_and_authority_scores_weighted(3, *E([(0, 1), (1, 2)]), np.array([-1.0, -1.0]), False)
    assert np.allclose(h, x, atol=1e-9) and np.array_equal(h, a) and abs(lam2 - 2.0) < 1e-9
    # directed 2-cycle with weights -1, Out mode: the |strength| seed [1, 1] is
    # the lambda = -1 eigenvector of M and the shifted iteration keeps it;
    # negative weights skip the zero-eigenvalue rule
    x, lam, _ = O.eigenvector_centrality_full(2, *E([(0, 1), (1, 0)]), True, O.EIG_OUT, weights=[-1.0, -1.0])
    assert list(x) == [1.0, 1.0] and lam == -1.0
    # an extra edge of weight -1e-9 (signed rules) against +1e-9 (unsigned)
    rng = np.random.default_rng(7)
    f = rng.integers(0, 200, 1500).astype(np.uint32)
    t = rng.integers(0, 200, 1500).astype(np.uint32)
    w = rng.random(1500) + 0.5
    w[-1] = 1e-9
    x0, l0, _ = O.eigenvector_centrality_weighted(200, f, t, w)
    w[-1] = -1e-9
    x1, l1, _ = O.eigenvector_centrality_weighted(200, f, t, w)
    assert np.abs(x1 - x0).max() < 1e-6 and abs(l1 - l0) < 1e-6
