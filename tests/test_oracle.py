"""The CPU oracle, pinned against the reference's own golden vectors and unit
tests (CPU only).  The oracle is the checker for every GPU parity test, so
these run first and without a GPU."""
import numpy as np
import pytest

import oracle as O
from conftest import case_edges, within

D = 0.85


def run_case(case):
    f, t = case_edges(case)
    n, directed = case["n"], case["directed"]
    if case["algo"] == "pagerank":
        return O.pagerank(n, f, t, directed)
    if case["algo"] == "pagerank_weighted":
        return O.pagerank_weighted(n, f, t, directed, case["weights"])
    return O.personalized_pagerank(n, f, t, directed, case["params"]["reset"], case["params"]["damping"])


def test_golden_fixtures(golden_cases):
    assert len(golden_cases) == 19
    for case in golden_cases:
        got = run_case(case)
        assert within(got, case["expected"], case["tol_kind"], case["tol_tol"]), case["name"]


# ---- pagerank.rs:145-240 -------------------------------------------------

def E(pairs, directed):
    a = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
    f, t = a[:, 0].copy(), a[:, 1].copy()
    if not directed:
        f, t = np.minimum(f, t), np.maximum(f, t)
    return f, t


def test_pagerank_unit_cases():
    assert len(O.pagerank(0, *E([], False), False)) == 0
    assert list(O.pagerank(1, *E([], False), False)) == [1.0]
    assert np.allclose(O.pagerank(4, *E([], False), False), 0.25, atol=1e-9)
    assert np.allclose(O.pagerank(3, *E([[0, 1], [1, 2], [2, 0]], False), False), 1 / 3, atol=1e-9)
    assert np.allclose(O.pagerank(4, *E([[i, (i + 1) % 4] for i in range(4)], True), True), 0.25, atol=1e-9)
    pr = O.pagerank(4, *E([[0, 1], [0, 2], [1, 2], [1, 3], [2, 3]], False), False)
    assert abs(pr.sum() - 1) < 1e-9
    pr = O.pagerank(4, *E([[0, 1], [0, 2], [0, 3]], False), False)
    assert all(pr[0] > x for x in pr[1:]) and np.allclose(pr[1:], pr[1], atol=1e-9)
    pr = O.pagerank(2, *E([[0, 1]], True), True)
    assert abs(pr.sum() - 1) < 1e-9 and pr[1] > pr[0]


def test_pagerank_weighted_unit_cases():
    tri = E([[0, 1], [1, 2], [2, 0]], False)
    assert np.allclose(O.pagerank_weighted(3, *tri, False, [1.0] * 3), O.pagerank(3, *tri, False), atol=1e-9)
    cyc = E([[i, (i + 1) % 4] for i in range(4)], True)
    assert np.allclose(O.pagerank_weighted(4, *cyc, True, [1.0] * 4), O.pagerank(4, *cyc, True), atol=1e-9)
    pr = O.pagerank_weighted(4, *E([[0, 1], [0, 2], [1, 2], [1, 3], [2, 3]], False), False, [1, 2, .5, 1.5, 1])
    assert abs(pr.sum() - 1) < 1e-9
    pr = O.pagerank_weighted(3, *E([[0, 1], [0, 2]], True), True, [100.0, 0.01])
    assert abs(pr.sum() - 1) < 1e-9 and pr[1] > pr[2]


def test_personalized_unit_cases():
    g = E([[0, 1], [0, 2], [1, 2], [2, 3]], False)
    assert np.allclose(O.personalized_pagerank(4, *g, False, [0.25] * 4, D), O.pagerank(4, *g, False), atol=1e-9)
    star = E([[0, 1], [0, 2], [0, 3]], False)
    pb = O.personalized_pagerank(4, *star, False, [0, 1, 0, 0], D)
    assert pb[1] > pb[2] and pb[1] > pb[3] and pb[0] > pb[1]
    chain = E([[0, 1], [1, 2]], True)
    pr = O.personalized_pagerank(3, *chain, True, [1, 0, 0], D)
    assert pr[0] > pr[1] > pr[2] and abs(pr.sum() - 1) < 1e-9
    tri = E([[0, 1], [1, 2], [2, 0]], False)
    assert O.personalized_pagerank(3, *tri, False, [1, 0, 0], 0.5)[0] > \
        O.personalized_pagerank(3, *tri, False, [1, 0, 0], 0.99)[0]
    assert np.allclose(O.personalized_pagerank(3, *tri, False, [10, 0, 0], D),
                       O.personalized_pagerank(3, *tri, False, [1, 0, 0], D), atol=1e-9)
    pr = O.personalized_pagerank(4, *E([], False), False, [0, 0, 1, 0], D)
    assert abs(pr[2] - 1) < 1e-9 and np.all(np.abs(pr[[0, 1, 3]]) < 1e-9)


def test_splitmix64_known_answers():
    # SplitMix64 (Steele, Lea, Flood 2014) from state 0: first output of the
    # published generator; rng.rs:40-46 uses the same constants.
    assert O.splitmix_stream(0, 1)[0] == 0xE220A8397B1DCDAF
    a, b = O.splitmix_stream(42, 50), O.splitmix_stream(42, 50)
    assert a == b and O.splitmix_stream(1, 5) != O.splitmix_stream(2, 5)


def test_generators_match_reference_fixture_invariants():
    import json
    import os

    from conftest import GOLDEN

    gens = json.load(open(os.path.join(GOLDEN, "reference_fixtures.json")))["generators"]
    assert len(gens) == 29
    for g in gens:
        p, e = g["params"], g["expected"]
        if g["algo"] == "erdos_renyi_gnm":
            f, t = O.erdos_renyi_gnm(p["n"], p["m"], p["directed"], p["loops"], p["seed"])
            assert len(f) == e["ecount"]
            pairs = set(zip(f.tolist(), t.tolist()))
            assert len(pairs) == len(f)  # simple graph
            if not p["loops"]:
                assert np.all(f != t)
        elif g["algo"] == "barabasi_game_bag":
            f, t = O.barabasi_game_bag(p["n"], p["m"], p["outpref"], p["directed"], p["seed"])
            assert len(f) == e["ecount"]
            if p["directed"] and len(f):
                assert np.all(t < f)  # BA temporal order: new vertex -> older
        else:
            k = len(p["block_sizes"])
            f, t = O.sbm_game(p["pref_matrix"], p["block_sizes"], p["directed"], p["loops"], p["multiple"],
                              p["seed"])
            assert e["ecount_min"] <= len(f) <= e["ecount_max"], g["name"]
            if e.get("diagonal_only_pref"):
                off = np.cumsum([0] + p["block_sizes"])
                bf = np.searchsorted(off, f, side="right") - 1
                bt = np.searchsorted(off, t, side="right") - 1
                assert np.all(bf == bt)
            if e.get("is_simple"):
                assert len(set(zip(f.tolist(), t.tolist()))) == len(f) and np.all(f != t)
            assert k == len(p["block_sizes"])


def test_rmat_generator_thread_invariant():
    a = O.rmat(12, 1 << 14, seed=7, nthreads=1)
    b = O.rmat(12, 1 << 14, seed=7, nthreads=5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[0].max() < 4096 and a[1].max() < 4096


def test_tight_oracle_brackets_restatement():
    f, t = O.erdos_renyi_gnm(2000, 20000, True, False, 11)
    ref, iters = O.pagerank(2000, f, t, True, return_iters=True)
    tight, it2, last = O.pagerank_tight(2000, f, t, True, tol=1e-15)
    assert last < 1e-14
    # successive-change stop at 1e-10 => error <= d/(1-d) * 1e-10
    assert np.abs(ref - tight).sum() <= D / (1 - D) * 1e-10 * 1.01
    assert 5 < iters < 1000


def test_tight_oracle_weighted_and_reset():
    f, t = O.barabasi_game_bag(500, 3, False, False, 5)
    w = O.uniform_weights(len(f), 9)
    ref = O.pagerank_weighted(500, f, t, False, w)
    tight, _, _ = O.pagerank_tight(500, f, t, False, weights=w, tol=1e-15)
    assert np.abs(ref - tight).sum() <= D / (1 - D) * 1e-10 * 1.01
    r = np.zeros(500)
    r[[3, 7, 11]] = 1.0
    ref = O.personalized_pagerank(500, f, t, False, r, D)
    tight, _, _ = O.pagerank_tight(500, f, t, False, reset=r, tol=1e-15)
    assert np.abs(ref - tight).sum() <= D / (1 - D) * 1e-10 * 1.01


def test_ppr_residuals_certify_batched_columns():
    # the residual pass behind the full-size batched check: the restatement's
    # own answers (stored in FP32) have residuals near FP32 rounding, and a
    # perturbation of one entry shows up with the factor (1 + d) it must have
    n = 3000
    f, t = O.erdos_renyi_gnm(n, 15_000, False, False, 5)
    seeds = [np.array([1, 2, 2, 50], np.uint32), np.array([7], np.uint32), np.array([0, 2999], np.uint32)]
    X = np.zeros((n, 3), np.float32)
    for k, sl in enumerate(seeds):
        r = np.zeros(n)
        for v in sl:
            r[v] += 1 / len(sl)
        X[:, k] = O.personalized_pagerank(n, f, t, False, r, 0.85)
    res = O.ppr_residuals(n, f, t, False, seeds, X)
    assert res.max() < 1e-7
    X2 = X.copy()
    X2[10, 1] += np.float32(1e-4)
    res2 = O.ppr_residuals(n, f, t, False, seeds, X2)
    assert abs(res2[1] - 1e-4 * (1 + 0.85)) < 2e-5 and np.allclose(res2[[0, 2]], res[[0, 2]])
