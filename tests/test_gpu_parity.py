"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

FP64 drop-in: max-abs <= 1e-10 against the restatement of the reference's
pagerank()/pagerank_weighted()/personalized_pagerank() on identical seeded
graphs, and within each reference fixture's own tolerance.  Refined and
error-bound forms: L1 <= 1e-10 against the tight FP64 oracle.
"""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O
from conftest import case_edges, within

pytestmark = pytest.mark.gpu

D = 0.85
PARITY = 1e-10  # max-abs, FP64 drop-in vs reference restatement
L1_TOL = 1e-10  # L1 vs tight FP64 oracle for refined / error-bound forms


def G(n, f, t, directed):
    return ig.Graph.from_edge_arrays(n, f, t, directed)


def maxabs(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if len(a) else 0.0


def test_reference_fixtures(cuda_ok, golden_cases):
    for case in golden_cases:
        f, t = case_edges(case)
        g = G(case["n"], f, t, case["directed"])
        if case["algo"] == "pagerank":
            got, ref = ig.pagerank(g), O.pagerank(case["n"], f, t, case["directed"])
        elif case["algo"] == "pagerank_weighted":
            got = ig.pagerank_weighted(g, case["weights"])
            ref = O.pagerank_weighted(case["n"], f, t, case["directed"], case["weights"])
        else:
            p = case["params"]
            got = ig.personalized_pagerank(g, p["reset"], p["damping"])
            ref = O.personalized_pagerank(case["n"], f, t, case["directed"], p["reset"], p["damping"])
        assert within(got, case["expected"], case["tol_kind"], case["tol_tol"]), case["name"]
        assert maxabs(got, ref) <= PARITY, case["name"]


def test_reference_unit_cases(cuda_ok):
    # pagerank.rs:145-240
    assert np.allclose(ig.pagerank(ig.Graph.with_vertices(4)), 0.25, atol=1e-9)
    g = ig.Graph.with_vertices(3)
    g.add_edges([(0, 1), (1, 2), (2, 0)])
    assert np.allclose(ig.pagerank(g), 1 / 3, atol=1e-9)
    assert np.allclose(ig.pagerank_weighted(g, [1.0] * 3), ig.pagerank(g), atol=1e-9)
    star = ig.Graph.with_vertices(4)
    star.add_edges([(0, 1), (0, 2), (0, 3)])
    pr = ig.pagerank(star)
    assert all(pr[0] > x for x in pr[1:])
    d = ig.Graph.new(2, True)
    d.add_edge(0, 1)
    pr = ig.pagerank(d)
    assert abs(pr.sum() - 1) < 1e-9 and pr[1] > pr[0]
    # personalized_pagerank.rs:270-522
    pb = ig.personalized_pagerank(star, [0, 1, 0, 0], D)
    assert pb[1] > pb[2] and pb[0] > pb[1]
    iso = ig.personalized_pagerank(ig.Graph.with_vertices(4), [0, 0, 1, 0], D)
    assert abs(iso[2] - 1) < 1e-9
    c4 = ig.Graph.with_vertices(4)
    c4.add_edges([(0, 1), (1, 2), (2, 3), (3, 0)])
    assert np.allclose(ig.personalized_pagerank_vs(c4, [0, 1], D),
                       ig.personalized_pagerank(c4, [0.5, 0.5, 0, 0], D), atol=1e-12)
    assert np.allclose(ig.personalized_pagerank_default(g, [1, 0, 0]),
                       ig.personalized_pagerank(g, [1, 0, 0], 0.85), atol=1e-15)


def test_config1_erdos_renyi_parity(cuda_ok):
    # directed G(n=10,000, m=100,000), no loops, unweighted, d=0.85, f64
    n, m = 10_000, 100_000
    f, t = O.erdos_renyi_gnm(n, m, True, False, 20240601)
    ref, iters = O.pagerank(n, f, t, True, return_iters=True)
    got = ig.pagerank(G(n, f, t, True))
    assert maxabs(got, ref) <= PARITY
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        x, st = dg.solve(ig.Options())
        assert maxabs(x, ref) <= PARITY
        assert abs(st.iterations - iters) <= 1


def test_weighted_barabasi_parity(cuda_ok):
    n = 30_000
    f, t = O.barabasi_game_bag(n, 8, False, False, 7)
    w = O.uniform_weights(len(f), 99)
    ref = O.pagerank_weighted(n, f, t, False, w)
    got = ig.pagerank_weighted(G(n, f, t, False), w)
    assert maxabs(got, ref) <= PARITY


def test_weighted_directed_with_zero_weights(cuda_ok):
    n = 5000
    f, t = O.erdos_renyi_gnm(n, 40_000, True, True, 3)
    w = O.uniform_weights(len(f), 5)
    w[::7] = 0.0  # zero-weight arcs stay in the adjacency; all-zero vertices are dangling
    w[f == 17] = 0.0
    ref = O.pagerank_weighted(n, f, t, True, w)
    got = ig.pagerank_weighted(G(n, f, t, True), w)
    assert maxabs(got, ref) <= PARITY


def test_personalized_parity_sbm(cuda_ok):
    sizes = [500] * 8
    pin, pout = 12 / 499, 2 / (7 * 500)
    pref = [[pin if i == j else pout for j in range(8)] for i in range(8)]
    f, t = O.sbm_game(pref, sizes, False, False, False, 77)
    n = sum(sizes)
    rng = np.random.default_rng(5)
    g = G(n, f, t, False)
    for k in range(3):
        r = np.zeros(n)
        r[rng.choice(n, size=1 + 10 * k, replace=False)] = rng.random(1 + 10 * k) + 0.1
        ref = O.personalized_pagerank(n, f, t, False, r, 0.85 - 0.1 * k)
        got = ig.personalized_pagerank(g, r, 0.85 - 0.1 * k)
        assert maxabs(got, ref) <= PARITY
    vids = [3, 3, 900, 1500]
    r = np.zeros(n)
    for v in vids:
        r[v] += 1 / len(vids)
    assert maxabs(ig.personalized_pagerank_vs(g, vids, D), O.personalized_pagerank(n, f, t, False, r, D)) <= PARITY


def test_self_loops_multi_edges_and_hubs(cuda_ok):
    # undirected self-loops count twice (graph.rs:877-900); multi-edges count per copy;
    # a 40,000-arc hub row takes the split-row path, 3,000-arc rows the long-row path
    rng = np.random.default_rng(1)
    n = 50_000
    f = rng.integers(0, n, 120_000, dtype=np.uint32)
    t = rng.integers(0, n, 120_000, dtype=np.uint32)
    hub = np.full(40_000, 5, np.uint32)
    f = np.concatenate([f, rng.integers(0, n, 40_000, dtype=np.uint32), np.arange(0, 3000, dtype=np.uint32),
                        np.full(3000, 11, np.uint32)])
    t = np.concatenate([t, hub, np.full(3000, 9, np.uint32), np.full(3000, 11, np.uint32)])
    for directed in (True, False):
        ff, tt = (f, t) if directed else (np.minimum(f, t), np.maximum(f, t))
        ref = O.pagerank(n, ff, tt, directed)
        with ig.DeviceGraph.from_host(n, ff, tt, directed) as dg:
            assert dg.n_hubs >= 1
            x, _ = dg.solve(ig.Options())
        assert maxabs(x, ref) <= PARITY


def test_all_dangling_and_isolated(cuda_ok):
    n = 1000
    f = np.array([1, 2, 3], np.uint32)
    t = np.array([0, 0, 0], np.uint32)
    assert maxabs(ig.pagerank(G(n, f, t, True)), O.pagerank(n, f, t, True)) <= PARITY
    assert maxabs(ig.pagerank(ig.Graph.new(n, True)), np.full(n, 1 / n)) <= PARITY


def test_rmat_device_generator_bitexact(cuda_ok):
    import torch

    scale, m = 14, 1 << 18
    df = torch.empty(m, dtype=torch.int32, device="cuda")
    dt = torch.empty(m, dtype=torch.int32, device="cuda")
    ig.rmat_device(scale, m, df.data_ptr(), dt.data_ptr(), seed=12345)
    torch.cuda.synchronize()
    cf, ct = O.rmat(scale, m, seed=12345)
    assert np.array_equal(df.cpu().numpy().view(np.uint32), cf)
    assert np.array_equal(dt.cpu().numpy().view(np.uint32), ct)


def test_deterministic_bits(cuda_ok):
    f, t = O.rmat(14, 16 << 14, seed=3)
    with ig.DeviceGraph.from_host(1 << 14, f, t, True) as dg:
        a, _ = dg.solve(ig.Options())
        b, _ = dg.solve(ig.Options())
        c, _ = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
        d, _ = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert np.array_equal(c.view(np.uint64), d.view(np.uint64))


@pytest.mark.parametrize("scale", [12, 16])
def test_refined_and_error_bound_reach_tolerance(cuda_ok, scale):
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=scale)
    tight, _, last = O.pagerank_tight(n, f, t, True, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        xr, sr = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
        xb, sb = dg.solve(ig.Options(stop=ig.STOP_ERROR_BOUND))
    assert np.abs(xr - tight).sum() <= L1_TOL, (np.abs(xr - tight).sum(), sr)
    assert np.abs(xb - tight).sum() <= L1_TOL
    assert sr.error_bound <= L1_TOL and sb.error_bound <= L1_TOL
    assert sr.fp32_passes > 0 and sr.residual_passes >= 2


def test_refined_weighted_and_personalized(cuda_ok):
    n = 20_000
    f, t = O.barabasi_game_bag(n, 6, False, False, 2)
    w = O.uniform_weights(len(f), 4)
    tight, _, _ = O.pagerank_tight(n, f, t, False, weights=w, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, False, weights=w) as dg:
        x, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
    assert np.abs(x - tight).sum() <= L1_TOL
    r = np.zeros(n)
    r[[1, 50, 999]] = [1.0, 2.0, 0.5]
    tight, _, _ = O.pagerank_tight(n, f, t, False, reset=r, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        x, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED), reset=r)
    assert np.abs(x - tight).sum() <= L1_TOL


def test_large_rmat_properties(cuda_ok):
    # scale 20: size-independent properties instead of a CPU run
    import torch

    scale = 20
    n, m = 1 << scale, 16 << scale
    df = torch.empty(m, dtype=torch.int32, device="cuda")
    dt = torch.empty(m, dtype=torch.int32, device="cuda")
    ig.rmat_device(scale, m, df.data_ptr(), dt.data_ptr(), seed=99)
    dg = ig.DeviceGraph.from_device(n, m, df.data_ptr(), dt.data_ptr(), True)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    s64 = dg.solve_device(out.data_ptr(), ig.Options(stop=ig.STOP_ERROR_BOUND))
    x64 = out.cpu().numpy().copy()
    s32 = dg.solve_device(out.data_ptr(), ig.Options(precision=ig.PRECISION_FP32_REFINED))
    x32 = out.cpu().numpy().copy()
    dg.close()
    assert abs(x64.sum() - 1) < 1e-9 and abs(x32.sum() - 1) < 1e-12
    assert np.all(x64 > 0) and np.all(x32 > 0)
    # both certified within 1e-10 of the fixed point => within 2e-10 of each other
    assert np.abs(x64 - x32).sum() <= 2 * L1_TOL
    assert s32.error_bound <= L1_TOL and s64.error_bound <= L1_TOL


@pytest.mark.parametrize("relabel", [0, 1])
def test_relabel_modes_match_oracle(cuda_ok, relabel):
    # degree-sorted internal ids must not change any result (caller ids out)
    ig.set_tuning("relabel", relabel)
    try:
        n = 20_000
        f, t = O.barabasi_game_bag(n, 5, False, True, 21)
        g = G(n, f, t, True)
        assert maxabs(ig.pagerank(g), O.pagerank(n, f, t, True)) <= PARITY
        w = O.uniform_weights(len(f), 8)
        assert maxabs(ig.pagerank_weighted(g, w), O.pagerank_weighted(n, f, t, True, w)) <= PARITY
        r = np.zeros(n)
        r[[5, 17, 19000]] = [1.0, 0.5, 2.0]
        assert maxabs(ig.personalized_pagerank(g, r, 0.8), O.personalized_pagerank(n, f, t, True, r, 0.8)) <= PARITY
        with ig.DeviceGraph.from_host(n, f, t, True) as dg:
            assert dg.relabelled == bool(relabel)
            tight, _, _ = O.pagerank_tight(n, f, t, True, tol=1e-15)
            x, _ = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
            assert np.abs(x - tight).sum() <= L1_TOL
            # a warm start in caller ids is honoured
            xs, st = dg.solve(ig.Options(stop=ig.STOP_ERROR_BOUND), start=tight)
            assert st.iterations <= 3 and np.abs(xs - tight).sum() <= L1_TOL
    finally:
        ig.reset_tuning()


def test_rmat_auto_relabel(cuda_ok):
    scale = 15
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=4)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        assert dg.relabelled
        x, _ = dg.solve(ig.Options())
    assert maxabs(x, O.pagerank(n, f, t, True)) <= PARITY


@pytest.mark.parametrize("directed", [True, False])
def test_relabel_order(cuda_ok, directed):
    # internal ids: on directed graphs the vertices with in-arcs first; then
    # out-degree descending, then caller id
    import ctypes as C
    import torch

    scale = 14
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=5)
    fa, ta = np.asarray(f, np.int64), np.asarray(t, np.int64)
    if directed:
        od, noin = np.bincount(fa, minlength=n), np.bincount(ta, minlength=n) == 0
    else:
        od = np.bincount(fa, minlength=n) + np.bincount(ta, minlength=n)
        noin = np.zeros(n, bool)
    want = np.lexsort((np.arange(n), -od, noin))
    ig.set_tuning("relabel", 1)
    try:
        with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
            assert dg.relabelled
            rp, col, perm, inv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
            L = ig.lib()
            L.prg_graph_device_csr.restype = C.c_int32
            L.prg_graph_device_csr.argtypes = [C.c_void_p] + [C.POINTER(C.c_void_p)] * 4
            assert L.prg_graph_device_csr(dg._h, C.byref(rp), C.byref(col), C.byref(perm), C.byref(inv)) == 0

            class _View:
                __cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (perm.value, False), "version": 3}

            got = torch.as_tensor(_View(), device="cuda").cpu().numpy()
            x, _ = dg.solve(ig.Options())
    finally:
        ig.reset_tuning()
    assert np.array_equal(got, want)
    # the rows with arcs are ids 0 .. k-1
    e = noin[got] if directed else od[got] == 0
    assert not e[: int((~e).sum())].any()
    assert maxabs(x, O.pagerank(n, f, t, directed)) <= PARITY


def test_shared_memory_hot_prefix_keeps_parity(cuda_ok):
    # the optional per-block shared-memory copy of the hot prefix changes where
    # gathers read from, never what they read
    ig.set_tuning("hot_cache", 2048)
    ig.set_tuning("relabel", 1)  # the hot prefix applies to degree-sorted ids
    try:
        n = 30_000
        f, t = O.barabasi_game_bag(n, 5, False, True, 23)
        g = G(n, f, t, True)
        assert maxabs(ig.pagerank(g), O.pagerank(n, f, t, True)) <= PARITY
        w = O.uniform_weights(len(f), 9)
        assert maxabs(ig.pagerank_weighted(g, w), O.pagerank_weighted(n, f, t, True, w)) <= PARITY
        with ig.DeviceGraph.from_host(n, f, t, True) as dg:
            assert dg.relabelled
            tight, _, _ = O.pagerank_tight(n, f, t, True, tol=1e-15)
            for prec in (ig.PRECISION_FP32_REFINED, ig.PRECISION_FP64_KRYLOV):
                x, st = dg.solve(ig.Options(precision=prec))
                assert np.abs(x - tight).sum() <= L1_TOL and st.error_bound <= L1_TOL
    finally:
        ig.reset_tuning()


def test_graph_methods_delegate(cuda_ok):
    # Graph.pagerank / .pagerank_weighted / .personalized_pagerank /
    # .pagerank_linsys call the free functions (graph.rs:1857-1859,
    # 5454-5456, 6285-6289, 7002-7004); personalized uses damping 0.85
    n = 2_000
    f, t = O.erdos_renyi_gnm(n, 12_000, False, False, 41)
    g = ig.Graph.from_edge_arrays(n, f, t, False)
    w = O.uniform_weights(len(f), 42)
    r = np.zeros(n)
    r[[3, 7, 1999]] = [1.0, 0.5, 0.5]
    assert np.abs(g.pagerank() - O.pagerank(n, f, t, False)).max() <= 1e-10
    assert np.abs(g.pagerank_weighted(w) - O.pagerank_weighted(n, f, t, False, w)).max() <= 1e-10
    assert np.abs(g.personalized_pagerank(r) - O.personalized_pagerank(n, f, t, False, r, 0.85)).max() \
        <= 1e-10
    assert np.array_equal(g.pagerank_linsys(), ig.pagerank_linsys(g))


@pytest.mark.parametrize("case", ["rmat", "er_sparse", "ba_undirected"])
def test_segmented_power_step_matches_row_block(cuda_ok, case):
    # The FP64 power step of unweighted graphs runs as the tile-segmented
    # pass (seg_plain64 = 1, the default) or the row-block kernel (0); both
    # meet the restatement of pagerank() / personalized_pagerank(), with the
    # same iteration count to within one
    if case == "rmat":
        n = 1 << 16
        f, t = O.rmat(16, 16 * n, seed=61)
        directed = True
    elif case == "er_sparse":
        n = 100_000
        f, t = O.erdos_renyi_gnm(n, 150_000, True, False, 62)
        directed = True
    else:
        n = 40_000
        f, t = O.barabasi_game_bag(n, 4, False, False, 63)
        directed = False
    ref, iters = O.pagerank(n, f, t, directed, return_iters=True)
    r = np.zeros(n)
    r[[1, 7, n - 1]] = [1.0, 2.0, 0.5]
    pref = O.personalized_pagerank(n, f, t, directed, r, 0.85)
    out = {}
    try:
        for seg in (1, 0):
            ig.set_tuning("seg_plain64", seg)
            with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
                x, st = dg.solve(ig.Options())
            g = G(n, f, t, directed)
            out[seg] = (x, st.iterations, ig.personalized_pagerank(g, r, 0.85))
    finally:
        ig.reset_tuning()
    for seg, (x, it, xp) in out.items():
        assert maxabs(x, ref) <= PARITY, seg
        assert abs(it - iters) <= 1, (seg, it, iters)
        assert maxabs(xp, pref) <= PARITY, seg
    assert maxabs(out[1][0], out[0][0]) <= 1e-13
