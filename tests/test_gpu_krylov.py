"""GPU Krylov solves of the PageRank linear system (krylov.cu) through the C ABI.

* FP32-refined (BiCGStab inner solves in FP32, FP64 residual passes) and FP64
  Krylov: L1 <= 1e-10 against the tight FP64 oracle, with a certified bound.
* pagerank_linsys() drop-in: the reference's own unit expectations
  (pagerank_linsys.rs:370-479), its parity contract with pagerank() on the
  reference fixtures (1e-9, pagerank_linsys.rs:25-30) and its stop rule
  ||b - A x||_2 < 1e-13 ||b||_2 re-checked in float64 on the CPU.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import igraph_b200 as ig
import oracle as O
from conftest import case_edges, within

pytestmark = pytest.mark.gpu

L1_TOL = 1e-10

FORMS = [
    pytest.param(dict(precision=ig.PRECISION_FP32_REFINED), id="fp32-krylov"),
    pytest.param(dict(precision=ig.PRECISION_FP32_REFINED, inner=ig.INNER_RICHARDSON), id="fp32-richardson"),
    pytest.param(dict(precision=ig.PRECISION_FP64_KRYLOV), id="fp64-krylov"),
]


def _check(x, st, tight):
    assert np.abs(x - tight).sum() <= L1_TOL, (np.abs(x - tight).sum(), st)
    assert st.error_bound <= L1_TOL
    assert abs(x.sum() - 1.0) < 1e-12


@pytest.mark.parametrize("form", FORMS)
def test_krylov_forms_directed_rmat(cuda_ok, form):
    scale = 15
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=31)
    tight, _, _ = O.pagerank_tight(n, f, t, True, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        x, st = dg.solve(ig.Options(**form))
    _check(x, st, tight)


@pytest.mark.parametrize("form", FORMS)
def test_krylov_forms_weighted_and_personalized(cuda_ok, form):
    n = 20_000
    f, t = O.barabasi_game_bag(n, 6, False, False, 2)
    w = O.uniform_weights(len(f), 4)
    tight, _, _ = O.pagerank_tight(n, f, t, False, weights=w, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, False, weights=w) as dg:
        x, st = dg.solve(ig.Options(**form))
    _check(x, st, tight)
    r = np.zeros(n)
    r[[1, 50, 999]] = [1.0, 2.0, 0.5]
    tight, _, _ = O.pagerank_tight(n, f, t, False, reset=r, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, False) as dg:
        x, st = dg.solve(ig.Options(**form), reset=r)
    _check(x, st, tight)


@pytest.mark.parametrize("form", FORMS)
def test_krylov_forms_loops_dangling_isolated(cuda_ok, form):
    rng = np.random.default_rng(7)
    n = 5000
    f = rng.integers(0, n // 2, 40_000).astype(np.uint32)  # upper half: dangling or isolated
    t = rng.integers(0, n, 40_000).astype(np.uint32)
    f[:300] = t[:300] = 3  # self-loops on one vertex, repeated
    f[300:3300] = 11  # a hub source
    tight, _, _ = O.pagerank_tight(n, f, t, True, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        x, st = dg.solve(ig.Options(**form))
    _check(x, st, tight)


def test_krylov_warm_start_and_pass_counts(cuda_ok):
    scale = 14
    n = 1 << scale
    f, t = O.rmat(scale, 16 * n, seed=5)
    tight, _, _ = O.pagerank_tight(n, f, t, True, tol=1e-15)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        x, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
        _, sp64 = dg.solve(ig.Options(stop=ig.STOP_ERROR_BOUND))
        xs, ss = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED), start=tight)
    _check(x, st, tight)
    # a few FP32 inner solves (each a relative reduction of at most ~1e-7, the
    # FP32 rounding level) between FP64 residual passes; on this small graph
    # the power iteration needs about as many passes, the gain comes at scale
    assert 2 <= st.residual_passes <= 5 and st.fp32_passes <= 2 * sp64.iterations, (st, sp64)
    # a start at the fixed point is certified by the first residual pass
    assert ss.fp32_passes == 0 and ss.residual_passes == 1
    assert np.abs(xs - tight).sum() <= L1_TOL


def test_krylov_device_rmat_scale20(cuda_ok):
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
    xs = {}
    for name, form in (("k32", dict(precision=ig.PRECISION_FP32_REFINED)),
                       ("k64", dict(precision=ig.PRECISION_FP64_KRYLOV))):
        st = dg.solve_device(out.data_ptr(), ig.Options(**form))
        xs[name] = out.cpu().numpy().copy()
        assert st.error_bound <= L1_TOL
        assert st.iterations < s64.iterations
    dg.close()
    for x in xs.values():
        assert abs(x.sum() - 1) < 1e-12 and np.all(x > 0)
        # both certified within 1e-10 of the fixed point
        assert np.abs(x - x64).sum() <= 2 * L1_TOL


# ---------------------------------------------------------------- linsys


def _g(n, edges, directed=False):
    g = ig.Graph.new(n, directed)
    g.add_edges(edges)
    return g


def test_linsys_reference_unit_cases(cuda_ok):
    # pagerank_linsys.rs:370-479
    assert np.allclose(ig.pagerank_linsys(ig.Graph.with_vertices(4)), 0.25, atol=1e-12, rtol=0)
    tri = _g(3, [(0, 1), (1, 2), (2, 0)])
    assert np.allclose(ig.pagerank_linsys(tri), 1 / 3, atol=1e-12, rtol=0)
    assert np.allclose(ig.pagerank_linsys(tri), ig.pagerank(tri), atol=1e-12, rtol=0)
    cyc = _g(4, [(i, (i + 1) % 4) for i in range(4)], directed=True)
    assert np.allclose(ig.pagerank_linsys(cyc), 0.25, atol=1e-12, rtol=0)
    for g in (_g(4, [(0, 1), (0, 2), (1, 2), (1, 3), (2, 3)]), _g(2, [(0, 1)], directed=True),
              _g(8, [(0, v) for v in range(1, 8)])):
        assert np.allclose(ig.pagerank_linsys(g), ig.pagerank(g), atol=1e-9, rtol=0)
    ring = _g(6, [(i, (i + 1) % 6) for i in range(6)])
    assert abs(ig.pagerank_linsys(ring).sum() - 1.0) < 1e-9


def test_linsys_matches_pagerank_fixtures(cuda_ok, golden_cases):
    # the reference pins linsys to pagerank() within 1e-9 on the pagerank fixtures
    seen = 0
    for case in golden_cases:
        if case["algo"] != "pagerank":
            continue
        f, t = case_edges(case)
        g = ig.Graph.from_edge_arrays(case["n"], f, t, case["directed"])
        got = ig.pagerank_linsys(g)
        assert within(got, case["expected"], case["tol_kind"], max(case["tol_tol"], 1e-9)), case["name"]
        tight, _, _ = O.pagerank_tight(case["n"], f, t, case["directed"], tol=1e-15)
        assert np.max(np.abs(got - tight)) <= 1e-12, case["name"]
        seen += 1
    assert seen >= 3


def _linsys_residual(n, f, t, directed, x, d=0.85):
    """||b - A x||_2 / ||b||_2 in float64 (pagerank_linsys.rs:221-238)."""
    f = f.astype(np.int64)
    t = t.astype(np.int64)
    if not directed:
        f, t = np.concatenate([f, t]), np.concatenate([t, f])
    deg = np.bincount(f, minlength=n).astype(np.float64)
    inv = np.where(deg > 0, 1.0 / np.maximum(deg, 1.0), 0.0)
    P = sp.csr_matrix((inv[f], (t, f)), shape=(n, n))
    dang = x[deg == 0].sum()
    ax = x - d * (P @ x) - d * dang / n
    b = np.full(n, (1 - d) / n)
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


@pytest.mark.parametrize("directed", [True, False])
def test_linsys_stop_rule_erdos_renyi(cuda_ok, directed):
    n, m = 10_000, 100_000
    f, t = O.erdos_renyi_gnm(n, m, directed, False, 17)
    g = ig.Graph.from_edge_arrays(n, f, t, directed)
    x = ig.pagerank_linsys(g)
    assert _linsys_residual(n, f, t, directed, x) < 3e-13
    tight, _, _ = O.pagerank_tight(n, f, t, directed, tol=1e-15)
    assert np.max(np.abs(x - tight)) <= 1e-13
    # the power-iteration drop-in agrees within the reference's 1e-9 contract
    assert np.max(np.abs(x - ig.pagerank(g))) <= 1e-9


@pytest.mark.parametrize("case", ["rmat_relabelled", "star_hub", "tiny", "sparse_many_empty", "undirected_ba"])
def test_segmented_fp32_matvec_matches_row_block_kernel(cuda_ok, case):
    # The FP32 Krylov matvec of unweighted graphs runs as the tile-segmented
    # pass (segspmv.cu, tuning seg_kry32 = 1, the default) or as the
    # row-block kernel (0).  Both refined solves meet the tight oracle, and
    # the segmented one is bit-reproducible.  The cases cover rows that span
    # many tiles (a hub with every arc), graphs smaller than one tile, rows
    # without arcs, and undirected graphs.
    directed = True
    if case == "rmat_relabelled":
        n = 1 << 15
        f, t = O.rmat(15, 16 * n, seed=44)
    elif case == "star_hub":
        n = 5000
        f = np.arange(1, n, dtype=np.uint32).repeat(3)
        t = np.zeros(len(f), np.uint32)
        f = np.concatenate([f, np.array([0, 0, 7], np.uint32)])
        t = np.concatenate([t, np.array([1, 2, 3], np.uint32)])
    elif case == "tiny":
        n = 40
        f, t = O.erdos_renyi_gnm(n, 120, True, False, 3)
    elif case == "sparse_many_empty":
        n = 200_000
        f, t = O.erdos_renyi_gnm(n, 150_000, True, False, 9)
    else:
        n = 30_000
        f, t = O.barabasi_game_bag(n, 5, False, False, 12)
        directed = False
    tight, _, _ = O.pagerank_tight(n, f, t, directed, tol=1e-15)
    xs = {}
    try:
        # (seg_kry32, seg_res64): both segmented passes, the 4-arc-quad
        # matvec, the row-block kernels only
        for seg in ((2, 1), (1, 1), (0, 0)):
            ig.set_tuning("seg_kry32", seg[0])
            ig.set_tuning("seg_res64", seg[1])
            with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
                x, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
                assert np.abs(x - tight).sum() <= 1e-10, (seg, np.abs(x - tight).sum())
                assert st.error_bound <= 1e-10
                if seg[0]:
                    x2, _ = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
                    assert np.array_equal(x.view(np.uint64), x2.view(np.uint64))
                xs[seg] = x
    finally:
        ig.reset_tuning()
    for seg in ((2, 1), (1, 1)):
        assert np.abs(xs[seg] - xs[(0, 0)]).sum() <= 2e-10


def _power_step(n, f, t, directed, x, d=0.85):
    """G(x) of pagerank.rs:107-140 in float64 (numpy)."""
    f = np.asarray(f, np.int64)
    t = np.asarray(t, np.int64)
    if directed:
        deg = np.bincount(f, minlength=n)
        src, dst = f, t
    else:
        deg = np.bincount(f, minlength=n) + np.bincount(t, minlength=n)
        src, dst = np.concatenate([f, t]), np.concatenate([t, f])
    xt = np.where(deg > 0, x / np.maximum(deg, 1), 0.0)
    y = np.bincount(dst, weights=xt[src], minlength=n)
    return (1.0 - d) / n + d * (y + x[deg == 0].sum() / n)


@pytest.mark.parametrize("case", ["rmat_relabelled", "star_hub", "sparse_many_empty", "undirected_ba"])
@pytest.mark.parametrize("seg_res64", [1, 0])
def test_residual_pass_matches_fp64_restatement(cuda_ok, case, seg_res64):
    # The FP64 residual pass (the tile-segmented one by default on unweighted
    # graphs, or the row-block kernel) gives the certificate
    # ||x - x*||_1 <= ||G(x) - x||_1 d / (1 - d).  From a start within the
    # final threshold the refined solve stops after that one pass, so its
    # residual_l1 is ||G(x0) - x0||_1, checked here against numpy.
    directed = True
    if case == "rmat_relabelled":  # n above the FP64 hot prefix: both gather paths
        n = 1 << 17
        f, t = O.rmat(17, 16 * n, seed=45)
    elif case == "star_hub":
        n = 5000
        f = np.arange(1, n, dtype=np.uint32).repeat(3)
        t = np.zeros(len(f), np.uint32)
    elif case == "sparse_many_empty":
        n = 200_000
        f, t = O.erdos_renyi_gnm(n, 150_000, True, False, 10)
    else:
        n = 30_000
        f, t = O.barabasi_game_bag(n, 5, False, False, 13)
        directed = False
    tight, _, _ = O.pagerank_tight(n, f, t, directed, tol=1e-15)
    rng = np.random.default_rng(3)
    x0 = tight * (1.0 + 2e-12 * rng.standard_normal(n))
    want = np.abs(_power_step(n, f, t, directed, x0) - x0).sum()
    ig.set_tuning("seg_res64", seg_res64)
    try:
        with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
            x, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED), start=x0)
    finally:
        ig.reset_tuning()
    assert st.residual_passes == 1 and st.fp32_passes == 0, st
    assert abs(st.residual_l1 - want) <= 1e-3 * want + 1e-15, (st.residual_l1, want)
    assert np.abs(x - tight).sum() <= 1e-10
