"""GPU Infomap flow model (prg_infomap_flow; rust-igraph community/infomap.rs:
233-355) against its CPU restatement.  Both stop at an L1 change < 1e-10, so
the flows agree to <= 1e-10 max-abs and the iteration counts to within one
(the GPU sums rows in CSR order, the reference in ascending-source order)."""
import math

import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def check(n, f, t, directed, ew=None, vw=None):
    g = ig.Graph.from_edge_arrays(n, f, t, directed)
    gf, gt = g.edge_arrays()
    x, it = ig.infomap_flow(g, edge_weights=ew, vertex_weights=vw, with_iterations=True)
    ref, rit = O.infomap_flow(n, gf, gt, directed, edge_weights=ew, vertex_weights=vw)
    assert np.max(np.abs(x - ref)) <= TOL, np.max(np.abs(x - ref))
    assert abs(it - rit) <= 1, (it, rit)
    assert abs(x.sum() - 1.0) < 1e-12
    return x


def test_small_cases(cuda_ok):
    x = ig.infomap_flow(ig.Graph.from_edge_arrays(2, np.array([0], np.uint32), np.array([1], np.uint32), True))
    p0 = (1.65 - math.sqrt(1.65 ** 2 - 4 * 0.15 * 0.575)) / 0.3
    assert abs(x[0] - p0) < 1e-11 and abs(x[1] - (1 - p0)) < 1e-11
    g = ig.Graph.with_vertices(4)
    assert np.abs(ig.infomap_flow(g, vertex_weights=[1.0, 2.0, 3.0, 4.0]) - [0.1, 0.2, 0.3, 0.4]).max() < 1e-15
    assert np.abs(ig.infomap_flow(g) - 0.25).max() < 1e-15
    # two triangles joined by a bridge (the reference's doc example)
    pairs = [(0, 1), (0, 2), (1, 2), (3, 4), (3, 5), (4, 5), (2, 3)]
    f = np.array([p[0] for p in pairs], np.uint32)
    t = np.array([p[1] for p in pairs], np.uint32)
    check(6, f, t, False)
    check(6, f, t, False, ew=[10.0] * 6 + [0.01])
    check(6, f, t, True)


@pytest.mark.parametrize("kind", ["er_directed", "er_undirected", "ba_weighted", "rmat", "loops_vw"])
def test_matches_restatement(cuda_ok, kind):
    ew = vw = None
    if kind == "er_directed":
        n, directed = 20_000, True
        f, t = O.erdos_renyi_gnm(n, 60_000, True, False, 41)  # many dangling vertices
    elif kind == "er_undirected":
        n, directed = 20_000, False
        f, t = O.erdos_renyi_gnm(n, 30_000, False, False, 42)
    elif kind == "ba_weighted":
        n, directed = 50_000, False
        f, t = O.barabasi_game_bag(n, 4, True, False, 43)
        ew = O.uniform_weights(len(f), 44, 0.0, 2.0)
        ew[::13] = 0.0
    elif kind == "rmat":
        n, directed = 1 << 16, True
        f, t = O.rmat(16, 8 * n, seed=45)
    else:
        rng = np.random.default_rng(46)
        n, directed = 5000, False
        f = rng.integers(0, n, 20_000).astype(np.uint32)
        t = rng.integers(0, n, 20_000).astype(np.uint32)
        f[:300] = t[:300] = 11  # loops count twice in the strength
        vw = rng.random(n)
        vw[::5] = 0.0
    if ew is not None:
        # weights follow the canonical edge order the Graph mirror keeps
        g = ig.Graph.from_edge_arrays(n, f, t, directed)
        gf, gt = g.edge_arrays()
        check(n, gf, gt, directed, ew=ew)
    else:
        check(n, f, t, directed, vw=vw)


def test_unit_weights_match_unweighted(cuda_ok):
    n = 10_000
    f, t = O.erdos_renyi_gnm(n, 40_000, True, False, 47)
    g = ig.Graph.from_edge_arrays(n, f, t, True)
    a = ig.infomap_flow(g)
    b = ig.infomap_flow(g, edge_weights=np.ones(g.ecount()))
    assert np.max(np.abs(a - b)) <= 1e-15
