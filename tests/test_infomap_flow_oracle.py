"""The CPU restatement of Infomap's flow model (oracle/prg_oracle.c,
or_infomap_flow; rust-igraph community/infomap.rs:233-355).  The reference
keeps the function private and its tests check memberships only, so the
restatement is pinned by properties of the reference's equations: without
dangling vertices and with uniform teleportation it is the reference's
pagerank (d = 0.85, itself pinned to the conformance fixtures); a two-vertex
path has a closed form; flows always sum to 1."""
import math

import numpy as np

import oracle as O


def E(pairs):
    a = np.array(pairs, np.uint32).reshape(-1, 2)
    return a[:, 0].copy(), a[:, 1].copy()


def test_two_vertex_path_closed_form():
    # p0 (1 + 0.15 p1) = 0.075 + 0.5 p1 with p1 = 1 - p0
    x, it = O.infomap_flow(2, *E([(0, 1)]), True)
    p0 = (1.65 - math.sqrt(1.65 ** 2 - 4 * 0.15 * 0.575)) / 0.3
    assert abs(x[0] - p0) < 1e-11 and abs(x[1] - (1 - p0)) < 1e-11 and it < 1000


def test_equals_pagerank_without_dangling_vertices():
    n = 2000
    f, t = O.erdos_renyi_gnm(n, 20000, False, False, 5)
    x, _ = O.infomap_flow(n, f, t, False)
    assert np.abs(x - O.pagerank(n, f, t, False)).max() < 1e-12
    # directed: a ring plus random arcs, so every vertex has out-arcs
    rng = np.random.default_rng(3)
    f = np.concatenate([np.arange(n), rng.integers(0, n, 8000)]).astype(np.uint32)
    t = np.concatenate([(np.arange(n) + 1) % n, rng.integers(0, n, 8000)]).astype(np.uint32)
    x, _ = O.infomap_flow(n, f, t, True)
    assert np.abs(x - O.pagerank(n, f, t, True)).max() < 1e-12


def test_weights_and_teleportation():
    n = 500
    f, t = O.erdos_renyi_gnm(n, 1500, True, False, 9)  # dangling vertices present
    x, _ = O.infomap_flow(n, f, t, True)
    assert abs(x.sum() - 1.0) < 1e-12 and x.min() > 0
    xw, _ = O.infomap_flow(n, f, t, True, edge_weights=np.ones(len(f)))
    assert np.array_equal(x, xw)  # unit weights are the unweighted model
    xv, _ = O.infomap_flow(n, f, t, True, vertex_weights=np.full(n, 7.0))
    assert np.abs(xv - x).max() < 1e-15  # uniform teleport weights of any scale
    vw = np.random.default_rng(1).random(n)
    xv, _ = O.infomap_flow(n, f, t, True, vertex_weights=vw)
    assert abs(xv.sum() - 1.0) < 1e-12 and np.abs(xv - x).max() > 1e-6
    # no edges: every vertex is dangling and the flow is the teleport distribution
    x0, it = O.infomap_flow(4, *E([]), True, vertex_weights=[1.0, 2.0, 3.0, 4.0])
    assert np.abs(x0 - np.array([0.1, 0.2, 0.3, 0.4])).max() < 1e-15
