"""ctypes binding for the CPU oracle (``prg_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, and there only as the checker or the
timed CPU baseline.  The product library never calls it.

Functions mirror the reference's (rust-igraph) arithmetic; see the citations
in ``prg_oracle.c``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "prg_oracle.c")
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_splitmix_next.restype = C.c_uint64
        L.or_splitmix_next.argtypes = [C.POINTER(C.c_uint64)]
        L.or_splitmix_unit.restype = C.c_double
        L.or_splitmix_unit.argtypes = [C.POINTER(C.c_uint64)]
        pp = C.POINTER(C.POINTER(C.c_uint32))
        L.or_er_gnm.restype = C.c_int64
        L.or_er_gnm.argtypes = [C.c_uint32, C.c_uint64, C.c_int, C.c_int, C.c_uint64, pp, pp]
        L.or_ba_bag.restype = C.c_int64
        L.or_ba_bag.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_uint64, pp, pp]
        L.or_sbm.restype = C.c_int64
        L.or_sbm.argtypes = [C.c_uint32, _f64p, _u32p, C.c_int, C.c_int, C.c_int, C.c_uint64, pp, pp]
        L.or_rmat.restype = None
        L.or_rmat.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                              _u32p, _u32p, C.c_int]
        L.or_uniform_weights.restype = None
        L.or_uniform_weights.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, _f64p]
        L.or_ppr_residuals.restype = C.c_int
        L.or_ppr_residuals.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, C.c_uint32, C.c_void_p,
                                       C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        L.or_free.restype = None
        L.or_free.argtypes = [C.c_void_p]
        L.or_pagerank.restype = C.c_int
        L.or_pagerank.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, _f64p, C.POINTER(C.c_uint32)]
        L.or_pagerank_weighted.restype = C.c_int
        L.or_pagerank_weighted.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, _f64p, _f64p,
                                           C.POINTER(C.c_uint32)]
        L.or_personalized_pagerank.restype = C.c_int
        L.or_personalized_pagerank.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, _f64p, C.c_double,
                                               _f64p, C.POINTER(C.c_uint32)]
        L.or_pagerank_tight.restype = C.c_int64
        L.or_pagerank_tight.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_double, C.c_uint32, C.c_int, _f64p,
                                        C.POINTER(C.c_double), C.c_int]
        L.or_eigenvector_centrality.restype = C.c_int
        L.or_eigenvector_centrality.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, _f64p, C.POINTER(C.c_double)]
        L.or_hits.restype = C.c_int
        L.or_hits.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, _f64p, _f64p, C.POINTER(C.c_double)]
        L.or_eigenvector_weighted.restype = C.c_int
        L.or_eigenvector_weighted.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, _f64p, _f64p,
                                              C.POINTER(C.c_double)]
        L.or_hits_weighted.restype = C.c_int
        L.or_hits_weighted.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, _f64p, C.c_int, _f64p, _f64p,
                                       C.POINTER(C.c_double)]
        L.or_eigenvector_full.restype = C.c_int
        L.or_eigenvector_full.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, C.c_int, C.c_void_p,
                                          _f64p, C.POINTER(C.c_double)]
        L.or_infomap_flow.restype = C.c_int
        L.or_infomap_flow.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int, C.c_void_p, C.c_void_p,
                                      _f64p]
        L.or_adj_build.restype = C.c_void_p
        L.or_adj_build.argtypes = [C.c_uint32, C.c_uint64, _u32p, _u32p, C.c_int]
        L.or_adj_free.restype = None
        L.or_adj_free.argtypes = [C.c_void_p]
        L.or_adj_arcs.restype = C.c_uint64
        L.or_adj_arcs.argtypes = [C.c_void_p]
        L.or_adj_iterate.restype = C.c_double
        L.or_adj_iterate.argtypes = [C.c_void_p, C.c_uint32, _f64p]
        _lib = L
    return _lib


# ---------------------------------------------------------------- RNG / generators

def splitmix_stream(seed: int, count: int) -> list[int]:
    st = C.c_uint64(seed)
    return [lib().or_splitmix_next(C.byref(st)) for _ in range(count)]


def _take_edges(cnt, pf, pt):
    if cnt < 0:
        raise ValueError(f"generator failed ({cnt})")
    f = np.ctypeslib.as_array(pf, shape=(max(cnt, 1),))[:cnt].copy()
    t = np.ctypeslib.as_array(pt, shape=(max(cnt, 1),))[:cnt].copy()
    lib().or_free(C.cast(pf, C.c_void_p))
    lib().or_free(C.cast(pt, C.c_void_p))
    return f.astype(np.uint32), t.astype(np.uint32)


def erdos_renyi_gnm(n: int, m: int, directed: bool, loops: bool, seed: int):
    """Edge list of rust-igraph erdos_renyi_gnm (erdos_renyi.rs:328-353)."""
    pf, pt = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    cnt = lib().or_er_gnm(n, m, int(directed), int(loops), seed, C.byref(pf), C.byref(pt))
    return _take_edges(cnt, pf, pt)


def barabasi_game_bag(n: int, m: int, outpref: bool, directed: bool, seed: int):
    """Edge list of rust-igraph barabasi_game_bag (barabasi.rs:114-179)."""
    pf, pt = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    cnt = lib().or_ba_bag(n, m, int(outpref), int(directed), seed, C.byref(pf), C.byref(pt))
    return _take_edges(cnt, pf, pt)


def sbm_game(pref, sizes, directed: bool, loops: bool, multiple: bool, seed: int):
    """Edge list of rust-igraph sbm_game (sbm.rs:307-372)."""
    k = len(sizes)
    P = np.ascontiguousarray(np.asarray(pref, dtype=np.float64).reshape(k * k) if k else np.zeros(1))
    S = np.ascontiguousarray(np.asarray(sizes, dtype=np.uint32) if k else np.zeros(1, np.uint32))
    pf, pt = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    cnt = lib().or_sbm(k, P, S, int(directed), int(loops), int(multiple), seed, C.byref(pf), C.byref(pt))
    return _take_edges(cnt, pf, pt)


def rmat(scale: int, m: int, a=0.57, b=0.19, c=0.19, seed=1, nthreads=0):
    """Project R-MAT edge list (counter-based; matches the CUDA generator)."""
    f = np.empty(m, np.uint32)
    t = np.empty(m, np.uint32)
    lib().or_rmat(scale, m, a, b, c, seed, f, t, nthreads or (os.cpu_count() or 1))
    return f, t


def uniform_weights(m: int, seed: int, lo=0.5, hi=2.0):
    w = np.empty(max(m, 1), np.float64)
    lib().or_uniform_weights(m, seed, lo, hi, w)
    return w[:m]


# ---------------------------------------------------------------- restatements

def _edges(frm, to):
    return (np.ascontiguousarray(frm, dtype=np.uint32), np.ascontiguousarray(to, dtype=np.uint32))


def pagerank(n, frm, to, directed, return_iters=False):
    """Restatement of rust-igraph pagerank() (pagerank.rs:52-143)."""
    f, t = _edges(frm, to)
    out = np.zeros(max(n, 1), np.float64)
    it = C.c_uint32(0)
    lib().or_pagerank(n, len(f), f, t, int(directed), out, C.byref(it))
    out = out[:n]
    return (out, it.value) if return_iters else out


def pagerank_weighted(n, frm, to, directed, weights, return_iters=False):
    """Restatement of rust-igraph pagerank_weighted() (pagerank_weighted.rs:52-161)."""
    f, t = _edges(frm, to)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    if len(w) == 0:
        w = np.zeros(1)
    out = np.zeros(max(n, 1), np.float64)
    it = C.c_uint32(0)
    lib().or_pagerank_weighted(n, len(f), f, t, int(directed), w, out, C.byref(it))
    out = out[:n]
    return (out, it.value) if return_iters else out


def personalized_pagerank(n, frm, to, directed, reset, damping, return_iters=False):
    """Restatement of rust-igraph personalized_pagerank() (personalized_pagerank.rs:65-182)."""
    f, t = _edges(frm, to)
    r = np.ascontiguousarray(reset, dtype=np.float64)
    if len(r) == 0:
        r = np.zeros(1)
    out = np.zeros(max(n, 1), np.float64)
    it = C.c_uint32(0)
    lib().or_personalized_pagerank(n, len(f), f, t, int(directed), r, damping, out, C.byref(it))
    out = out[:n]
    return (out, it.value) if return_iters else out


def eigenvector_centrality(n, frm, to):
    """rust-igraph eigenvector_centrality (undirected, unweighted; eigenvector.rs:286-372):
    (vector, eigenvalue, iterations)."""
    f, t = _edges(frm, to)
    out = np.zeros(max(n, 1), np.float64)
    lam = C.c_double(0.0)
    it = lib().or_eigenvector_centrality(n, len(f), f, t, out, C.byref(lam))
    return out[:n], lam.value, it


def hub_and_authority_scores(n, frm, to, directed):
    """rust-igraph hub_and_authority_scores (unweighted; hits.rs:122-230):
    (hub, authority, eigenvalue, iterations)."""
    f, t = _edges(frm, to)
    hub = np.zeros(max(n, 1), np.float64)
    auth = np.zeros(max(n, 1), np.float64)
    lam = C.c_double(0.0)
    it = lib().or_hits(n, len(f), f, t, int(directed), hub, auth, C.byref(lam))
    return hub[:n], auth[:n], lam.value, it


def eigenvector_centrality_weighted(n, frm, to, weights):
    """rust-igraph eigenvector_centrality_weighted, non-negative weights
    (eigenvector.rs:375-538): (vector, eigenvalue, iterations)."""
    f, t = _edges(frm, to)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros(max(n, 1), np.float64)
    lam = C.c_double(0.0)
    it = lib().or_eigenvector_weighted(n, len(f), f, t, w if len(w) else np.zeros(1), out, C.byref(lam))
    return out[:n], lam.value, it


def hub_and_authority_scores_weighted(n, frm, to, weights, directed):
    """rust-igraph hub_and_authority_scores_weighted, non-negative weights
    (hits.rs:245-470): (hub, authority, eigenvalue, iterations)."""
    f, t = _edges(frm, to)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    hub = np.zeros(max(n, 1), np.float64)
    auth = np.zeros(max(n, 1), np.float64)
    lam = C.c_double(0.0)
    it = lib().or_hits_weighted(n, len(f), f, t, w if len(w) else np.zeros(1), int(directed), hub, auth,
                                C.byref(lam))
    return hub[:n], auth[:n], lam.value, it


EIG_OUT, EIG_IN, EIG_ALL = 0, 1, 2


def eigenvector_centrality_full(n, frm, to, directed, mode, weights=None):
    """rust-igraph eigenvector_centrality_full (eigenvector.rs:238-285,
    539-756), non-negative weights: (vector, eigenvalue, iterations)."""
    f, t = _edges(frm, to)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros(max(n, 1), np.float64)
    lam = C.c_double(0.0)
    it = lib().or_eigenvector_full(n, len(f), f, t, int(directed), int(mode),
                                   None if w is None else w.ctypes.data_as(C.c_void_p), out, C.byref(lam))
    return out[:n], lam.value, it


def infomap_flow(n, frm, to, directed, edge_weights=None, vertex_weights=None):
    """Node flows of rust-igraph's Infomap flow model (infomap.rs:233-355):
    (flow, iterations)."""
    f, t = _edges(frm, to)
    ew = None if edge_weights is None else np.ascontiguousarray(edge_weights, dtype=np.float64)
    vw = None if vertex_weights is None else np.ascontiguousarray(vertex_weights, dtype=np.float64)
    out = np.zeros(max(n, 1), np.float64)
    it = lib().or_infomap_flow(n, len(f), f, t, int(directed),
                               None if ew is None else ew.ctypes.data_as(C.c_void_p),
                               None if vw is None else vw.ctypes.data_as(C.c_void_p), out)
    return out[:n], int(it)


def pagerank_tight(n, frm, to, directed, weights=None, reset=None, damping=0.85, tol=1e-14,
                   max_iter=5000, start=None, nthreads=0):
    """Tight FP64 fixed point (compensated sums).  Returns (x, iterations, last_diff)."""
    f, t = _edges(frm, to)
    out = np.zeros(max(n, 1), np.float64)
    if start is not None:
        out[:n] = start
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    r = None if reset is None else np.ascontiguousarray(reset, dtype=np.float64)
    ld = C.c_double(0)
    it = lib().or_pagerank_tight(
        n, len(f), f, t, int(directed),
        None if w is None else w.ctypes.data_as(C.c_void_p),
        None if r is None else r.ctypes.data_as(C.c_void_p),
        damping, tol, max_iter, int(start is not None), out, C.byref(ld), nthreads or (os.cpu_count() or 1))
    return out[:n], int(it), ld.value


def ppr_residuals(n, frm, to, directed, seed_lists, X, damping=0.85, nthreads=0):
    """||G_k(x_k) - x_k||_1 per column of a batched result X (float32 [n, K])
    under the personalized_pagerank operator with the _vs reset of each
    seed list; ||x_k - x*_k||_1 <= res / (1 - damping)."""
    f, t = _edges(frm, to)
    K = len(seed_lists)
    off = np.zeros(K + 1, np.uint64)
    off[1:] = np.cumsum([len(x) for x in seed_lists])
    seeds = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint32) for x in seed_lists]), dtype=np.uint32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    assert X.shape == (n, K)
    res = np.zeros(K, np.float64)
    L = lib()
    L.or_ppr_residuals(n, len(f), f, t, int(directed), K, off.ctypes.data_as(C.c_void_p),
                       seeds.ctypes.data_as(C.c_void_p), damping, X.ctypes.data_as(C.c_void_p),
                       res.ctypes.data_as(C.c_void_p), nthreads or (os.cpu_count() or 1))
    return res


class RefAdjacency:
    """Prebuilt reference in-adjacency for timing the CPU baseline loop."""

    def __init__(self, n, frm, to, directed):
        f, t = _edges(frm, to)
        self.n = n
        self.h = lib().or_adj_build(n, len(f), f, t, int(directed))
        self.arcs = lib().or_adj_arcs(self.h)

    def iterate(self, iters, pr):
        return lib().or_adj_iterate(self.h, iters, pr)

    def close(self):
        if self.h:
            lib().or_adj_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
