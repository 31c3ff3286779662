"""Python host side of the B200 PageRank library.

Mirrors the slice of rust-igraph's public API that the PageRank hot path
uses, with the same names, argument meaning and error behaviour:

* ``Graph`` — ``with_vertices``, ``new``, ``add_edge``, ``add_edges``,
  ``vcount``, ``ecount``, ``is_directed``, ``edge`` (src/core/graph.rs:126-152,
  :518, :170, :740-785, :547, :564, :582, :1152).  Undirected edges are stored
  as (min, max) like ``Graph::add_edges``.
* ``pagerank``, ``pagerank_weighted``, ``personalized_pagerank``,
  ``personalized_pagerank_default``, ``personalized_pagerank_vs``
  (src/algorithms/properties/pagerank.rs:52, pagerank_weighted.rs:52,
  personalized_pagerank.rs:65, :206, :241) returning a float64 numpy array
  or raising the ``IgraphError`` subclass the reference would return.
* ``DeviceGraph`` — a graph kept resident in HBM for repeated solves with
  the extended options (FP32 + FP64-refined precision, error-bound stop,
  warm start) and the batched personalized solver.

Every call goes through ``libprg_b200.so`` (include/prg_b200.h).  There is no
CPU implementation here: if the library or a GPU is missing the call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Iterable, Optional, Sequence

import numpy as np

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_PKG_DIR), "libprg_b200.so")

# ------------------------------------------------------------------ errors


class IgraphError(Exception):
    """Base of the error variants (rust-igraph src/core/error.rs:14-66)."""


class InvalidArgument(IgraphError):
    pass


class VertexOutOfRange(IgraphError):
    pass


class Internal(IgraphError):
    pass


class DidNotConverge(IgraphError):
    pass


class DeviceTimeout(Internal):
    pass


class ParseError(IgraphError):
    """IgraphError::Parse { line, message } (displayed as the reference does)."""

    def __init__(self, line: int, message: str):
        super().__init__(f"parse error at line {line}: {message}")
        self.line = line
        self.message = message


class IoError(IgraphError):
    """IgraphError::Io."""


class Unsupported(IgraphError):
    """IgraphError::Unsupported."""


PRG_OK = 0
_ERRORS = {1: InvalidArgument, 2: VertexOutOfRange, 3: Internal, 4: Internal, 5: Internal, 6: DidNotConverge,
           7: DeviceTimeout, 9: IoError, 10: Unsupported}

# ------------------------------------------------------------------ library


class prg_options(C.Structure):
    _fields_ = [("damping", C.c_double), ("eps", C.c_double), ("max_iter", C.c_uint32),
                ("precision", C.c_int32), ("stop", C.c_int32), ("normalise", C.c_int32),
                ("start", C.c_void_p), ("inner", C.c_int32)]


class prg_stats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("fp64_passes", C.c_uint32), ("fp32_passes", C.c_uint32),
                ("residual_passes", C.c_uint32), ("last_diff", C.c_double), ("residual_l1", C.c_double),
                ("error_bound", C.c_double), ("solve_ms", C.c_double), ("build_ms", C.c_double),
                ("arcs", C.c_uint64), ("n_dangling", C.c_uint32), ("kernel_launches", C.c_uint32),
                ("fp32_ms", C.c_double), ("fp64_ms", C.c_double), ("spmv_ms", C.c_double),
                ("spmv_launches", C.c_uint32)]


class prg_batch_stats(C.Structure):
    _fields_ = [("column_iterations", C.c_uint64), ("max_iters", C.c_uint32), ("tiles", C.c_uint32),
                ("tile_width", C.c_uint32), ("kernel_launches", C.c_uint32), ("ms", C.c_double),
                ("chebyshev", C.c_uint32), ("pad", C.c_uint32)]


class prg_tune_result(C.Structure):
    _fields_ = [("capw", C.c_uint32), ("shortmax", C.c_uint32), ("split", C.c_uint32),
                ("blocks_per_sm", C.c_uint32), ("batch_tile_width", C.c_uint32), ("candidates", C.c_uint32),
                ("from_cache", C.c_int32), ("pad", C.c_uint32), ("default_ms", C.c_double), ("best_ms", C.c_double),
                ("seg_hot", C.c_uint32), ("seg_hot64", C.c_uint32), ("seg_default_ms", C.c_double),
                ("seg_best_ms", C.c_double)]


_lib = None


def library_path() -> str:
    return _LIB_PATH


def lib():
    """Loads libprg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python rust-igraph_b200/build.py`")
    L = C.CDLL(_LIB_PATH)
    u32p, f64p, vp = C.c_void_p, C.c_void_p, C.c_void_p
    L.prg_default_options.restype = None
    L.prg_default_options.argtypes = [C.POINTER(prg_options)]
    L.prg_last_error.restype = C.c_void_p
    L.prg_last_error.argtypes = []
    L.prg_last_error_len.restype = C.c_uint64
    L.prg_last_error_len.argtypes = []
    L.prg_pagerank.restype = C.c_int32
    L.prg_pagerank.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p]
    L.prg_pagerank_linsys.restype = C.c_int32
    L.prg_pagerank_linsys.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p]
    L.prg_pagerank_weighted.restype = C.c_int32
    L.prg_pagerank_weighted.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p, C.c_uint64, f64p]
    L.prg_personalized_pagerank.restype = C.c_int32
    L.prg_personalized_pagerank.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p, C.c_uint64,
                                            C.c_double, f64p]
    L.prg_personalized_pagerank_vs.restype = C.c_int32
    L.prg_personalized_pagerank_vs.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, u32p, C.c_uint64,
                                               C.c_double, f64p]
    L.prg_graph_create.restype = C.c_int32
    L.prg_graph_create.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, f64p, C.c_int32, C.POINTER(C.c_void_p)]
    L.prg_graph_create_device.restype = C.c_int32
    L.prg_graph_create_device.argtypes = [C.c_uint32, C.c_uint64, vp, vp, vp, C.c_int32, C.POINTER(C.c_void_p)]
    L.prg_graph_destroy.restype = None
    L.prg_graph_destroy.argtypes = [vp]
    L.prg_graph_info.restype = C.c_int32
    L.prg_graph_info.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
    L.prg_graph_stream.restype = C.c_void_p
    L.prg_graph_stream.argtypes = [vp]
    L.prg_solve.restype = C.c_int32
    L.prg_solve.argtypes = [vp, C.POINTER(prg_options), f64p, f64p, C.POINTER(prg_stats)]
    L.prg_solve_device.restype = C.c_int32
    L.prg_solve_device.argtypes = [vp, C.POINTER(prg_options), vp, vp, C.POINTER(prg_stats)]
    L.prg_set_tuning.restype = C.c_int32
    L.prg_set_tuning.argtypes = [C.c_char_p, C.c_int64]
    L.prg_graph_relabelled.restype = C.c_int32
    L.prg_graph_relabelled.argtypes = [vp]
    for name in ("prg_ppr_batch", "prg_ppr_batch_device"):
        f = getattr(L, name)
        f.restype = C.c_int32
        f.argtypes = [vp, C.c_uint32, vp, vp, C.c_double, C.c_double, C.c_uint32, C.c_uint32, vp, vp,
                      C.POINTER(prg_batch_stats)]
    L.prg_autotune.restype = C.c_int32
    L.prg_autotune.argtypes = [vp, C.c_int32, C.c_char_p, C.POINTER(prg_tune_result)]
    L.prg_generate_device.restype = C.c_int32
    L.prg_generate_device.argtypes = [C.c_int32, C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                      C.c_uint64, vp, vp, vp]
    L.prg_gnn_param_count.restype = C.c_uint32
    L.prg_gnn_param_count.argtypes = []
    L.prg_gnn_create.restype = C.c_int32
    L.prg_gnn_create.argtypes = [C.c_uint64, C.POINTER(C.c_void_p)]
    L.prg_gnn_destroy.restype = None
    L.prg_gnn_destroy.argtypes = [vp]
    L.prg_gnn_get_params.restype = C.c_int32
    L.prg_gnn_get_params.argtypes = [vp, vp]
    L.prg_gnn_set_params.restype = C.c_int32
    L.prg_gnn_set_params.argtypes = [vp, vp]
    L.prg_gnn_predict.restype = C.c_int32
    L.prg_gnn_predict.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
    L.prg_gnn_loss_grad.restype = C.c_int32
    L.prg_gnn_loss_grad.argtypes = [vp, vp, vp, C.POINTER(C.c_double), vp]
    L.prg_gnn_train_step.restype = C.c_int32
    L.prg_gnn_train_step.argtypes = [vp, vp, vp, C.c_float, C.POINTER(C.c_double)]
    L.prg_solve_noalloc.restype = C.c_int32
    L.prg_solve_noalloc.argtypes = [vp, C.POINTER(prg_options), vp, vp, C.POINTER(prg_stats)]
    L.prg_rmat_device.restype = C.c_int32
    L.prg_rmat_device.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                  vp, vp, vp]
    L.prg_eigenvector_centrality.restype = C.c_int32
    L.prg_eigenvector_centrality.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p,
                                             C.POINTER(C.c_double)]
    L.prg_eigenvector_centrality_weighted.restype = C.c_int32
    L.prg_eigenvector_centrality_weighted.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p,
                                                      C.c_uint64, f64p, f64p]
    L.prg_hub_and_authority_scores_weighted.restype = C.c_int32
    L.prg_hub_and_authority_scores_weighted.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p,
                                                        C.c_uint64, f64p, f64p, f64p]
    L.prg_eigenvector_centrality_full.restype = C.c_int32
    L.prg_eigenvector_centrality_full.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, C.c_int32, f64p,
                                                  C.c_uint64, f64p, f64p]
    L.prg_graph_gather_probe.restype = C.c_int32
    L.prg_graph_gather_probe.argtypes = [vp, C.c_int32, C.POINTER(C.c_double)]
    L.prg_graph_matvec32.restype = C.c_int32
    L.prg_graph_matvec32.argtypes = [vp, C.c_int32, vp, vp, C.c_double, C.c_double, vp, f64p,
                                     C.POINTER(C.c_double)]
    L.prg_graph_device_csr.restype = C.c_int32
    L.prg_graph_device_csr.argtypes = [vp] + [C.POINTER(vp)] * 4
    L.prg_infomap_flow.restype = C.c_int32
    L.prg_infomap_flow.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p, C.c_uint64, f64p,
                                   C.c_uint64, f64p, C.POINTER(C.c_uint32)]
    L.prg_hub_and_authority_scores.restype = C.c_int32
    L.prg_hub_and_authority_scores.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int32, f64p, f64p,
                                               C.POINTER(C.c_double)]
    L.prg_parse_edgelist.restype = C.c_int32
    L.prg_parse_edgelist.argtypes = [C.c_char_p, C.c_uint64, vp, vp, C.c_uint64, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.prg_read_edgelist.restype = C.c_int32
    L.prg_read_edgelist.argtypes = [C.c_char_p, C.c_uint64, C.POINTER(vp), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    _lib = L
    return L


def last_error() -> str:
    """The library's last error message on this thread (all of its bytes)."""
    L = lib()
    n = L.prg_last_error_len()
    return C.string_at(L.prg_last_error(), n).decode("utf-8", "replace") if n else ""


def _check(rc: int, err_line: int = 0) -> None:
    if rc != PRG_OK:
        msg = last_error()
        if rc == 8:
            raise ParseError(err_line, msg)
        raise _ERRORS.get(rc, Internal)(msg)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ Graph mirror


class Graph:
    """The edge-list view of rust-igraph's Graph that crosses the boundary."""

    def __init__(self, n: int = 0, directed: bool = False):
        self._n = int(n)
        self._directed = bool(directed)
        self._from: list[int] = []
        self._to: list[int] = []
        self._arr = None

    # constructors (graph.rs:170, :518)
    @classmethod
    def new(cls, n: int, directed: bool) -> "Graph":
        return cls(n, directed)

    @classmethod
    def with_vertices(cls, n: int) -> "Graph":
        return cls(n, False)

    @classmethod
    def from_edge_arrays(cls, n: int, frm, to, directed: bool) -> "Graph":
        """Bulk constructor equivalent to ``new(n, directed)`` + ``add_edges``."""
        g = cls(n, directed)
        f = np.ascontiguousarray(frm, dtype=np.uint32)
        t = np.ascontiguousarray(to, dtype=np.uint32)
        if f.shape != t.shape:
            raise InvalidArgument("from/to length mismatch")
        if len(f) and max(int(f.max()), int(t.max())) >= n:
            raise VertexOutOfRange(f"vertex out of range (vcount = {n})")
        if not directed:
            lo, hi = np.minimum(f, t), np.maximum(f, t)
            f, t = lo, hi
        g._arr = (f, t)
        return g

    def _materialise(self):
        if self._arr is None:
            self._arr = (np.asarray(self._from, dtype=np.uint32), np.asarray(self._to, dtype=np.uint32))
        return self._arr

    def add_edge(self, u: int, v: int) -> None:
        self.add_edges([(u, v)])

    def add_edges(self, edges: Iterable[Sequence[int]]) -> None:
        if self._arr is not None:
            f, t = self._arr
            self._from, self._to = f.tolist(), t.tolist()
            self._arr = None
        new = []
        for u, v in edges:
            if not (0 <= u < self._n):
                raise VertexOutOfRange(f"vertex {u} out of range (vcount = {self._n})")
            if not (0 <= v < self._n):
                raise VertexOutOfRange(f"vertex {v} out of range (vcount = {self._n})")
            new.append((v, u) if (not self._directed and u > v) else (u, v))
        for u, v in new:
            self._from.append(u)
            self._to.append(v)

    def vcount(self) -> int:
        return self._n

    def ecount(self) -> int:
        return len(self._materialise()[0]) if self._arr is not None else len(self._from)

    def is_directed(self) -> bool:
        return self._directed

    def edge(self, e: int):
        f, t = self._materialise()
        return int(f[e]), int(t[e])

    def edge_arrays(self):
        return self._materialise()


# ------------------------------------------------------------------ drop-ins

    # Graph methods that delegate to the free functions, as the reference's
    # do (src/core/graph.rs:1857-1859, 5454-5456, 6285-6289, 7002-7004).
    def pagerank(self) -> np.ndarray:
        return pagerank(self)

    def pagerank_weighted(self, weights) -> np.ndarray:
        return pagerank_weighted(self, weights)

    def personalized_pagerank(self, reset) -> np.ndarray:
        """personalized_pagerank_default: damping 0.85 (graph.rs:6285-6289)."""
        return personalized_pagerank_default(self, reset)

    def pagerank_linsys(self) -> np.ndarray:
        return pagerank_linsys(self)


def pagerank(graph: Graph) -> np.ndarray:
    """rust-igraph ``pagerank(&Graph)`` (pagerank.rs:52-143) on the GPU."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    out = np.empty(max(n, 1), np.float64)
    _check(lib().prg_pagerank(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), _ptr(out)))
    return out[:n]


def pagerank_linsys(graph: Graph) -> np.ndarray:
    """rust-igraph ``pagerank_linsys(&Graph)`` (pagerank_linsys.rs:99-160): the
    linear-system form solved on the GPU to ||b - Ax||_2 < 1e-13 ||b||_2."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    out = np.empty(max(n, 1), np.float64)
    _check(lib().prg_pagerank_linsys(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), _ptr(out)))
    return out[:n]


def eigenvector_centrality(graph: Graph, with_eigenvalue: bool = False):
    """rust-igraph ``eigenvector_centrality`` (eigenvector.rs:118-125, 286-372),
    undirected and unweighted, on the GPU.  with_eigenvalue: also return the
    Rayleigh quotient."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    out = np.empty(max(n, 1), np.float64)
    lam = C.c_double()
    _check(lib().prg_eigenvector_centrality(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), _ptr(out),
                                            C.byref(lam)))
    return (out[:n], lam.value) if with_eigenvalue else out[:n]


@dataclass
class HitsScores:
    hub: np.ndarray
    authority: np.ndarray
    eigenvalue: float


def hub_and_authority_scores(graph: Graph) -> HitsScores:
    """rust-igraph ``hub_and_authority_scores`` (hits.rs:122-230), unweighted, on the GPU."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    hub = np.empty(max(n, 1), np.float64)
    auth = np.empty(max(n, 1), np.float64)
    lam = C.c_double()
    _check(lib().prg_hub_and_authority_scores(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), _ptr(hub),
                                              _ptr(auth), C.byref(lam)))
    return HitsScores(hub[:n], auth[:n], lam.value)


def eigenvector_centrality_weighted(graph: Graph, weights, with_eigenvalue: bool = False):
    """rust-igraph ``eigenvector_centrality_weighted`` (eigenvector.rs:157-168,
    375-538), undirected, weights[e] >= 0 per edge id, on the GPU."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = np.empty(max(n, 1), np.float64)
    lam = C.c_double()
    _check(lib().prg_eigenvector_centrality_weighted(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()),
                                                     _ptr(w) if len(w) else None, len(w), _ptr(out), C.byref(lam)))
    return (out[:n], lam.value) if with_eigenvalue else out[:n]


EIG_OUT, EIG_IN, EIG_ALL = 0, 1, 2  # EigenvectorMode (eigenvector.rs:63-76)


@dataclass
class EigenvectorScores:
    vector: np.ndarray
    eigenvalue: float


def eigenvector_centrality_full(graph: Graph, mode: int, weights=None) -> EigenvectorScores:
    """rust-igraph ``eigenvector_centrality_full`` (eigenvector.rs:238-285) on
    the GPU; non-negative weights."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.empty(max(n, 1), np.float64)
    lam = C.c_double()
    _check(lib().prg_eigenvector_centrality_full(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), int(mode),
                                                 None if w is None else (_ptr(w) if len(w) else _ptr(np.zeros(1))),
                                                 0 if w is None else len(w), _ptr(out), C.byref(lam)))
    return EigenvectorScores(out[:n], lam.value)


def eigenvector_centrality_directed(graph: Graph, mode: int) -> EigenvectorScores:
    """rust-igraph ``eigenvector_centrality_directed`` (eigenvector.rs:189-194)."""
    return eigenvector_centrality_full(graph, mode)


def eigenvector_centrality_directed_weighted(graph: Graph, mode: int, weights) -> EigenvectorScores:
    """rust-igraph ``eigenvector_centrality_directed_weighted`` (eigenvector.rs:218-224)."""
    return eigenvector_centrality_full(graph, mode, weights)


def hub_and_authority_scores_weighted(graph: Graph, weights) -> HitsScores:
    """rust-igraph ``hub_and_authority_scores_weighted`` (hits.rs:245-470),
    weights[e] >= 0 per edge id, on the GPU."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    w = np.ascontiguousarray(weights, dtype=np.float64)
    hub = np.empty(max(n, 1), np.float64)
    auth = np.empty(max(n, 1), np.float64)
    lam = C.c_double()
    _check(lib().prg_hub_and_authority_scores_weighted(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()),
                                                       _ptr(w) if len(w) else None, len(w), _ptr(hub), _ptr(auth),
                                                       C.byref(lam)))
    return HitsScores(hub[:n], auth[:n], lam.value)


def infomap_flow(graph: Graph, edge_weights=None, vertex_weights=None, with_iterations: bool = False):
    """Node flows of rust-igraph's Infomap flow model (community/infomap.rs:
    233-355) on the GPU: tau = 0.15 teleportation to vertex_weights (uniform
    when None), arc weights edge_weights (unit when None)."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    ew = None if edge_weights is None else np.ascontiguousarray(edge_weights, dtype=np.float64)
    vw = None if vertex_weights is None else np.ascontiguousarray(vertex_weights, dtype=np.float64)
    out = np.empty(max(n, 1), np.float64)
    it = C.c_uint32()
    _check(lib().prg_infomap_flow(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()),
                                  None if ew is None else (_ptr(ew) if len(ew) else _ptr(np.zeros(1))),
                                  0 if ew is None else len(ew),
                                  None if vw is None else (_ptr(vw) if len(vw) else _ptr(np.zeros(1))),
                                  0 if vw is None else len(vw), _ptr(out), C.byref(it)))
    return (out[:n], it.value) if with_iterations else out[:n]


def parse_edgelist(data: bytes):
    """Edges of an edge-list text parsed on the GPU: (n, from, to) in file
    order (read_edgelist's rules, io/edgelist.rs:25-72)."""
    data = bytes(data)
    cap = data.count(b"\n") + 1
    f = np.empty(cap, np.uint32)
    t = np.empty(cap, np.uint32)
    m, n, line = C.c_uint64(), C.c_uint32(), C.c_uint64()
    _check(lib().prg_parse_edgelist(data, len(data), _ptr(f), _ptr(t), cap, C.byref(m), C.byref(n), C.byref(line)),
           line.value)
    return n.value, f[:m.value].copy(), t[:m.value].copy()


def read_edgelist(data: bytes) -> Graph:
    """rust-igraph ``read_edgelist`` (io/edgelist.rs:25-61): an undirected
    graph with n = max id + 1, parsed on the GPU."""
    n, f, t = parse_edgelist(data)
    return Graph.from_edge_arrays(n, f, t, False)


def pagerank_weighted(graph: Graph, weights) -> np.ndarray:
    """rust-igraph ``pagerank_weighted(&Graph, &[f64])`` (pagerank_weighted.rs:52-161)."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = np.empty(max(n, 1), np.float64)
    wp = _ptr(w) if len(w) else None
    _check(lib().prg_pagerank_weighted(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), wp, len(w),
                                       _ptr(out)))
    return out[:n]


def personalized_pagerank(graph: Graph, reset, damping: float) -> np.ndarray:
    """rust-igraph ``personalized_pagerank`` (personalized_pagerank.rs:65-182)."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    r = np.ascontiguousarray(reset, dtype=np.float64)
    out = np.empty(max(n, 1), np.float64)
    rp = _ptr(r) if len(r) else None
    _check(lib().prg_personalized_pagerank(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), rp, len(r),
                                           float(damping), _ptr(out)))
    return out[:n]


def personalized_pagerank_default(graph: Graph, reset) -> np.ndarray:
    """rust-igraph ``personalized_pagerank_default`` (personalized_pagerank.rs:206-208)."""
    return personalized_pagerank(graph, reset, 0.85)


def personalized_pagerank_vs(graph: Graph, reset_vids, damping: float) -> np.ndarray:
    """rust-igraph ``personalized_pagerank_vs`` (personalized_pagerank.rs:241-268)."""
    n = graph.vcount()
    f, t = graph.edge_arrays()
    v = np.ascontiguousarray(reset_vids, dtype=np.uint32)
    out = np.empty(max(n, 1), np.float64)
    vp = _ptr(v) if len(v) else None
    _check(lib().prg_personalized_pagerank_vs(n, len(f), _ptr(f), _ptr(t), int(graph.is_directed()), vp, len(v),
                                              float(damping), _ptr(out)))
    return out[:n]


# ------------------------------------------------------------------ resident graphs

PRECISION_FP64 = 0
PRECISION_FP32_REFINED = 1
PRECISION_FP64_KRYLOV = 2
PRECISION_LINSYS = 3
INNER_KRYLOV = 0
INNER_RICHARDSON = 1
STOP_SUCCESSIVE = 0
STOP_ERROR_BOUND = 1


@dataclass
class Options:
    damping: float = 0.85
    eps: float = 1e-10
    max_iter: int = 1000
    precision: int = PRECISION_FP64
    stop: int = STOP_SUCCESSIVE
    normalise: bool = True
    inner: int = INNER_KRYLOV

    def to_c(self, start_ptr=None) -> prg_options:
        o = prg_options()
        o.damping, o.eps, o.max_iter = self.damping, self.eps, self.max_iter
        o.precision, o.stop, o.normalise = self.precision, self.stop, int(self.normalise)
        o.start = start_ptr
        o.inner = self.inner
        return o


@dataclass
class Stats:
    iterations: int
    fp64_passes: int
    fp32_passes: int
    residual_passes: int
    last_diff: float
    residual_l1: float
    error_bound: float
    solve_ms: float
    build_ms: float
    arcs: int
    n_dangling: int
    kernel_launches: int
    fp32_ms: float
    fp64_ms: float
    spmv_ms: float = 0.0
    spmv_launches: int = 0

    @classmethod
    def from_c(cls, s: prg_stats) -> "Stats":
        return cls(s.iterations, s.fp64_passes, s.fp32_passes, s.residual_passes, s.last_diff, s.residual_l1,
                   s.error_bound, s.solve_ms, s.build_ms, s.arcs, s.n_dangling, s.kernel_launches, s.fp32_ms,
                   s.fp64_ms, s.spmv_ms, s.spmv_launches)


class DeviceGraph:
    """A graph resident in HBM (prg_graph handle)."""

    def __init__(self, handle):
        self._h = handle
        n, arcs, nd, nrb, nhub, bms = C.c_uint32(), C.c_uint64(), C.c_uint32(), C.c_uint32(), C.c_uint32(), \
            C.c_double()
        _check(lib().prg_graph_info(self._h, C.byref(n), C.byref(arcs), C.byref(nd), C.byref(nrb), C.byref(nhub),
                                    C.byref(bms)))
        self.n, self.arcs, self.n_dangling = n.value, arcs.value, nd.value
        self.n_rowblocks, self.n_hubs, self.build_ms = nrb.value, nhub.value, bms.value

    @classmethod
    def from_host(cls, n: int, frm, to, directed: bool, weights=None) -> "DeviceGraph":
        f = np.ascontiguousarray(frm, dtype=np.uint32)
        t = np.ascontiguousarray(to, dtype=np.uint32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        h = C.c_void_p()
        _check(lib().prg_graph_create(n, len(f), _ptr(f), _ptr(t), _ptr(w), int(directed), C.byref(h)))
        return cls(h)

    @classmethod
    def from_graph(cls, g: Graph, weights=None) -> "DeviceGraph":
        f, t = g.edge_arrays()
        return cls.from_host(g.vcount(), f, t, g.is_directed(), weights)

    @classmethod
    def from_edgelist(cls, data: bytes) -> Optional["DeviceGraph"]:
        """Resident graph straight from an edge-list text (prg_read_edgelist):
        parsed on the GPU, the edges never leave it.  None when the text has
        no edges."""
        data = bytes(data)
        h = C.c_void_p()
        n, m, line = C.c_uint32(), C.c_uint64(), C.c_uint64()
        _check(lib().prg_read_edgelist(data, len(data), C.byref(h), C.byref(n), C.byref(m), C.byref(line)),
               line.value)
        return cls(h) if h.value else None

    @classmethod
    def from_device(cls, n: int, m: int, d_from: int, d_to: int, directed: bool, d_weights: int = 0):
        h = C.c_void_p()
        _check(lib().prg_graph_create_device(n, m, C.c_void_p(d_from), C.c_void_p(d_to),
                                             C.c_void_p(d_weights) if d_weights else None, int(directed),
                                             C.byref(h)))
        return cls(h)

    @property
    def handle(self):
        return self._h

    @property
    def relabelled(self) -> bool:
        return bool(lib().prg_graph_relabelled(self._h))

    def stream(self) -> int:
        return lib().prg_graph_stream(self._h) or 0

    def solve(self, options: Optional[Options] = None, reset=None, start=None, out=None):
        """Host solve: returns (x float64[n], Stats).  `out` may be a caller
        float64 buffer (e.g. pinned memory) of length >= n."""
        o = options or Options()
        st = prg_stats()
        if out is None:
            out = np.empty(max(self.n, 1), np.float64)
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and len(out) >= self.n
        r = None if reset is None else np.ascontiguousarray(reset, dtype=np.float64)
        s0 = None if start is None else np.ascontiguousarray(start, dtype=np.float64)
        co = o.to_c(_ptr(s0))
        _check(lib().prg_solve(self._h, C.byref(co), _ptr(r), _ptr(out), C.byref(st)))
        return out[: self.n], Stats.from_c(st)

    def solve_device(self, d_out: int, options: Optional[Options] = None, d_reset: int = 0, d_start: int = 0):
        """Device solve into a device pointer (e.g. a torch tensor's data_ptr())."""
        o = options or Options()
        st = prg_stats()
        co = o.to_c(C.c_void_p(d_start) if d_start else None)
        _check(lib().prg_solve_device(self._h, C.byref(co), C.c_void_p(d_reset) if d_reset else None,
                                      C.c_void_p(d_out), C.byref(st)))
        return Stats.from_c(st)

    def autotune(self, batch: bool = True, cache_path: Optional[str] = None) -> dict:
        """Times row-block shapes, grid occupancy and batched tile widths on
        this graph and keeps the fastest (prg_autotune)."""
        r = prg_tune_result()
        _check(lib().prg_autotune(self._h, int(batch), cache_path.encode() if cache_path else None, C.byref(r)))
        return {k: getattr(r, k) for k, _ in prg_tune_result._fields_ if k != "pad"}

    def solve_noalloc(self, d_out: int, options: Optional[Options] = None, d_reset: int = 0, d_start: int = 0):
        """FP64 solve into a device buffer with no device allocation inside
        the call (prg_solve_noalloc); d_reset: normalised teleport vector,
        d_start: optional device start vector (caller ids)."""
        o = options or Options()
        st = prg_stats()
        co = o.to_c(C.c_void_p(d_start) if d_start else None)
        _check(lib().prg_solve_noalloc(self._h, C.byref(co), C.c_void_p(d_reset) if d_reset else None,
                                       C.c_void_p(d_out), C.byref(st)))
        return Stats.from_c(st)

    def ppr_batch(self, seed_lists, damping: float = 0.85, tol: float = 1e-8, max_iter: int = 1000,
                  vec: int = 0, d_out: int = 0):
        """Batched personalized PageRank (one column per seed list, like
        personalized_pagerank_vs).  Returns (X float32[n, K] or None when
        d_out is given, column_iters uint32[K], stats dict)."""
        K = len(seed_lists)
        off = np.zeros(K + 1, np.uint64)
        off[1:] = np.cumsum([len(x) for x in seed_lists])
        seeds = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint32) for x in seed_lists])
                                     if K else np.zeros(1, np.uint32), dtype=np.uint32)
        iters = np.zeros(max(K, 1), np.uint32)
        st = prg_batch_stats()
        if d_out:
            _check(lib().prg_ppr_batch_device(self._h, K, _ptr(off), _ptr(seeds), damping, tol, max_iter, vec,
                                              C.c_void_p(d_out), _ptr(iters), C.byref(st)))
            X = None
        else:
            X = np.empty((self.n, K), np.float32)
            _check(lib().prg_ppr_batch(self._h, K, _ptr(off), _ptr(seeds), damping, tol, max_iter, vec, _ptr(X),
                                       _ptr(iters), C.byref(st)))
        stats = {"column_iterations": st.column_iterations, "max_iters": st.max_iters, "tiles": st.tiles,
                 "tile_width": st.tile_width, "kernel_launches": st.kernel_launches, "ms": st.ms,
                 "chebyshev": bool(st.chebyshev)}
        return X, iters[:K], stats

    def gather_probe(self, reps: int = 20) -> float:
        """Milliseconds of a gather-only pass over this graph's index stream
        (the floor of the FP32 matvec's memory access pattern)."""
        ms = C.c_double()
        _check(lib().prg_graph_gather_probe(self._h, int(reps), C.byref(ms)))
        return ms.value

    def matvec32(self, kernel: int, d_p: int, d_pt: int, dz: float, damping: float, d_y: int):
        """One FP32 Krylov matvec y = p - d (A pt + dz / n) on internal ids
        through kernel 0 (row-block), 1 or 2 (tile-segmented); device
        pointers of n float32 each.  Returns ((p.y, y.p, y.y), ms)."""
        dots = np.zeros(3)
        ms = C.c_double()
        _check(lib().prg_graph_matvec32(self._h, int(kernel), C.c_void_p(d_p), C.c_void_p(d_pt), float(dz),
                                        float(damping), C.c_void_p(d_y), _ptr(dots), C.byref(ms)))
        return tuple(dots), ms.value

    def device_csr(self):
        """Device pointers (row_ptr, col, perm or 0, inv32) of the resident
        in-CSR, in internal ids."""
        out = [C.c_void_p() for _ in range(4)]
        _check(lib().prg_graph_device_csr(self._h, *[C.byref(o) for o in out]))
        return tuple(o.value or 0 for o in out)

    def close(self):
        if self._h:
            lib().prg_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


GEN_RMAT, GEN_POWERLAW, GEN_BLOCKS = 0, 1, 2


def generate_device(kind: int, n: int, m: int, d_from: int, d_to: int, p0=0.0, p1=0.0, p2=0.0, seed=1,
                    stream: int = 0) -> None:
    """Seeded device edge generators (prg_generate_device)."""
    _check(lib().prg_generate_device(kind, n, m, p0, p1, p2, seed, C.c_void_p(d_from), C.c_void_p(d_to),
                                     C.c_void_p(stream) if stream else None))


def set_tuning(key: str, value: int) -> None:
    """Process-wide tuning for graphs created afterwards (see prg_set_tuning)."""
    _check(lib().prg_set_tuning(key.encode(), int(value)))


def reset_tuning() -> None:
    """Every tuning key back to its default (prg_set_tuning("defaults", 0))."""
    set_tuning("defaults", 0)


def rmat_device(scale: int, m: int, d_from: int, d_to: int, a=0.57, b=0.19, c=0.19, seed=1, stream: int = 0):
    """Counter-based R-MAT edge list written straight into device arrays."""
    _check(lib().prg_rmat_device(scale, m, a, b, c, seed, C.c_void_p(d_from), C.c_void_p(d_to),
                                 C.c_void_p(stream) if stream else None))
