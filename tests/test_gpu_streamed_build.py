"""The streamed build from host edge arrays (edge lists of >= 2^23 edges:
chunked host -> device copies overlapped with per-chunk sorts, then one scan
and one scatter) against the one-shot build from device arrays: the same
row_ptr, col and vertex numbering, hence bit-identical solves; the weighted
case is also checked against the restatement of pagerank_weighted()."""
import ctypes as C

import numpy as np
import pytest
import torch

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu


class _View:
    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def csr(dg):
    rp, col, perm, inv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    L = ig.lib()
    L.prg_graph_device_csr.restype = C.c_int32
    L.prg_graph_device_csr.argtypes = [C.c_void_p] + [C.POINTER(C.c_void_p)] * 4
    assert L.prg_graph_device_csr(dg._h, C.byref(rp), C.byref(col), C.byref(perm), C.byref(inv)) == 0
    n, arcs = dg.n, dg.arcs
    host = lambda p, k, ts: torch.as_tensor(_View(p.value, k, ts), device="cuda").cpu().numpy().copy()
    out = {"row_ptr": host(rp, n + 1, "<i4"), "col": host(col, arcs, "<i4"), "inv32": host(inv, n, "<f4")}
    out["perm"] = host(perm, n, "<i4") if perm.value else None
    return out


def same_graph(a, b):
    ca, cb = csr(a), csr(b)
    for k in ("row_ptr", "col", "inv32"):
        assert np.array_equal(ca[k], cb[k]), k
    assert (ca["perm"] is None) == (cb["perm"] is None)
    if ca["perm"] is not None:
        assert np.array_equal(ca["perm"], cb["perm"])


def device_arrays(f, t, w=None):
    df = torch.from_numpy(f.view(np.int32)).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    dw = None if w is None else torch.from_numpy(w).cuda()
    return df, dt, dw


def test_rmat_directed_matches_device_build(cuda_ok):
    scale = 22
    n, m = 1 << scale, 16 << scale
    df = torch.empty(m, dtype=torch.int32, device="cuda")
    dt = torch.empty(m, dtype=torch.int32, device="cuda")
    ig.rmat_device(scale, m, df.data_ptr(), dt.data_ptr(), seed=77)
    torch.cuda.synchronize()
    f = df.cpu().numpy().view(np.uint32)
    t = dt.cpu().numpy().view(np.uint32)
    with ig.DeviceGraph.from_device(n, m, df.data_ptr(), dt.data_ptr(), True) as a, \
            ig.DeviceGraph.from_host(n, f, t, True) as b:
        same_graph(a, b)
        key = lambda g: (g.n, g.arcs, g.n_dangling, g.n_rowblocks, g.n_hubs)
        assert key(a) == key(b)
        for opt in (ig.Options(), ig.Options(precision=ig.PRECISION_FP32_REFINED)):
            xa, _ = a.solve(opt)
            xb, _ = b.solve(opt)
            assert np.array_equal(xa, xb)


def test_undirected_weighted_matches_device_build(cuda_ok):
    n = 1_500_000
    f, t = O.barabasi_game_bag(n, 6, True, False, 78)  # ~9e6 edges, loops and multi-edges possible
    assert len(f) >= 1 << 23
    w = O.uniform_weights(len(f), 79)
    df, dt, dw = device_arrays(f, t, w)
    with ig.DeviceGraph.from_device(n, len(f), df.data_ptr(), dt.data_ptr(), False, d_weights=dw.data_ptr()) as a, \
            ig.DeviceGraph.from_host(n, f, t, False, weights=w) as b:
        same_graph(a, b)
        xa, _ = a.solve(ig.Options())
        xb, _ = b.solve(ig.Options())
        assert np.array_equal(xa, xb)
    # the drop-in goes through the streamed build as well
    got = ig.pagerank_weighted(ig.Graph.from_edge_arrays(n, f, t, False), w)
    assert np.max(np.abs(got - xa)) <= 1e-12
    # and both agree with the restatement of pagerank_weighted() (the host
    # sorts of graph.rs:1708-1768 that the streamed build replaces)
    ref = O.pagerank_weighted(n, f, t, False, w)
    assert np.max(np.abs(xb - ref)) <= 1e-10
    assert np.max(np.abs(got - ref)) <= 1e-10


def test_out_of_range_endpoint_is_reported(cuda_ok):
    n, m = 1000, (1 << 23) + 5
    rng = np.random.default_rng(80)
    f = rng.integers(0, n, m).astype(np.uint32)
    t = rng.integers(0, n, m).astype(np.uint32)
    t[m - 3] = 5000
    with pytest.raises(ig.VertexOutOfRange, match=r"vertex id 5000 out of range \(vcount = 1000\)"):
        ig.DeviceGraph.from_host(n, f, t, True)
    f[7] = 4000  # an early chunk too: the largest id is reported
    t[m - 3] = 3000
    with pytest.raises(ig.VertexOutOfRange, match=r"vertex id 4000 out of range"):
        ig.DeviceGraph.from_host(n, f, t, False)
    # the context stays usable
    x = ig.pagerank(ig.Graph.from_edge_arrays(3, [0, 1], [1, 2], True))
    assert abs(x.sum() - 1.0) < 1e-12
