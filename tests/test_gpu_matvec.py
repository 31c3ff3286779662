"""The FP32 Krylov matvec y = p - d (A pt + dz / n) kernel by kernel
(prg_graph_matvec32): the row-block pass (0) and the two tile-segmented
passes (1: 4-arc lane quads, 2: 8 consecutive arcs per lane) against an FP64
restatement on the resident CSR, on graphs that reach every path of the
segmented passes: rows spanning many tiles (short and long span lists), tiles
with more than 32 row ends, rows without arcs, a last partial tile, graphs
smaller than one tile, relabelled ids with the shared-memory hot prefix.
The operator is the one pagerank.rs:107-140 iterates, in the form
pagerank_linsys() solves (pagerank_linsys.rs)."""
import numpy as np
import pytest
import torch

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu

D = 0.85


class _View:
    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def _host(ptr, count, typestr):
    return torch.as_tensor(_View(ptr, count, typestr), device="cuda").cpu().numpy().copy()


def _graph(case):
    directed = True
    if case == "rmat_relabelled":  # larger than the hot prefix: both gather paths
        n = 1 << 17
        f, t = O.rmat(17, 16 * n, seed=44)
    elif case == "star_hub":  # one row of ~15 K arcs: a span of ~60 tiles
        n = 5000
        f = np.arange(1, n, dtype=np.uint32).repeat(3)
        t = np.zeros(len(f), np.uint32)
        f = np.concatenate([f, np.array([0, 0, 7], np.uint32)])
        t = np.concatenate([t, np.array([1, 2, 3], np.uint32)])
    elif case == "cycle":  # every row one arc: 256 row ends per tile
        n = 70_001
        f = np.arange(n, dtype=np.uint32)
        t = ((f + 1) % n).astype(np.uint32)
    elif case == "tiny":
        n = 40
        f, t = O.erdos_renyi_gnm(n, 120, True, False, 3)
    elif case == "sparse_many_empty":
        n = 200_000
        f, t = O.erdos_renyi_gnm(n, 150_000, True, False, 9)
    elif case == "mixed_spans":  # rows of 1 .. 20 000 arcs
        rng = np.random.default_rng(5)
        n = 20_000
        lens = np.minimum(rng.zipf(1.6, n), 20_000).astype(np.int64)
        t = np.repeat(np.arange(n, dtype=np.uint32), lens)
        f = rng.integers(0, n, len(t)).astype(np.uint32)
    else:
        n = 30_000
        f, t = O.barabasi_game_bag(n, 5, False, False, 12)
        directed = False
    return n, np.asarray(f, np.uint32), np.asarray(t, np.uint32), directed


@pytest.mark.parametrize("case", ["rmat_relabelled", "star_hub", "cycle", "tiny", "sparse_many_empty",
                                  "mixed_spans", "undirected_ba"])
def test_matvec_kernels_match_fp64_restatement(cuda_ok, case):
    n, f, t, directed = _graph(case)
    rng = np.random.default_rng(7)
    with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
        rp_d, col_d, perm_d, inv_d = dg.device_csr()
        arcs = dg.arcs
        rp = _host(rp_d, n + 1, "<u4").astype(np.int64)
        col = _host(col_d, arcs, "<u4").astype(np.int64)
        inv = _host(inv_d, n, "<f4")
        # a Krylov direction has both signs
        p = rng.standard_normal(n).astype(np.float32) / np.float32(n)
        pt = (p * inv).astype(np.float32)  # FP32 product, as the solver forms it
        dz = float(p[inv == 0].astype(np.float64).sum())
        # FP64 restatement: y = p - d (sum over in-arcs of pt + dz / n)
        rows = np.repeat(np.arange(n), np.diff(rp))
        acc = np.bincount(rows, weights=pt[col].astype(np.float64), minlength=n)
        mag = np.bincount(rows, weights=np.abs(pt[col]).astype(np.float64), minlength=n)
        ref = p.astype(np.float64) - D * (acc + dz / n)
        # FP32 epilogue and row sum: a few ulps of the operands' magnitude
        tol = 6e-7 * (np.abs(p) + D * mag + D * abs(dz) / n) + 1e-30
        dp = torch.from_numpy(p).cuda()
        dpt = torch.from_numpy(pt).cuda()
        ys = {}
        for kernel in (0, 1, 2):
            dy = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
            dots, _ = dg.matvec32(kernel, dp.data_ptr(), dpt.data_ptr(), dz, D, dy.data_ptr())
            y = dy.cpu().numpy()
            err = np.abs(y.astype(np.float64) - ref)
            assert np.all(err <= tol), (kernel, int(np.argmax(err / tol)), float(np.max(err / tol)))
            y64 = y.astype(np.float64)
            p64 = p.astype(np.float64)
            want = (float(p64 @ y64), float(y64 @ p64), float(y64 @ y64))
            scale = float(np.abs(p64) @ np.abs(y64)) + float(y64 @ y64)
            for got, w in zip(dots, want):
                assert abs(got - w) <= 1e-12 * scale, (kernel, dots, want)
            if kernel:
                # the segmented passes are bit-reproducible
                dy2 = torch.empty_like(dy)
                dots2, _ = dg.matvec32(kernel, dp.data_ptr(), dpt.data_ptr(), dz, D, dy2.data_ptr())
                assert torch.equal(dy, dy2) and dots2 == dots
            ys[kernel] = y
        # both segmented passes sum rows in FP64 and round them once: they
        # differ by at most an ulp or so of the operands' magnitude
        d12 = np.abs(ys[1].astype(np.float64) - ys[2].astype(np.float64))
        assert np.all(d12 <= 2.5e-7 * (np.abs(p) + D * mag + D * abs(dz) / n) + 1e-30)


def test_matvec_rejects_bad_arguments(cuda_ok):
    n = 100
    f, t = O.erdos_renyi_gnm(n, 400, True, False, 1)
    w = O.uniform_weights(len(f), 2)
    dp = torch.zeros(n, dtype=torch.float32, device="cuda")
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        with pytest.raises(ig.IgraphError):
            dg.matvec32(3, dp.data_ptr(), dp.data_ptr(), 0.0, D, dp.data_ptr())
        with pytest.raises(ig.IgraphError):
            dg.matvec32(1, dp.data_ptr(), dp.data_ptr(), 0.0, 1.5, dp.data_ptr())
    with ig.DeviceGraph.from_host(n, f, t, True, weights=w) as dg:
        with pytest.raises(ig.IgraphError):
            dg.matvec32(2, dp.data_ptr(), dp.data_ptr(), 0.0, D, dp.data_ptr())


@pytest.mark.parametrize("case", ["rmat_relabelled", "star_hub", "cycle", "sparse_many_empty"])
def test_segmented_launch_shapes_agree(cuda_ok, case):
    # The tile kernel's block size and its pipelined tile loads change which
    # warp takes a tile, never how a tile is summed: y is bit-identical, the
    # block records agree to rounding.
    n, f, t, directed = _graph(case)
    rng = np.random.default_rng(8)
    p = rng.standard_normal(n).astype(np.float32) / np.float32(n)
    dp = torch.from_numpy(p).cuda()
    out = {}
    try:
        for shape in ((1024, 0), (1024, 1), (768, 0), (768, 1), (512, 1)):
            ig.set_tuning("seg_kry32", 2)
            ig.set_tuning("seg_threads", shape[0])
            ig.set_tuning("seg_pipe", shape[1])
            with ig.DeviceGraph.from_host(n, f, t, directed) as dg:
                inv = _host(dg.device_csr()[3], n, "<f4")
                dpt = torch.from_numpy((p * inv).astype(np.float32)).cuda()
                dz = float(p[inv == 0].astype(np.float64).sum())
                dy = torch.empty(n, dtype=torch.float32, device="cuda")
                dots, _ = dg.matvec32(2, dp.data_ptr(), dpt.data_ptr(), dz, D, dy.data_ptr())
                out[shape] = (dy.cpu().numpy(), dots)
    finally:
        ig.reset_tuning()
    y0, d0 = out[(1024, 0)]
    for shape, (y, dots) in out.items():
        assert np.array_equal(y.view(np.int32), y0.view(np.int32)), shape
        for a, b in zip(dots, d0):
            assert abs(a - b) <= 1e-12 * (abs(b) + float(np.abs(y0.astype(np.float64)) @ np.abs(p))), shape

