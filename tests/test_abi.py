"""The C-ABI library on the CPU: it loads, exports every entry point the
header declares, and validates arguments exactly like rust-igraph before any
device work (these paths never touch CUDA)."""
import ctypes as C
import glob
import math
import os
import re

import numpy as np
import pytest

import igraph_b200 as ig
from conftest import ROOT


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(prg_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_all_symbols():
    L = ig.lib()
    names = declared_functions()
    assert len(names) >= 14
    raw = C.CDLL(ig.library_path())
    for n in names:
        assert hasattr(raw, n), f"missing export {n}"


def test_rust_binding_declares_the_header():
    """The Rust crate's FFI module (rust-igraph_b200/rust/src/ffi.rs, built
    by cargo where a Rust toolchain exists) declares exactly the header's
    entry points, and the status codes agree."""
    src = open(os.path.join(ROOT, "rust-igraph_b200", "rust", "src", "ffi.rs")).read()
    rust = sorted(set(re.findall(r"pub fn (prg_\w+)\s*\(", src)))
    assert rust == declared_functions()
    hdr = open(os.path.join(ROOT, "include", "prg_b200.h")).read()
    for name, val in re.findall(r"pub const (PRG_\w+): i32 = (\d+);", src):
        m = re.search(rf"\b{name}\s*=\s*(\d+)", hdr)
        assert m and int(m.group(1)) == int(val), name


def test_default_options_match_reference_constants():
    o = ig.prg_options()
    ig.lib().prg_default_options(C.byref(o))
    # pagerank.rs:23-25
    assert (o.damping, o.eps, o.max_iter, o.precision, o.stop, o.normalise) == (0.85, 1e-10, 1000, 0, 0, 1)
    assert o.inner == ig.INNER_KRYLOV


def test_linsys_trivial_graphs_need_no_device():
    # pagerank_linsys.rs:102-107 and its tests :382-392
    assert len(ig.pagerank_linsys(ig.Graph.with_vertices(0))) == 0
    assert list(ig.pagerank_linsys(ig.Graph.with_vertices(1))) == [1.0]


def test_unknown_options_are_rejected_before_device_work():
    L = ig.lib()
    for field, value, msg in (("precision", 7, "unknown precision 7"), ("inner", 5, "unknown inner solver 5"),
                              ("stop", 3, "unknown stop rule 3")):
        o = ig.prg_options()
        L.prg_default_options(C.byref(o))
        setattr(o, field, value)
        out = np.empty(1)
        rc = L.prg_solve(C.c_void_p(1), C.byref(o), None, out.ctypes.data_as(C.POINTER(C.c_double)), None)
        assert rc == 1, field
        assert ig.last_error() == msg


def test_trivial_graphs_need_no_device():
    # pagerank.rs:55-60 / pagerank_weighted.rs:55-60
    assert len(ig.pagerank(ig.Graph.with_vertices(0))) == 0
    assert list(ig.pagerank(ig.Graph.with_vertices(1))) == [1.0]
    assert list(ig.pagerank_weighted(ig.Graph.with_vertices(1), [])) == [1.0]
    # n == 1 returns before the weight-length check, as in the reference
    assert list(ig.pagerank_weighted(ig.Graph.with_vertices(1), [1.0, 2.0])) == [1.0]
    assert len(ig.personalized_pagerank(ig.Graph.with_vertices(0), [], 0.85)) == 0
    assert list(ig.personalized_pagerank(ig.Graph.with_vertices(1), [1.0], 0.85)) == [1.0]


def g2():
    g = ig.Graph.with_vertices(2)
    g.add_edge(0, 1)
    return g


def test_weighted_validation_messages():
    # pagerank_weighted.rs:62-76 and its tests :264-285
    with pytest.raises(ig.InvalidArgument, match=r"^weights vector size \(0\) differs from edge count \(1\)$"):
        ig.pagerank_weighted(g2(), [])
    with pytest.raises(ig.InvalidArgument, match=r"^weight at edge 0 must be non-negative and finite \(got -1\)$"):
        ig.pagerank_weighted(g2(), [-1.0])
    with pytest.raises(ig.InvalidArgument, match=r"\(got NaN\)$"):
        ig.pagerank_weighted(g2(), [math.nan])
    with pytest.raises(ig.InvalidArgument, match=r"\(got inf\)$"):
        ig.pagerank_weighted(g2(), [math.inf])
    with pytest.raises(ig.InvalidArgument, match=r"\(got -0.5\)$"):
        ig.pagerank_weighted(g2(), [-0.5])


def test_personalized_validation_order_and_messages():
    g3 = ig.Graph.with_vertices(3)
    with pytest.raises(ig.InvalidArgument, match="reset vector non-empty but graph has no vertices"):
        ig.personalized_pagerank(ig.Graph.with_vertices(0), [1.0], 0.85)
    with pytest.raises(ig.InvalidArgument, match=r"reset length \(2\) does not match vcount \(3\)"):
        ig.personalized_pagerank(g3, [1.0, 1.0], 0.85)
    for d, txt in ((0.0, "0"), (1.0, "1"), (-0.1, "-0.1"), (1.5, "1.5")):
        with pytest.raises(ig.InvalidArgument, match=rf"damping \({re.escape(txt)}\) must be in \(0, 1\)"):
            ig.personalized_pagerank(ig.Graph.with_vertices(2), [0.5, 0.5], d)
    with pytest.raises(ig.InvalidArgument, match="reset vector must sum to a positive value"):
        ig.personalized_pagerank(g3, [0.0, 0.0, 0.0], 0.85)
    with pytest.raises(ig.InvalidArgument, match=r"negative reset value \(-0.5\) at index 1"):
        ig.personalized_pagerank(g3, [1.0, -0.5, 0.5], 0.85)
    # length is checked before damping (personalized_pagerank.rs:78-90)
    with pytest.raises(ig.InvalidArgument, match="reset length"):
        ig.personalized_pagerank(g3, [1.0], 7.0)


def test_personalized_vs_validation():
    g3 = ig.Graph.with_vertices(3)
    with pytest.raises(ig.InvalidArgument, match="^reset_vids must not be empty$"):
        ig.personalized_pagerank_vs(g3, [], 0.85)
    with pytest.raises(ig.InvalidArgument, match=r"^reset vertex 5 out of range \(vcount = 3\)$"):
        ig.personalized_pagerank_vs(g3, [5], 0.85)


def test_graph_mirror_canonicalises_and_checks_range():
    g = ig.Graph.with_vertices(4)
    g.add_edges([(3, 1), (0, 2), (2, 2)])
    assert [g.edge(e) for e in range(3)] == [(1, 3), (0, 2), (2, 2)]
    d = ig.Graph.new(4, True)
    d.add_edge(3, 1)
    assert d.edge(0) == (3, 1) and d.is_directed()
    with pytest.raises(ig.VertexOutOfRange):
        g.add_edge(0, 4)
    with pytest.raises(ig.VertexOutOfRange):
        ig.Graph.from_edge_arrays(3, [0], [3], True)


def test_rust_float_display():
    # messages format f64 like Rust's Display (no exponent, shortest digits)
    with pytest.raises(ig.InvalidArgument, match=r"\(got -0.0000001\)$"):
        ig.pagerank_weighted(g2(), [-1e-7])
    with pytest.raises(ig.InvalidArgument, match=r"\(got -12345678901234567000\)$"):
        ig.pagerank_weighted(g2(), [-1.2345678901234567e19])


def test_infomap_flow_validation_and_trivial_graphs():
    # infomap.rs:175-218 (checked before n == 0), 299-310
    g = g2()
    with pytest.raises(ig.InvalidArgument, match=r"^edge weight vector length 2 does not match edge count 1$"):
        ig.infomap_flow(g, edge_weights=[1.0, 1.0])
    with pytest.raises(ig.InvalidArgument,
                       match=r"^edge weight\[0\] = -1 is invalid \(must be non-negative and finite\)$"):
        ig.infomap_flow(g, edge_weights=[-1.0])
    with pytest.raises(ig.InvalidArgument, match=r"^edge weight\[0\] = NaN is invalid"):
        ig.infomap_flow(g, edge_weights=[math.nan])
    with pytest.raises(ig.InvalidArgument, match=r"^vertex weight vector length 1 does not match vertex count 2$"):
        ig.infomap_flow(g, vertex_weights=[1.0])
    with pytest.raises(ig.InvalidArgument, match=r"^vertex weight\[1\] = inf is invalid$"):
        ig.infomap_flow(g, vertex_weights=[1.0, math.inf])
    with pytest.raises(ig.InvalidArgument, match=r"^all vertex weights are zero$"):
        ig.infomap_flow(g, vertex_weights=[0.0, 0.0])
    with pytest.raises(ig.InvalidArgument, match="edge weight vector length 1 does not match edge count 0"):
        ig.infomap_flow(ig.Graph.with_vertices(0), edge_weights=[1.0])
    assert len(ig.infomap_flow(ig.Graph.with_vertices(0))) == 0
    assert list(ig.infomap_flow(ig.Graph.with_vertices(1))) == [1.0]
    assert list(ig.infomap_flow(ig.Graph.with_vertices(1), vertex_weights=[3.0])) == [1.0]


def test_tuning_keys_are_validated_on_the_host():
    # prg_set_tuning checks its values before any graph uses them
    for key, bad, msg in (("hot_threads", 300, "hot_threads must be 256, 512 or 1024"),
                          ("hot_cache64", 70000, "hot_cache64 must be at most 65536 entries"),
                          ("hot_cache32", 70000, "hot_cache32 must be at most 65536 entries"),
                          ("batch_cheb", 2, "batch_cheb must be 0 or 1"),
                          ("seg_kry32", 3, "seg_kry32 must be 0, 1 or 2"),
                          ("seg_res64", 2, "seg_res64 must be 0 or 1"),
                          ("seg_hot64", 20481, "seg_hot64 must be at most 20480 entries"),
                          ("seg_threads", 640, "seg_threads must be 1024, 768 or 512"),
                          ("seg_pipe", 2, "seg_pipe must be 0 or 1"),
                          ("seg_plain64", 2, "seg_plain64 must be 0 or 1"),
                          ("seg_eig64", 2, "seg_eig64 must be 0 or 1")):
        with pytest.raises(ig.InvalidArgument, match=msg):
            ig.set_tuning(key, bad)
    try:
        for key, good in (("hot_threads", 512), ("hot_cache64", 16384), ("batch_cheb", 0), ("seg_res64", 0),
                          ("seg_hot64", 20480)):
            ig.set_tuning(key, good)
    finally:
        ig.reset_tuning()
