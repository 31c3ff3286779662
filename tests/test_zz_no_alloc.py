"""The allocation-free entry point, prg_solve_noalloc, against prg_solve_device.

Some callers cannot let a library allocate device memory while they solve:
a real-time loop that reserves all its memory up front, or code that runs
under another framework's memory budget.  prg_solve_noalloc serves them by
keeping every piece of solve scratch in one static device array, which CUDA
allocates (with the kernels the solve launches) when a graph handle within
the entry point's limits is created.  This file checks that the call
returns what the allocating entry point returns (max-abs <= 1e-10, the FP64
parity tolerance of the other tests) on two calls in a row, that it matches
the oracle, that the device's free memory does not move across a call (the
first one on a fresh graph included), and that it rejects what it cannot
serve.  It is collected last so that a stop at the first failure has
already run every other test.
"""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu
PARITY = 1e-10


def _maxabs(a, b):
    return float((a - b).abs().max().item())


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _graph(kind):
    """(n, from, to, weights or None, oracle result)."""
    if kind == "erdos_renyi":
        n = 10_000
        f, t = O.erdos_renyi_gnm(n, 100_000, True, False, 31)
        return n, f, t, None, O.pagerank(n, f, t, True)
    if kind == "rmat_relabelled":
        n = 1 << 15
        f, t = O.rmat(15, 16 * n, seed=8)
        return n, f, t, None, O.pagerank(n, f, t, True)
    # directed and weighted, with zero-weight arcs and vertices whose
    # out-strength is zero (sinks, and sources of zero-weight arcs only)
    n = 20_000
    f, t = O.erdos_renyi_gnm(n, 120_000, True, False, 77)
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 2.0, len(f))
    w[rng.random(len(f)) < 0.1] = 0.0
    w[f < 300] = 0.0  # vertices 0..299 keep their arcs but have out-strength 0
    keep = t != 12345  # vertex 12345 loses its in-arcs only
    keep &= f != 777  # vertex 777 has no out-arcs at all
    f, t, w = f[keep], t[keep], w[keep]
    return n, f, t, w, O.pagerank_weighted(n, f, t, True, w)


@pytest.mark.parametrize("kind", ["erdos_renyi", "rmat_relabelled", "weighted_zero_strength"])
def test_noalloc_matches_allocating_solve(cuda_ok, kind):
    import torch

    n, f, t, w, ref_cpu = _graph(kind)
    r = torch.zeros(n, dtype=torch.float64, device="cuda")
    r[[1, 2, 500]] = torch.tensor([0.5, 0.25, 0.25], dtype=torch.float64, device="cuda")
    outs = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(4)]
    with ig.DeviceGraph.from_host(n, f, t, True, weights=w) as dg:
        if kind == "rmat_relabelled":
            assert dg.relabelled and dg.n_hubs >= 1
        # the first call on this graph, before any allocating solve: the
        # handle's creation loaded the scratch array and the kernels
        free0 = _free_bytes()
        st0 = dg.solve_noalloc(outs[0].data_ptr(), ig.Options())
        assert _free_bytes() == free0, "the allocation-free solve changed the device's free memory"
        ref = torch.empty(n, dtype=torch.float64, device="cuda")
        st_ref = dg.solve_device(ref.data_ptr(), ig.Options())
        ref_p = torch.empty(n, dtype=torch.float64, device="cuda")
        dg.solve_device(ref_p.data_ptr(), ig.Options(), d_reset=r.data_ptr())
        assert _maxabs(outs[0], ref) <= PARITY and st0.iterations == st_ref.iterations
        for k in range(2):  # two calls in a row share (and must clear) the static scratch
            out, out_p = outs[2 * k], outs[2 * k + 1]
            out.fill_(float("nan"))
            out_p.fill_(float("nan"))
            free0 = _free_bytes()
            st = dg.solve_noalloc(out.data_ptr(), ig.Options())
            dg.solve_noalloc(out_p.data_ptr(), ig.Options(), d_reset=r.data_ptr())
            assert _free_bytes() == free0
            assert _maxabs(out, ref) <= PARITY
            assert st.iterations == st_ref.iterations
            assert float(np.abs(out.cpu().numpy() - ref_cpu).max()) <= PARITY
            assert _maxabs(out_p, ref_p) <= PARITY


def test_noalloc_start_vector_and_option_checks(cuda_ok):
    import torch

    n = 10_000
    f, t = O.erdos_renyi_gnm(n, 100_000, True, False, 3)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        start = torch.rand(n, dtype=torch.float64, device="cuda")
        start /= start.sum()
        ref = torch.empty(n, dtype=torch.float64, device="cuda")
        st_ref = dg.solve_device(ref.data_ptr(), ig.Options(), d_start=start.data_ptr())
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        st = dg.solve_noalloc(out.data_ptr(), ig.Options(), d_start=start.data_ptr())
        assert _maxabs(out, ref) <= PARITY and st.iterations == st_ref.iterations
        with pytest.raises(ig.InvalidArgument, match="unknown stop rule"):
            dg.solve_noalloc(out.data_ptr(), ig.Options(stop=7))
        with pytest.raises(ig.InvalidArgument, match="eps must be positive"):
            dg.solve_noalloc(out.data_ptr(), ig.Options(eps=float("nan")))


def test_noalloc_rejects_inputs_beyond_its_limits(cuda_ok):
    import torch

    n = 600_000  # above the 524,288-vertex limit of the static scratch
    f = np.arange(1, n, dtype=np.uint32)
    t = np.zeros(n - 1, np.uint32)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        with pytest.raises(ig.InvalidArgument, match="supports at most 524288"):
            dg.solve_noalloc(out.data_ptr(), ig.Options())
        with pytest.raises(ig.InvalidArgument, match="FP64 path only"):
            dg.solve_noalloc(out.data_ptr(), ig.Options(precision=ig.PRECISION_FP32_REFINED))
