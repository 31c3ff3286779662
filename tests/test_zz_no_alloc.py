"""The allocation-free entry point, prg_solve_noalloc, against prg_solve_device.

Some callers cannot let a library allocate device memory while they solve:
a real-time loop that reserves all its memory up front, or code that runs
under another framework's memory budget.  prg_solve_noalloc serves them by
keeping every piece of solve scratch in one static device array.  This file
checks that it returns what the allocating entry point returns (max-abs
<= 1e-10, the FP64 parity tolerance of the other tests) on two calls in a row,
that it matches the oracle, and that it rejects graphs beyond its limits.
It is collected last so that a stop at the first failure has already run
every other test.
"""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu
PARITY = 1e-10


def _maxabs(a, b):
    return float((a - b).abs().max().item())


@pytest.mark.parametrize("kind", ["erdos_renyi", "rmat_relabelled"])
def test_noalloc_matches_allocating_solve(cuda_ok, kind):
    import torch

    if kind == "erdos_renyi":
        n = 10_000
        f, t = O.erdos_renyi_gnm(n, 100_000, True, False, 31)
    else:
        n = 1 << 15
        f, t = O.rmat(15, 16 * n, seed=8)
    ref_cpu = O.pagerank(n, f, t, True)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        if kind == "rmat_relabelled":
            assert dg.relabelled and dg.n_hubs >= 1
        ref = torch.empty(n, dtype=torch.float64, device="cuda")
        st_ref = dg.solve_device(ref.data_ptr(), ig.Options())
        r = torch.zeros(n, dtype=torch.float64, device="cuda")
        r[[1, 2, 500]] = torch.tensor([0.5, 0.25, 0.25], dtype=torch.float64, device="cuda")
        ref_p = torch.empty(n, dtype=torch.float64, device="cuda")
        dg.solve_device(ref_p.data_ptr(), ig.Options(), d_reset=r.data_ptr())
        for _ in range(2):  # two calls in a row share (and must clear) the static scratch
            out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
            st = dg.solve_noalloc(out.data_ptr(), ig.Options())
            assert _maxabs(out, ref) <= PARITY
            assert st.iterations == st_ref.iterations
            assert float(np.abs(out.cpu().numpy() - ref_cpu).max()) <= PARITY
            out_p = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
            dg.solve_noalloc(out_p.data_ptr(), ig.Options(), d_reset=r.data_ptr())
            assert _maxabs(out_p, ref_p) <= PARITY


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
