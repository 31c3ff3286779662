"""The gather probe (prg_graph_gather_probe): a gather-only pass over the
graph's index stream, which bench.py reports as the floor of the FP32
matvec's access pattern."""
import numpy as np
import pytest

import igraph_b200 as ig
import oracle as O

pytestmark = pytest.mark.gpu


def test_gather_probe_is_a_floor_for_the_matvec(cuda_ok):
    n = 1 << 18
    f, t = O.rmat(18, 16 * n, seed=90)
    with ig.DeviceGraph.from_host(n, f, t, True) as dg:
        floor = dg.gather_probe(10)
        assert floor > 0.0
        _, st = dg.solve(ig.Options(precision=ig.PRECISION_FP32_REFINED))
        matvec = st.spmv_ms / max(st.spmv_launches, 1)
        # the matvec reads the same stream and does more per arc
        assert floor < 1.5 * matvec, (floor, matvec)
        with pytest.raises(ig.InvalidArgument, match="reps must be"):
            dg.gather_probe(0)
