"""The float64 warm-start oracle's gradient against central finite
differences (CPU only; rounding off so the loss is smooth)."""
import numpy as np

import gnn_oracle as GO
import oracle as O


def test_oracle_gradient_finite_differences():
    n = 400
    f, t = O.barabasi_game_bag(n, 3, False, True, 11)
    x = O.pagerank(n, f, t, True)
    rng = np.random.default_rng(4)
    P = rng.normal(0, 0.2, GO.NPARAM)
    P[GO.oW3 + GO.Z:GO.oB3] = 0.0  # rows 1..7 of W3 are unused
    _, g, _ = GO.loss_and_grad(P, n, f, t, True, x, rounding=False)
    live = [i for i in range(GO.NPARAM) if not (GO.oW3 + GO.Z <= i < GO.oB3 or GO.oB3 < i)]
    for i in rng.choice(live, 40, replace=False):
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp, _, _ = GO.loss_and_grad(Pp, n, f, t, True, x, rounding=False)
        lm, _, _ = GO.loss_and_grad(Pm, n, f, t, True, x, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])
