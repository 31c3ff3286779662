"""CPU (float64) restatement of the warm-start network's forward pass, loss
and gradient, used as the checker of the CUDA kernels in gnn.cu.  It rounds
to BF16 at the same points as the device code (features, weights, hidden
activations, aggregated messages) and, like the device backward pass, uses
the FP32 master weights for gradients and treats those roundings as identity
in the backward direction."""
import numpy as np

F, H, CH, Z = 16, 32, 8, 48
oW1 = 0
oB1 = oW1 + H * F
oWm1 = oB1 + H
oW2 = oWm1 + CH * H
oB2 = oW2 + H * Z
oWm2 = oB2 + H
oW3 = oWm2 + CH * H
oB3 = oW3 + 8 * Z
NPARAM = oB3 + 8


def bf16(x):
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def degrees(n, src, dst, directed):
    """(in-arc count per row, out-degree) with rust-igraph's arc semantics."""
    if directed:
        s, d = src, dst
    else:
        s = np.concatenate([src, dst])
        d = np.concatenate([dst, src])
    indeg = np.bincount(d, minlength=n).astype(np.float64)
    outdeg = np.bincount(s, minlength=n).astype(np.float64)
    return indeg, outdeg, s, d


def features(indeg, outdeg):
    n = len(indeg)
    li = np.log1p(indeg.astype(np.float32)).astype(np.float32)
    lo = np.log1p(outdeg.astype(np.float32)).astype(np.float32)
    f = np.zeros((n, F), np.float32)
    f[:, 0] = li * np.float32(0.125)
    f[:, 1] = lo * np.float32(0.125)
    f[:, 2] = (outdeg == 0).astype(np.float32)
    f[:, 3] = 1.0
    f[:, 4] = (li - lo) * np.float32(0.125)
    f[:, 5] = np.float32(np.log(np.float32(n))) * np.float32(0.0625)
    return bf16(f)


def slog(z):
    return np.sign(z) * np.log1p(np.abs(z))


def loss_and_grad(P, n, src, dst, directed, target, rounding=True):
    """(loss, gradient, normalised prediction).  rounding=False drops every
    BF16 rounding, which makes the forward pass smooth for finite differences."""
    global bf16
    rb = bf16
    if not rounding:
        bf16 = lambda x: np.asarray(x, np.float64)  # noqa: E731
    try:
        return _loss_and_grad(P, n, src, dst, directed, target)
    finally:
        bf16 = rb


def _loss_and_grad(P, n, src, dst, directed, target):
    P = np.asarray(P, np.float64)
    indeg, outdeg, s_arc, d_arc = degrees(n, np.asarray(src, np.int64), np.asarray(dst, np.int64), directed)
    W1 = P[oW1:oB1].reshape(H, F)
    b1 = P[oB1:oWm1]
    Wm1 = P[oWm1:oW2].reshape(CH, H)
    W2 = P[oW2:oB2].reshape(H, Z)
    b2 = P[oB2:oWm2]
    Wm2 = P[oWm2:oW3].reshape(CH, H)
    W3 = P[oW3:oB3].reshape(8, Z)
    b3 = P[oB3]
    sc = np.where(outdeg > 0, 1.0 / np.maximum(outdeg, 1), 0.0).astype(np.float32).astype(np.float64)
    X0 = features(indeg, outdeg)
    H0 = bf16(np.maximum(X0 @ bf16(W1).T + b1, 0.0))
    M0 = (H0 @ bf16(Wm1).T) * sc[:, None]
    S1 = np.zeros((n, CH))
    np.add.at(S1, d_arc, M0[s_arc])
    A1 = bf16(slog(S1))
    Z1 = np.concatenate([H0, A1, np.zeros((n, 8))], axis=1)
    H1 = bf16(np.maximum(Z1 @ bf16(W2).T + b2, 0.0))
    M1 = (H1 @ bf16(Wm2).T) * sc[:, None]
    S2 = np.zeros((n, CH))
    np.add.at(S2, d_arc, M1[s_arc])
    A2 = bf16(slog(S2))
    Z2 = np.concatenate([H1, A2, np.zeros((n, 8))], axis=1)
    y = Z2 @ bf16(W3[0]) + b3
    t = np.maximum(np.asarray(target, np.float64), 1e-300)
    w = n * t
    e = y - np.log(n * t)
    loss = float((w * e * e).sum() / n)
    dy = 2.0 * w * e / n
    g = np.zeros(NPARAM)
    g[oW3:oW3 + Z] = dy @ Z2
    g[oB3] = dy.sum()
    dH1 = dy[:, None] * W3[0, :H][None, :]
    dA2 = dy[:, None] * W3[0, H:H + CH][None, :]
    dS2 = dA2 / (1.0 + np.abs(S2))
    dM1 = np.zeros((n, CH))
    np.add.at(dM1, s_arc, dS2[d_arc])
    G1 = dM1 * sc[:, None]
    g[oWm2:oW3] = (G1.T @ H1).ravel()
    dH1 = dH1 + G1 @ Wm2
    dP1 = dH1 * (H1 > 0)
    g[oW2:oB2] = (dP1.T @ Z1).ravel()
    g[oB2:oWm2] = dP1.sum(0)
    dZ1 = dP1 @ W2
    dH0 = dZ1[:, :H]
    dA1 = dZ1[:, H:H + CH]
    dS1 = dA1 / (1.0 + np.abs(S1))
    dM0 = np.zeros((n, CH))
    np.add.at(dM0, s_arc, dS1[d_arc])
    G0 = dM0 * sc[:, None]
    g[oWm1:oW2] = (G0.T @ H0).ravel()
    dH0 = dH0 + G0 @ Wm1
    dP0 = dH0 * (H0 > 0)
    g[oW1:oB1] = (dP0.T @ X0).ravel()
    g[oB1:oWm1] = dP0.sum(0)
    pred = np.exp(y - y.max())
    return loss, g, pred / pred.sum()
