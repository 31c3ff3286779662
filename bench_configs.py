"""Timings of the five workload configurations on one GPU, plus the
edge-list ingest (text -> GPU parse -> resident CSR), eigenvector
centrality / HITS (7) and Infomap's flow model (8).

Inputs are generated on the device with the shapes of each configuration
(R-MAT; a Chung-Lu power law with the degree law of preferential attachment
for the Barabasi-Albert graph; a 64-block model for the SBM); parity at these
shapes is checked by the tests with the reference's own seeded generators.
Each configuration prints one JSON line per solver form: passes, device time
to tolerance, GTEPS (in-CSR arcs x passes / time), algorithmic bytes of one
SpMV pass, the SpMV launches' HBM rate against the measured copy peak, and
the L1 distance to a tight FP64 solve of the same graph.

    python bench_configs.py [--which 1,2,3,4,5,6,7,8] [--peak-gbs 6546]
"""
from __future__ import annotations

import argparse
import json
import math
import os

import sys

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rust-igraph_b200"))

from igraph_b200 import (GEN_BLOCKS, GEN_POWERLAW, GEN_RMAT, PRECISION_FP32_REFINED, PRECISION_FP64, PRECISION_FP64_KRYLOV,
               STOP_ERROR_BOUND, DeviceGraph, Options, generate_device)

D = 0.85


def _peak(arg):
    if arg:
        return arg
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"])
    except Exception:
        return 6650.0


def _bytes(n, arcs, p, w):
    """Algorithmic bytes of one pass: 4(n+1) + (4+w) arcs + 4 p n."""
    return 4 * (n + 1) + (4 + w) * arcs + 4 * p * n


def _device_graph(kind, n, m, p, seed, directed, weighted=False):
    import torch

    df = torch.empty(m, dtype=torch.int32, device="cuda")
    dt = torch.empty(m, dtype=torch.int32, device="cuda")
    generate_device(kind, n, m, df.data_ptr(), dt.data_ptr(), *p, seed=seed)
    dw = None
    if weighted:
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        dw = (0.5 + 1.5 * torch.rand(m, device="cuda", generator=g)).to(torch.float32).to(torch.float64)
    torch.cuda.synchronize()
    dg = DeviceGraph.from_device(n, m, df.data_ptr(), dt.data_ptr(), directed, dw.data_ptr() if dw is not None else 0)
    return dg


def _forms(dg, forms, peak, weighted, tag, reps=3, start=0):
    import torch

    n, arcs = dg.n, dg.arcs
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    tight = torch.empty(n, dtype=torch.float64, device="cuda")
    dg.solve_device(tight.data_ptr(), Options(stop=STOP_ERROR_BOUND, eps=1e-14))
    for name, opt, p in forms:
        dg.solve_device(out.data_ptr(), opt, d_start=start)
        sts = [dg.solve_device(out.data_ptr(), opt, d_start=start) for _ in range(reps)]
        st = min(sts, key=lambda s: s.solve_ms)
        bpp = _bytes(n, arcs, p, (8 if p == 8 else 4) if weighted else 0)
        spmv_us = st.spmv_ms / max(st.spmv_launches, 1) * 1e3
        gbs = bpp / (spmv_us * 1e-6) / 1e9 if st.spmv_launches else None
        print(json.dumps({
            "config": tag, "form": name, "n": n, "arcs": arcs, "passes": st.iterations,
            "fp32_passes": st.fp32_passes, "fp64_passes": st.fp64_passes, "solve_ms": round(st.solve_ms, 3),
            "gteps": arcs * st.iterations / (st.solve_ms * 1e-3) / 1e9, "bytes_per_pass": bpp,
            "spmv_us": round(spmv_us, 1), "spmv_hbm_gbs": gbs, "spmv_frac_of_peak": gbs / peak if gbs else None,
            "error_bound": st.error_bound, "l1_vs_tight": float((out - tight).abs().sum()),
        }), flush=True)


FP64_DROPIN = ("fp64-dropin (reference stop)", Options(), 8)
FP64_BOUND = ("fp64-power (certified)", Options(stop=STOP_ERROR_BOUND), 8)
FP32_REFINED = ("fp32-refined (Krylov)", Options(precision=PRECISION_FP32_REFINED), 4)
FP64_KRYLOV = ("fp64-krylov", Options(precision=PRECISION_FP64_KRYLOV), 8)


def config1(peak):
    # directed G(n=10,000, m=100,000), no self-loops, no duplicates
    rng = np.random.default_rng(1)
    n, m = 10_000, 100_000
    seen = set()
    f, t = [], []
    while len(f) < m:
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if u != v and (u, v) not in seen:
            seen.add((u, v))
            f.append(u)
            t.append(v)
    dg = DeviceGraph.from_host(n, np.array(f, np.uint32), np.array(t, np.uint32), True)
    _forms(dg, [FP64_DROPIN, FP64_BOUND, FP32_REFINED, FP64_KRYLOV], peak, False, "1 ER 10k/100k")
    dg.close()


def config2(peak):
    n, m = 1_000_000, 8_000_000
    dg = _device_graph(GEN_POWERLAW, n, m, (0.5, 8.0, 0.0), 2, False, weighted=True)
    _forms(dg, [FP64_DROPIN, FP64_BOUND, FP32_REFINED, FP64_KRYLOV], peak, True, "2 BA-law 1M/8M weighted")
    dg.close()


def config3(peak):
    scale = 24
    n, m = 1 << scale, 16 << scale
    dg = _device_graph(GEN_RMAT, n, m, (0.57, 0.19, 0.19), 20241203, True)
    dg.autotune(batch=False)
    _forms(dg, [FP64_DROPIN, FP64_BOUND, FP32_REFINED, FP64_KRYLOV], peak, False, "3 R-MAT s24")
    dg.close()


def config4(peak):
    import torch

    n, blocks, K = 2_000_000, 64, 256
    m = n * 20 // 2
    dg = _device_graph(GEN_BLOCKS, n, m, (float(blocks), 0.8, 0.0), 4, False)
    dg.autotune(batch=True)
    rng = np.random.default_rng(4)
    seeds = []
    for _ in range(K):
        c = int(min(1000, max(1, math.floor(math.exp(rng.random() * math.log(1000.0))))))
        seeds.append(rng.choice(n, c, replace=False).astype(np.uint32))
    d_out = torch.empty((n, K), dtype=torch.float32, device="cuda")
    dg.ppr_batch(seeds, tol=1e-8, d_out=d_out.data_ptr())
    best = None
    for _ in range(3):
        _, iters, st = dg.ppr_batch(seeds, tol=1e-8, d_out=d_out.data_ptr())
        if best is None or st["ms"] < best[1]["ms"]:
            best = (iters, st)
    iters, st = best
    col_it = int(iters.sum())
    print(json.dumps({
        "config": "4 SBM 2M K=256", "form": "fp32 batched SpMM, per-column freeze at L1<=1e-8", "n": n,
        "arcs": dg.arcs, "columns": K, "column_iterations": col_it, "max_column_iterations": int(iters.max()),
        "min_column_iterations": int(iters.min()), "ms": st["ms"], "tiles": st["tiles"],
        "tile_width": st["tile_width"],
        "column_gteps": dg.arcs * col_it / (st["ms"] * 1e-3) / 1e9,
        "bytes_per_column_iteration": (4 * (n + 1) + 4 * dg.arcs) / st["tile_width"] + 12 * n,
    }), flush=True)
    dg.close()


def config5(peak):
    from igraph_b200 import warmstart as ws

    net = ws.WarmStartNet.load()
    for scale in (22, 23, 24):
        for refined in (False, True):
            print(json.dumps({"config": "5 warm start", **ws.evaluate(net, ws.heldout_rmat(scale), refined)}),
                  flush=True)
    net.close()


def edgelist_text(u, v):
    """An edge-list text ("u v" lines, ids without padding) from u32 arrays,
    formatted with numpy (decimal digits gathered per line)."""
    u = np.asarray(u, np.uint64)
    v = np.asarray(v, np.uint64)
    m = len(u)

    def digits(x):
        nd = np.ones(m, np.int64)
        t = x.copy()
        for k in range(1, 10):
            nd += (x >= 10 ** k)
        d = np.zeros((m, 10), np.uint8)
        for k in range(10):
            d[:, 9 - k] = (t % 10).astype(np.uint8) + 48
            t //= 10
        return d, nd

    du, nu = digits(u)
    dv, nv = digits(v)
    width = nu + nv + 2
    off = np.zeros(m + 1, np.int64)
    np.cumsum(width, out=off[1:])
    out = np.empty(int(off[-1]), np.uint8)
    for k in range(10):  # digit k of u (from the left of its 10-digit field) goes to off + k - (10 - nu)
        sel = k >= 10 - nu
        out[off[:-1][sel] + k - (10 - nu[sel])] = du[sel, k]
    out[off[:-1] + nu] = 32
    for k in range(10):
        sel = k >= 10 - nv
        out[off[:-1][sel] + nu[sel] + 1 + k - (10 - nv[sel])] = dv[sel, k]
    out[off[1:] - 1] = 10
    return out.tobytes()


def config6(peak):
    # edge-list ingest: text -> GPU parse -> resident CSR (the edges never leave the GPU)
    import time

    import torch

    for scale in (22,):
        n, m = 1 << scale, 16 << scale
        df = torch.empty(m, dtype=torch.int32, device="cuda")
        dt = torch.empty(m, dtype=torch.int32, device="cuda")
        generate_device(GEN_RMAT, n, m, df.data_ptr(), dt.data_ptr(), 0.57, 0.19, 0.19, seed=20241203)
        u = df.cpu().numpy().view(np.uint32)
        v = dt.cpu().numpy().view(np.uint32)
        del df, dt
        text = edgelist_text(u, v)
        from igraph_b200 import parse_edgelist

        res = {}
        for name, fn in (("parse (H2D + parse + D2H of edges)", lambda: parse_edgelist(text)),
                         ("read_edgelist to resident graph (H2D + parse + CSR build)",
                          lambda: DeviceGraph.from_edgelist(text))):
            r = fn()
            if isinstance(r, DeviceGraph):
                r.close()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            dt_s = time.perf_counter() - t0
            if isinstance(r, DeviceGraph):
                r.close()
            else:
                assert len(r[1]) == m and np.array_equal(r[1], u) and np.array_equal(r[2], v)
            res[name] = {"s": round(dt_s, 4), "text_gb_per_s": len(text) / dt_s / 1e9}
        print(json.dumps({"config": f"6 edge-list ingest R-MAT s{scale}", "lines": m, "text_bytes": len(text),
                          **res}), flush=True)


def config7(peak):
    # eigenvector centrality (undirected) and HITS (directed) on R-MAT graphs
    import time

    import torch

    from igraph_b200 import Graph, eigenvector_centrality, hub_and_authority_scores

    for scale in (16, 20, 22):
        n, m = 1 << scale, 16 << scale
        df = torch.empty(m, dtype=torch.int32, device="cuda")
        dt = torch.empty(m, dtype=torch.int32, device="cuda")
        generate_device(GEN_RMAT, n, m, df.data_ptr(), dt.data_ptr(), 0.57, 0.19, 0.19, seed=7)
        f = df.cpu().numpy().view(np.uint32).copy()
        t = dt.cpu().numpy().view(np.uint32).copy()
        del df, dt
        for name, directed, fn in (("eigenvector_centrality (undirected)", False, eigenvector_centrality),
                                   ("hub_and_authority_scores (directed)", True, hub_and_authority_scores)):
            g = Graph.from_edge_arrays(n, f, t, directed)
            fn(g)
            t0 = time.perf_counter()
            fn(g)
            dt_s = time.perf_counter() - t0
            print(json.dumps({"config": f"7 {name} R-MAT s{scale}", "n": n, "m": m,
                              "seconds_incl_upload_and_build": round(dt_s, 4)}), flush=True)


def config8(peak):
    # Infomap's flow model (node flows) on directed R-MAT graphs
    import time

    import torch

    from igraph_b200 import Graph, infomap_flow

    for scale in (16, 20, 22):
        n, m = 1 << scale, 16 << scale
        df = torch.empty(m, dtype=torch.int32, device="cuda")
        dt = torch.empty(m, dtype=torch.int32, device="cuda")
        generate_device(GEN_RMAT, n, m, df.data_ptr(), dt.data_ptr(), 0.57, 0.19, 0.19, seed=8)
        f = df.cpu().numpy().view(np.uint32).copy()
        t = dt.cpu().numpy().view(np.uint32).copy()
        del df, dt
        g = Graph.from_edge_arrays(n, f, t, True)
        infomap_flow(g)
        t0 = time.perf_counter()
        _, it = infomap_flow(g, with_iterations=True)
        dt_s = time.perf_counter() - t0
        print(json.dumps({"config": f"8 infomap_flow (directed) R-MAT s{scale}", "n": n, "m": m, "iterations": it,
                          "seconds_incl_upload_and_build": round(dt_s, 4),
                          "gteps_incl_upload_and_build": round(m * it / dt_s / 1e9, 2)}), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", default="1,2,3,4,5,6")
    ap.add_argument("--peak-gbs", type=float, default=0.0)
    a = ap.parse_args(argv)
    peak = _peak(a.peak_gbs)
    for k in a.which.split(","):
        {"1": config1, "2": config2, "3": config3, "4": config4, "5": config5, "6": config6,
         "7": config7, "8": config8}[k.strip()](peak)


if __name__ == "__main__":
    main()
