"""Learned warm start: training, persistence and use of the message-passing
network behind prg_gnn_* (include/prg_b200.h).

The network predicts the PageRank vector of a graph from degree features;
its normalised output is handed to the solver as a start vector, so the
fixed point and stop rule are untouched.  Training data are PageRank vectors
that the plain FP64 method computes on seeded synthetic graphs of three
families generated on the GPU: R-MAT, Chung-Lu power law (the degree law of
preferential attachment) and block models.

    python -m igraph_b200.warmstart train --graphs 200 --epochs 8 --out weights.f32
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import (GEN_BLOCKS, GEN_POWERLAW, GEN_RMAT, STOP_ERROR_BOUND, DeviceGraph, Options, _check, _ptr,
               generate_device, lib)

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights.f32")
MAGIC = b"PRGWS001"


class WarmStartNet:
    """Owns a prg_gnn handle."""

    def __init__(self, seed: int = 1):
        h = C.c_void_p()
        _check(lib().prg_gnn_create(seed, C.byref(h)))
        self._h = h
        self.count = lib().prg_gnn_param_count()

    @property
    def handle(self):
        return self._h

    def params(self) -> np.ndarray:
        p = np.empty(self.count, np.float32)
        _check(lib().prg_gnn_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.count,)
        _check(lib().prg_gnn_set_params(self._h, _ptr(p)))

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(MAGIC)
            f.write(np.uint32(self.count).tobytes())
            f.write(self.params().tobytes())

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS) -> "WarmStartNet":
        with open(path, "rb") as f:
            if f.read(8) != MAGIC:
                raise ValueError(f"{path}: not a warm-start weight file")
            cnt = int(np.frombuffer(f.read(4), np.uint32)[0])
            p = np.frombuffer(f.read(4 * cnt), np.float32)
        net = cls()
        if cnt != net.count:
            raise ValueError(f"{path}: {cnt} parameters, expected {net.count}")
        net.set_params(p)
        return net

    def predict(self, dg: DeviceGraph, d_start: int) -> float:
        """Start vector (caller ids, sums to 1) into a device double[n]; returns inference ms."""
        ms = C.c_double()
        _check(lib().prg_gnn_predict(self._h, dg.handle, C.c_void_p(d_start), C.byref(ms)))
        return ms.value

    def loss_grad(self, dg: DeviceGraph, d_target: int):
        loss = C.c_double()
        g = np.empty(self.count, np.float32)
        _check(lib().prg_gnn_loss_grad(self._h, dg.handle, C.c_void_p(d_target), C.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step(self, dg: DeviceGraph, d_target: int, lr: float) -> float:
        loss = C.c_double()
        _check(lib().prg_gnn_train_step(self._h, dg.handle, C.c_void_p(d_target), lr, C.byref(loss)))
        return loss.value

    def close(self):
        if self._h:
            lib().prg_gnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class GraphSpec:
    family: str
    n: int
    m: int
    p: tuple
    seed: int
    directed: bool


def training_specs(count: int = 200, seed: int = 2024, n_min: int = 100_000, n_max: int = 1_000_000):
    """Seeded mix of R-MAT, power-law and block-model graphs, 100k-1M vertices."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        fam = ("rmat", "powerlaw", "blocks")[i % 3]
        ef = int(rng.choice([8, 12, 16]))
        if fam == "rmat":
            scale = int(rng.integers(int(math.log2(n_min)) + 1, int(math.log2(n_max)) + 1))
            n = 1 << scale
            a = float(rng.uniform(0.45, 0.62))
            b = c = float((1 - a) * rng.uniform(0.3, 0.45))
            specs.append(GraphSpec(fam, n, ef * n, (a, b, c), int(rng.integers(1, 2**62)), True))
        elif fam == "powerlaw":
            n = int(rng.integers(n_min, n_max))
            alpha = float(rng.uniform(0.45, 0.75))
            specs.append(GraphSpec(fam, n, ef * n // 2, (alpha, float(rng.uniform(1, 20)), 0.0),
                                   int(rng.integers(1, 2**62)), bool(rng.integers(0, 2))))
        else:
            blocks = int(rng.choice([16, 32, 64]))
            n = int(rng.integers(n_min, n_max)) // blocks * blocks
            specs.append(GraphSpec(fam, n, ef * n // 2, (float(blocks), float(rng.uniform(0.6, 0.95)), 0.0),
                                   int(rng.integers(1, 2**62)), False))
    return specs


def heldout_rmat(scale: int, seed: int = 777):
    n = 1 << scale
    return GraphSpec("rmat", n, 16 * n, (0.57, 0.19, 0.19), seed, True)


def build(spec: GraphSpec):
    """(DeviceGraph, edge buffers) for a spec, generated on the GPU."""
    import torch

    kind = {"rmat": GEN_RMAT, "powerlaw": GEN_POWERLAW, "blocks": GEN_BLOCKS}[spec.family]
    df = torch.empty(spec.m, dtype=torch.int32, device="cuda")
    dt = torch.empty(spec.m, dtype=torch.int32, device="cuda")
    generate_device(kind, spec.n, spec.m, df.data_ptr(), dt.data_ptr(), *spec.p, seed=spec.seed)
    torch.cuda.synchronize()
    dg = DeviceGraph.from_device(spec.n, spec.m, df.data_ptr(), dt.data_ptr(), spec.directed)
    return dg


def label(dg: DeviceGraph):
    """PageRank of the plain FP64 method (certified L1 <= 1e-10), device tensor."""
    import torch

    x = torch.empty(dg.n, dtype=torch.float64, device="cuda")
    st = dg.solve_device(x.data_ptr(), Options(stop=STOP_ERROR_BOUND))
    return x, st


def train(net: WarmStartNet, specs, epochs: int = 8, lr: float = 3e-3, log=print, lr_decay: float = 0.7):
    """Adam over the graphs (one full-graph step each), `epochs` passes."""
    data = []
    t0 = time.time()
    for sp in specs:
        dg = build(sp)
        x, st = label(dg)
        data.append((dg, x))
    log(json.dumps({"event": "dataset", "graphs": len(data), "seconds": round(time.time() - t0, 1)}))
    rng = np.random.default_rng(5)
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(data))
        tot = 0.0
        for i in order:
            dg, x = data[i]
            tot += net.train_step(dg, x.data_ptr(), lr)
        hist.append(tot / len(data))
        log(json.dumps({"event": "epoch", "epoch": ep, "loss": hist[-1], "lr": lr}))
        lr *= lr_decay if ep >= epochs // 2 else 1.0
    for dg, _ in data:
        dg.close()
    return hist


def evaluate(net: WarmStartNet, spec: GraphSpec, refined: bool = False):
    """Iterations and device time to a certified L1 <= 1e-10 from the uniform
    start and from the network's start (inference included)."""
    import torch

    from . import PRECISION_FP32_REFINED, PRECISION_FP64

    dg = build(spec)
    x_ref, _ = label(dg)
    out = torch.empty(dg.n, dtype=torch.float64, device="cuda")
    start = torch.empty(dg.n, dtype=torch.float64, device="cuda")
    prec = PRECISION_FP32_REFINED if refined else PRECISION_FP64
    opts = Options(precision=prec, stop=STOP_ERROR_BOUND)
    dg.solve_device(out.data_ptr(), opts)  # warm caches and captured graphs
    st_u = dg.solve_device(out.data_ptr(), opts)
    uni = torch.full((dg.n,), 1.0 / dg.n, dtype=torch.float64, device="cuda")
    inf_ms = net.predict(dg, start.data_ptr())
    inf_ms = net.predict(dg, start.data_ptr())
    st_w = dg.solve_device(out.data_ptr(), opts, d_start=start.data_ptr())
    res = {
        "graph": f"{spec.family} n={spec.n} m={spec.m}",
        "precision": "fp32-refined" if refined else "fp64",
        "uniform": {"passes": st_u.iterations, "solve_ms": st_u.solve_ms},
        "warm": {"passes": st_w.iterations, "solve_ms": st_w.solve_ms, "inference_ms": inf_ms,
                 "total_ms": st_w.solve_ms + inf_ms},
        "start_l1_error": {"uniform": float((uni - x_ref).abs().sum()), "warm": float((start - x_ref).abs().sum())},
        "result_l1_vs_fp64": float((out - x_ref).abs().sum()),
    }
    dg.close()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--graphs", type=int, default=200)
    t.add_argument("--epochs", type=int, default=8)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--n-min", type=int, default=100_000)
    t.add_argument("--n-max", type=int, default=1_000_000)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--eval-scale", type=int, nargs="*", default=[22])
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--scale", type=int, nargs="*", default=[22, 23, 24])
    a = ap.parse_args(argv)
    if a.cmd == "train":
        net = WarmStartNet(a.seed)
        specs = training_specs(a.graphs, n_min=a.n_min, n_max=a.n_max)
        train(net, specs, a.epochs, a.lr)
        net.save(a.out)
        for sc in a.eval_scale:
            print(json.dumps(evaluate(net, heldout_rmat(sc))))
    else:
        net = WarmStartNet.load(a.weights)
        for sc in a.scale:
            for refined in (False, True):
                print(json.dumps(evaluate(net, heldout_rmat(sc), refined)))


if __name__ == "__main__":
    main()
