"""Benchmark: PageRank time-to-tolerance and GTEPS on one B200 (or N replicas).

Workload (the precision-at-scale configuration): directed R-MAT, scale 24
(16,777,216 vertices), edge factor 16 (268,435,456 edges), a/b/c/d =
0.57/0.19/0.19/0.05, duplicates and self-loops kept, unweighted, damping
0.85.  One step = one full solve to a certified L1 error <= 1e-10 against the
FP64 fixed point with FP32 SpMV + FP64 residual refinement, on a graph
resident in HBM.  value = GTEPS = in-CSR arcs x SpMV passes / time, summed
over ranks, max time over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times rust-igraph's own algorithm on the host cores (the
reference is Rust with no toolchain on this machine, so its line-for-line C
restatement in oracle/ stands in for it; single-threaded like the
reference).  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rust-igraph_b200"))

METRIC = "time-to-L1≤1e-10 & GTEPS: warm-start/FP32-refined vs plain FP64, 1 B200"
D = 0.85
EPS = 1e-10
RMAT = (0.57, 0.19, 0.19)
SEED = 20241203


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--cpu-iters", type=int, default=2)
    p.add_argument("--no-autotune", action="store_true")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(scale, ef):
    return {
        "workload": f"R-MAT scale {scale} edge factor {ef} (a,b,c,d=0.57,0.19,0.19,0.05), directed, duplicates kept, "
                    f"unweighted, d=0.85, solve to certified L1<=1e-10 vs FP64 fixed point",
        "scale": scale,
        "edge_factor": ef,
        "n": 1 << scale,
        "m": ef << scale,
        "damping": D,
        "eps_l1": EPS,
        "seed": SEED,
    }


# ------------------------------------------------------------------ clocks


class ClockSampler:
    """nvidia-smi sampling during the timed region (read-only queries)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev), "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ reference arm


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O

    n, m = 1 << args.scale, args.edge_factor << args.scale
    t0 = time.perf_counter()
    f, t = O.rmat(args.scale, m, *RMAT, seed=SEED)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    adj = O.RefAdjacency(n, f, t, True)
    build_s = time.perf_counter() - t0
    del f, t
    pr = np.full(n, 1.0 / n)
    for _ in range(args.warmup):
        adj.iterate(1, pr)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        adj.iterate(1, pr)
    el = time.perf_counter() - t0
    gteps = adj.arcs * args.steps / el / 1e9
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": gteps,
        "unit": "GTEPS",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload(args.scale, args.edge_factor),
        "cpu_baseline": {
            "value": gteps, "unit": "GTEPS", "cores": 1, "kind": "port",
            "sample": f"each step = one iteration of the pagerank.rs:107-140 loop (C restatement, oracle/prg_oracle.c) "
                      f"over the full graph; in-adjacency build {build_s:.1f} s and generation {gen_s:.1f} s not timed",
        },
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "host": {"nproc": os.cpu_count(), "cpu": _cpu_model()},
    }
    adj.close()
    print(json.dumps(line), flush=True)


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


# ------------------------------------------------------------------ our arm


def load_traffic():
    """Per-launch DRAM traffic of the FP32 iteration kernel from the committed
    ncu summary (profiles/ncu_traffic.txt: `key value` lines)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    try:
        for line in open(path):
            line = line.strip()
            if line and not line.startswith("#"):
                k, v = line.split()[:2]
                out[k] = float(v)
    except Exception:
        pass
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist

    import igraph_b200 as ig

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if ws > 1:
            dist.barrier()

    def allreduce(v, op):
        if ws == 1:
            return v
        t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    scale, ef = args.scale, args.edge_factor
    n, m = 1 << scale, ef << scale
    dev = torch.device("cuda", local)
    df = torch.empty(m, dtype=torch.int32, device=dev)
    dt = torch.empty(m, dtype=torch.int32, device=dev)
    ig.rmat_device(scale, m, df.data_ptr(), dt.data_ptr(), *RMAT, seed=SEED)
    torch.cuda.synchronize()
    dg = ig.DeviceGraph.from_device(n, m, df.data_ptr(), dt.data_ptr(), True)
    arcs = dg.arcs
    tune = None if args.no_autotune else dg.autotune(batch=False)
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    out = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > L2 (126 MB)
    opt_ref = ig.Options(precision=ig.PRECISION_FP32_REFINED, eps=EPS, damping=D)
    opt_64 = ig.Options(precision=ig.PRECISION_FP64, stop=ig.STOP_ERROR_BOUND, eps=EPS, damping=D)

    for _ in range(max(args.warmup, 0)):
        dg.solve_device(out.data_ptr(), opt_ref)
    torch.cuda.synchronize()

    def timed(opts, steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        stats = []
        barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(steps):
                flush.fill_(k & 255)
                stats.append(dg.solve_device(out.data_ptr(), opts))
            e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1), stats

    with ClockSampler(local) as clk:
        ms, stats = timed(opt_ref, args.steps)
    clocks = clk.summary()
    ms_max = allreduce(ms, dist.ReduceOp.MAX if ws > 1 else None)
    passes = sum(s.iterations for s in stats)
    total_units = allreduce(arcs * passes, dist.ReduceOp.SUM if ws > 1 else None)
    value = total_units / (ms_max / 1e3) / 1e9
    x_ref = out.clone()
    launches = sum(s.kernel_launches for s in stats) + args.steps  # + the L2-flush fill per step

    # roofline of the dominant kernel: the FP32 correction iteration
    fp32_ms = sum(s.fp32_ms for s in stats)
    fp32_passes = sum(s.fp32_passes for s in stats)
    bytes_launch = 4 * (n + 1) + 4 * arcs + 4 * 4 * n  # 4(n+1) + (4+w)m + 4*p*n, p=4, w=0
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    avg_launch_s = fp32_ms / max(fp32_passes, 1) / 1e3
    achieved = bytes_launch / avg_launch_s / 1e9
    tr = load_traffic()
    traffic = None
    if "corr32_bytes_per_arc" in tr:
        traffic = tr["corr32_bytes_per_arc"] * arcs + tr.get("corr32_bytes_per_vertex", 0.0) * n
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_src, "kernel": "iter_kernel<MODE_CORR32> (FP32 correction)",
                "bytes_per_launch": bytes_launch, "avg_launch_us": avg_launch_s * 1e6}

    # plain FP64 comparison (same stop rule: certified L1 <= 1e-10)
    plain = None
    if not args.no_plain:
        ms64, st64 = timed(opt_64, max(1, min(args.steps, 2)))
        x64 = out.clone()
        p64 = sum(s.iterations for s in st64)
        t64 = ms64 / len(st64)
        plain = {"ms_per_solve": t64, "passes": p64 / len(st64), "gteps": arcs * p64 / (ms64 / 1e3) / 1e9,
                 "fp64_iter_us": sum(s.fp64_ms for s in st64) / max(p64, 1) * 1e3,
                 "error_bound": st64[-1].error_bound,
                 "l1_refined_vs_fp64": float((x_ref - x64).abs().sum().item())}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        hf = torch.empty(m, dtype=torch.int32, pin_memory=True)
        ht = torch.empty(m, dtype=torch.int32, pin_memory=True)
        hf.copy_(df)
        ht.copy_(dt)
        hout = torch.empty(n, dtype=torch.float64, pin_memory=True)
        fnp, tnp, onp = hf.numpy().view(np.uint32), ht.numpy().view(np.uint32), hout.numpy()

        def e2e_step():
            g2 = ig.DeviceGraph.from_host(n, fnp, tnp, True)
            _, st = g2.solve(opt_ref, out=onp)
            g2.close()
            return st

        e2e_step()  # warm the allocator pool
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_stats = [e2e_step() for _ in range(args.steps)]
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        el = allreduce(el, dist.ReduceOp.MAX if ws > 1 else None)
        units = allreduce(arcs * sum(s.iterations for s in e2e_stats), dist.ReduceOp.SUM if ws > 1 else None)
        e2e = {"value": units / el / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": 2 * 4 * m,
               "d2h_bytes_per_step": 8 * n, "ms_per_step": el / args.steps * 1e3,
               "includes": "H2D of the edge list from pinned memory, CSR build, refined solve, D2H of the result",
               "build_ms": e2e_stats[-1].build_ms}
        del hf, ht, hout

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        f_np = df.cpu().numpy().view(np.uint32)
        t_np = dt.cpu().numpy().view(np.uint32)
        t0 = time.perf_counter()
        adj = O.RefAdjacency(n, f_np, t_np, True)
        b_s = time.perf_counter() - t0
        del f_np, t_np
        pr = np.full(n, 1.0 / n)
        t0 = time.perf_counter()
        adj.iterate(args.cpu_iters, pr)
        it_s = time.perf_counter() - t0
        cpu = {"value": adj.arcs * args.cpu_iters / it_s / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_iters} iterations of the pagerank.rs:107-140 loop (C restatement) over the "
                         f"full graph, {it_s:.1f} s; in-adjacency build {b_s:.1f} s not counted",
               "host_nproc": os.cpu_count(), "host_cpu": _cpu_model()}
        adj.close()

    s0 = stats[-1]
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GTEPS",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic",
        "config": {**workload(scale, ef), "arcs": arcs, "n_dangling": dg.n_dangling,
                   "precision": "FP32 SpMV + FP64 residual refinement",
                   "l2": "inputs larger than L2 (CSR 1.07 GB) and a 256 MiB write between steps",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "time_to_tol_ms": ms_max / args.steps,
        "solve_ms_each": [round(s.solve_ms, 2) for s in stats],
        "kernel_ms_each": [round(s.fp32_ms + s.fp64_ms, 2) for s in stats],
        "passes_per_solve": passes / args.steps,
        "fp32_passes_per_solve": fp32_passes / args.steps,
        "residual_passes_per_solve": s0.residual_passes,
        "error_bound": s0.error_bound,
        "build_ms": dg.build_ms,
        "autotune": tune,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "plain_fp64": plain,
        "speedup_vs_plain_fp64": (plain["ms_per_solve"] / (ms_max / args.steps)) if plain else None,
    }
    dg.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
