"""Benchmark of the B200 edge-elimination screen (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Workload (default "batch"): the 4,096-instance batching mix (n log-uniform in [100, 5000],
uniform / clustered 50/50, 10-NN, EUC_2D; seeded synthetic stand-ins for the reference's TSPLIB
inputs), screened as one snapshot. A step is one JV screen of every active edge of the batch in
one launch. metric = JV edges screened per second over the whole job.

  value      resident inputs (uploaded once), K launches timed with CUDA events on the
             launching stream; inputs (~1.1 GB) exceed L2, so no flush is needed
  e2e        the same step through the C ABI with pinned host buffers: cee_jv_screen per step
             (static-key compare, H2D of active bits + CSR, launch, D2H of the witnesses)
  roofline   jv_screen_kernel: algorithmic bytes per launch (12 n + 33 m) / launch time
  kopt       the 200,000-row k-opt leaf cost matrix (k = 3/4/5 in thirds, 15,000-node CEIL_2D
             instance): cells/s resident and end to end, with its own roofline
  cpu_baseline  the reference's own CPU FindJvCandidatesCpu (oracle/_ref, compiled from the
             reference sources) on a bounded sample of the same instances, threads over instances

--impl reference times the reference's CPU implementation of the same step on the host cores.
Multi-GPU: one process per GPU, independent replicas (the screen shards by instance with no
exchange), timing = max over ranks, value = all ranks' edges / that time.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import json
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "JV edges screened/s"
UNIT = "edges/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="batch", choices=["batch"])
    p.add_argument("--instances", type=int, default=4096)
    p.add_argument("--no-kopt", action="store_true")
    p.add_argument("--part", default="all", choices=["all", "jv", "kopt"],
                   help="profiling aid: run only the JV or only the k-opt part")
    p.add_argument("--cpu-budget-s", type=float, default=12.0)
    return p.parse_args()


def load_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    path = ROOT / "profiles" / "ncu_traffic.json"
    if path.exists():
        return json.loads(path.read_text())
    return {}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        mhz, max_mhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                max_mhz = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "0x1", "1"):
                    reasons.add(name)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": max_mhz, "reasons": sorted(reasons),
                "samples": len(mhz)}


# ---------------------------------------------------------------- CPU reference -----------

def reference_jv_rate(batch, budget_s: float, threads: int):
    """The reference's FindJvCandidatesCpu over instances in order until the time budget is
    spent; instances run concurrently on `threads` host threads. Returns (edges/s, sample)."""
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    if kind == "reference":
        ref = oracle.Reference()
        screen = lambda g: ref.graph(g).jv_cpu()  # noqa: E731
    else:
        port = oracle.Port()
        screen = port.jv_screen
    edges = 0
    done = 0
    lock = threading.Lock()
    stop = time.perf_counter() + budget_s
    start = time.perf_counter()

    def work(i):
        nonlocal edges, done
        if time.perf_counter() > stop:
            return
        g = batch.instance(i)
        screen(g)
        with lock:
            edges += int(g.active.sum())
            done += 1

    with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as pool:
        list(pool.map(work, range(batch.count)))
    elapsed = time.perf_counter() - start
    sample = f"{done} of {batch.count} instances ({edges} edges), {threads} threads, {elapsed:.1f} s"
    return edges / elapsed, kind, sample


# ---------------------------------------------------------------- our arm -----------------

def pinned_copy(arr: np.ndarray):
    """A page-locked copy of `arr` (any dtype) and a numpy view of it."""
    import torch
    arr = np.ascontiguousarray(arr)
    t = torch.from_numpy(arr.view(np.uint8).reshape(-1)).pin_memory()
    return t, t.numpy().view(arr.dtype).reshape(arr.shape)


def run_ours(args, rank: int, world: int, device: int):
    import torch
    from cudaedgeelimination_b200 import Context, GraphSnapshot, synth

    torch.cuda.set_device(device)
    if args.part == "kopt":
        ctx = Context(device)
        out = run_kopt(args, ctx, torch.cuda.ExternalStream(ctx.stream, device=device), device, world)
        ctx.close()
        return out
    batch = synth.BatchUnion(args.instances)
    g = batch.graph
    ctx = Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    n, m, adj = g.n, g.m, int(g.row_offsets[-1])

    # ---- resident timing of the screen kernel ----
    ctx.jv_prepare(g)
    for _ in range(args.warmup):
        ctx.jv_launch()
    ctx.synchronize()
    witness = ctx.jv_fetch(m)
    if rank == 0:
        import oracle
        port = oracle.Port()
        for i in range(0, batch.count, max(1, batch.count // 8)):  # spot parity check, cheap
            e0, e1 = int(batch.edge_begin[i]), int(batch.edge_begin[i + 1])
            inst = batch.instance(i)
            assert (witness[e0:e1] == np.where(port.jv_screen(inst) >= 0,
                                                port.jv_screen(inst) + int(batch.node_begin[i]), -1)).all()
    barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        torch.cuda.synchronize(device)
        barrier(world)
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.jv_launch()
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize(device)
        barrier(world)
    ms_total = ev0.elapsed_time(ev1)
    ms_total = max_over_ranks(ms_total, world)
    ms_step = ms_total / args.steps
    edges_step = int(g.active.sum())
    value = edges_step * world / (ms_step / 1e3)

    # ---- end to end through the C ABI with pinned host buffers ----
    keep = []
    arrays = {}
    for name in ("x", "y", "edge_u", "edge_v", "edge_w", "active", "row_offsets", "neighbors", "csr_edge_ids"):
        t, a = pinned_copy(getattr(g, name))
        keep.append(t)
        arrays[name] = a
    hg = GraphSnapshot.__new__(GraphSnapshot)
    hg.n, hg.dist_type = g.n, g.dist_type
    for name, a in arrays.items():
        setattr(hg, name, a)
    wt, wout = pinned_copy(np.empty(m, np.int32))
    keep.append(wt)
    import ctypes
    from cudaedgeelimination_b200 import _native
    view = hg.view()
    stats = _native.JvStats()
    L = _native.lib()

    def e2e_step():
        _native.check(ctx.handle, L.cee_jv_screen(ctx.handle, ctypes.byref(view),
                                                   wout.ctypes.data_as(_native.c_i32p), ctypes.byref(stats)))

    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    assert (wout == witness).all()
    e2e_value = edges_step * world / (e2e_s / args.steps)
    h2d_bytes = int(stats.h2d_bytes)
    d2h_bytes = int(stats.d2h_bytes)

    # ---- roofline of the dominant kernel ----
    peak, peak_kind = load_peaks()
    alg_bytes = 12 * n + 33 * m
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    traffic = load_traffic().get("jv_screen_kernel")

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded; TSPLIB/ElimTSP inputs not shipped)",
        "config": {"workload": f"batching mix: {batch.count} instances, n log-uniform [100,5000], "
                               "uniform/clustered 50/50, 10-NN, EUC_2D; JV screen of every active edge "
                               "in one launch", "instances": batch.count, "nodes": n, "edges": m,
                   "l2": "inputs (~1.1 GB) larger than L2, no flush", "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "ms_per_step": e2e_s / args.steps * 1e3, "api": "cee_jv_screen (pinned host buffers)"},
        "roofline": {"kernel": "jv_screen_kernel", "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                     "note": "JV is ALU/latency bound; see distance_evals_per_s"},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps,
    }

    # algorithmic distance evaluations (sequential CPU count) on a sample, scaled per edge
    if rank == 0:
        import oracle
        port = oracle.Port()
        ev_total = ev_edges = 0
        for i in range(0, batch.count, max(1, batch.count // 64)):
            inst = batch.instance(i)
            _, ev = port.jv_screen(inst, with_evals=True)
            ev_total += int(ev.sum())
            ev_edges += inst.m
        per_edge = ev_total / max(1, ev_edges)
        result["roofline"]["distance_evals_per_edge"] = per_edge
        result["roofline"]["distance_evals_per_s"] = per_edge * edges_step / (ms_step / 1e3)

    if not args.no_kopt and args.part == "all":
        result["kopt"] = run_kopt(args, ctx, stream, device, world)

    if rank == 0:
        rate, kind, sample = reference_jv_rate(batch, args.cpu_budget_s, os.cpu_count() or 1)
        result["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": kind,
                                  "sample": sample}
    ctx.close()
    return result


def run_kopt(args, ctx, stream, device, world):
    import torch
    from cudaedgeelimination_b200 import synth
    from cudaedgeelimination_b200.api import KOPT_TEMPLATE_COUNTS

    g, tasks = synth.kopt_instance()
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    rows = sum(t.shape[0] for t in lists)
    cells = sum(t.shape[0] * KOPT_TEMPLATE_COUNTS[k] for k, t in zip(ks, lists))
    ctx.kopt_prepare_multi(g, ks, lists)
    for _ in range(args.warmup):
        ctx.kopt_launch()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    total = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()  # evict L2 (126 MB) between timed launches
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.kopt_launch()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
    ms = max_over_ranks(total / args.steps, world)
    outs = [np.empty((t.shape[0], KOPT_TEMPLATE_COUNTS[k]), np.int64) for k, t in zip(ks, lists)]
    ctx.kopt_fetch(outs)
    # end to end: H2D of the rows, launch, D2H of the full matrices into pinned buffers
    keep = [pinned_copy(t) for t in lists]
    ptasks = [k[1] for k in keep]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out_arrays, stats = ctx.kopt_costs_multi(g, ks, ptasks)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, world)
    for a, b in zip(out_arrays, outs):
        assert (a == b).all()
    peak, peak_kind = load_peaks()
    alg_bytes = rows * 48 + cells * 8 + 8 * g.n
    achieved = alg_bytes / (ms / 1e3) / 1e9
    return {"metric": "k-opt cost cells/s", "value": cells * world / (ms / 1e3), "unit": "cells/s",
            "ms_per_step": ms, "rows": rows, "cells": cells,
            "config": "15,000-node CEIL_2D instance in [0,1e6)^2, 200,000 rows k=3/4/5 in thirds, one launch; "
                      "L2 flushed (256 MB write) between timed launches",
            "e2e": {"value": cells * world / e2e_s, "unit": "cells/s", "ms_per_step": e2e_s * 1e3,
                    "h2d_bytes_per_step": int(stats.h2d_bytes), "d2h_bytes_per_step": int(stats.d2h_bytes),
                    "api": "cee_kopt_costs_multi (host buffers)"},
            "roofline": {"kernel": "kopt_cost_kernel", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": load_traffic().get("kopt_cost_kernel"), "algorithmic_bytes_per_launch": alg_bytes}}


# ---------------------------------------------------------------- plumbing ----------------

def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    """The slowest rank's time (every rank gets it)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank: int):
    if rank != 0:
        return None
    from cudaedgeelimination_b200 import synth
    batch = synth.BatchUnion(args.instances)
    threads = os.cpu_count() or 1
    # each step: the reference's CPU JV screen over a bounded sample of the batch
    budget = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        reference_jv_rate(batch, budget / 4, threads)
    rates = []
    sample = ""
    kind = "reference"
    for _ in range(args.steps):
        rate, kind, sample = reference_jv_rate(batch, budget, threads)
        rates.append(rate)
    value = float(np.median(rates))
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
            "config": {"workload": f"batching mix: {batch.count} instances (bounded sample per step)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        result = run_ours(args, rank, world, local)
        if rank == 0:
            print(json.dumps(result), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
