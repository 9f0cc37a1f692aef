"""Benchmark of the B200 edge-elimination screen (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Workload (default "batch"): the 4,096-instance batching mix (n log-uniform in [100, 5000],
uniform / clustered 50/50, 10-NN, EUC_2D; seeded synthetic stand-ins for the reference's TSPLIB
inputs). A step is the batched screen of every instance in one persistent, CUDA-graph-captured
launch: the JV screen of every active edge plus the HT c,d root screen (neighbourhood 25,
degree cap 50, active-incompatible) of the first 64 SelectHtTargetEdgeIds targets of every
instance. metric = JV edges screened per second over the whole job (c,d tasks/s alongside).

  value      resident inputs (uploaded once), K graph launches timed with CUDA events on the
             launching stream; inputs (~1.1 GB) exceed L2, so no flush is needed
  plain      the same work as one synchronous launch per instance (cee_batch_launch_plain)
  e2e        the same step through the C ABI from pinned host buffers: cee_batch_screen per
             step (chunked H2D of the whole batch, screens, D2H of every result, overlapped)
  roofline   batch_screen_kernel: compulsory bytes per launch (12 n + 33 m for the JV part plus
             the c,d outputs) / launch time
  kopt       the 200,000-row k-opt leaf cost matrix (k = 3/4/5 in thirds, 15,000-node CEIL_2D
             instance): cells/s resident and end to end, with its own roofline
  cpu_baseline  the reference's own CPU code for the same step (oracle/_ref, compiled from the
             reference sources): FindJvCandidatesCpu plus BuildCdScreenTasks + ScreenCdTasksCpu
             for the same targets, every instance, threads over instances
  reference_gpu  the reference's own CUDA units built for sm_100a (oracle/_ref/libcudaee_refcuda.so)
             against this project's kernels behind the same reference API (the drop-in): JV,
             k-opt and c,d seam calls, and RunJvElimination(kCuda) end to end

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
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--serve-jobs", type=int, default=10_000)
    p.add_argument("--serve-slots", type=int, default=32, help="job slots of the serving loop (1..256)")
    p.add_argument("--no-epochs", action="store_true")
    p.add_argument("--no-refgpu", action="store_true")
    p.add_argument("--part", default="all", choices=["all", "batch", "kopt", "serve", "epochs", "refgpu", "replies"],
                   help="profiling aid: run only the batched screen, the k-opt part or the serving loop")
    p.add_argument("--cpu-budget-s", type=float, default=12.0)
    p.add_argument("--cpu-leg", default=None, help=argparse.SUPPRESS)
    p.add_argument("--record-traffic", nargs=6, default=None,
                   metavar=("CSV", "KEY", "KERNEL", "PROFILE", "CAPTURE", "SCALE"),
                   help="record one ncu capture's per-launch figures in profiles/ncu_traffic.json and exit")
    return p.parse_args()


def load_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# The product sources each profiled kernel is compiled from: a capture in profiles/ncu_traffic.json
# records their digest, and a figure whose sources changed since is reported as not current.
KERNEL_SOURCES = {
    "batch_screen_kernel": ["batch_screen.cuh", "jv_screen.cuh", "device_common.cuh", "batch.cu"],
    "kopt_rows_kernel": ["kopt_rows.cuh", "kopt_cost.cuh", "device_common.cuh"],
}


def strip_comments(text: str) -> str:
    """C/C++ source without its comments and trailing blanks (string and character literals kept),
    so that a digest names the code, not its commentary."""
    out, i, n = [], 0, len(text)
    while i < n:
        c = text[i]
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            out.append(text[i:j + 1])
            i = j + 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    lines = ("".join(out)).split("\n")
    return "\n".join(line.rstrip() for line in lines if line.strip())


def source_digest(kernel: str, read=None) -> str:
    """sha256 over the kernel's source files, comments stripped (`read(name)` gives a file's text;
    default: the working tree)."""
    import hashlib
    if read is None:
        read = lambda name: (ROOT / "cudaedgeelimination_b200" / "csrc" / name).read_text()
    h = hashlib.sha256()
    for name in KERNEL_SOURCES[kernel]:
        h.update(name.encode())
        h.update(strip_comments(read(name)).encode())
    return h.hexdigest()


def load_traffic():
    path = ROOT / "profiles" / "ncu_traffic.json"
    if path.exists():
        return json.loads(path.read_text()).get("captures", {})
    return {}


def traffic_fields(key: str) -> dict:
    """The ncu figures of capture `key` (DRAM bytes per launch and their provenance), marked
    current only while the kernel's sources still have the digest recorded with the capture."""
    rec = load_traffic().get(key)
    if rec is None:
        return {"traffic": None, "traffic_unit": "DRAM bytes per launch (ncu)"}
    return {"traffic": rec["dram_bytes"], "traffic_unit": "DRAM bytes per launch (ncu)",
            "traffic_source": rec["profile"], "traffic_capture": rec["capture"],
            "traffic_current": rec["source_sha256"] == source_digest(rec["kernel"])}


def record_traffic(csv_path: str, key: str, kernel: str, profile: str, capture: str, scale: float) -> None:
    """Adds capture `key` to profiles/ncu_traffic.json from an ncu CSV of one launch of `kernel`
    (`ncu ... --csv --page raw`, or `--metrics ... --csv`): dram__bytes_read.sum +
    dram__bytes_write.sum and smsp__inst_executed.sum, times `scale` (1 for a full-size launch),
    with the digest of the kernel's sources."""
    import csv
    rows = list(csv.reader(open(csv_path)))
    values = {}
    if "Metric Name" in rows[0]:  # --metrics --csv: one row per metric
        i_name, i_val = rows[0].index("Metric Name"), rows[0].index("Metric Value")
        for r in rows[1:]:
            values[r[i_name]] = float(r[i_val].replace(",", ""))
    else:  # --page raw --csv: header, units, one row per launch
        hdr = rows[0]
        for name in ("dram__bytes_read.sum", "dram__bytes_write.sum", "smsp__inst_executed.sum"):
            if name in hdr:
                raw = float(rows[2][hdr.index(name)].replace(",", ""))
                unit = rows[1][hdr.index(name)]
                values[name] = raw * {"Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}.get(unit, 1.0)
    path = ROOT / "profiles" / "ncu_traffic.json"
    data = json.loads(path.read_text()) if path.exists() else {}
    data.setdefault("note", "Per-launch ncu figures behind bench.py's roofline objects (bench.py --record-traffic).")
    entry = {"kernel": kernel, "dram_bytes": int(round((values["dram__bytes_read.sum"] +
                                                        values["dram__bytes_write.sum"]) * scale)),
             "profile": profile, "capture": capture, "scale": scale, "source_sha256": source_digest(kernel)}
    if "smsp__inst_executed.sum" in values:
        entry["warp_instructions"] = int(round(values["smsp__inst_executed.sum"] * scale))
    data.setdefault("captures", {})[key] = entry
    path.write_text(json.dumps(data, indent=1) + "\n")


def issue_roofline(key: str, ms_per_launch: float, sm_mhz, device):
    """The instruction-issue ceiling of an ALU-bound kernel: its warp instructions per launch (capture
    `key` of profiles/ncu_traffic.json) over the live launch time, against SMs x 4 schedulers x the
    SM clock sampled during the timed region (one warp instruction per scheduler per cycle)."""
    import torch
    rec = load_traffic().get(key)
    count = None if rec is None else rec.get("warp_instructions")
    if count is None or not sm_mhz:
        return None
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    peak = sms * 4 * float(sm_mhz) * 1e6
    achieved = count / (ms_per_launch / 1e3)
    return {"unit": "warp instructions/s", "warp_instructions_per_launch": count, "achieved": achieved,
            "peak": peak, "frac": achieved / peak,
            "peak_source": f"{sms} SMs x 4 schedulers x {float(sm_mhz):.0f} MHz sampled",
            "current": rec["source_sha256"] == source_digest(rec["kernel"])}


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
            deadline = time.time() + 3.0  # nvidia-smi takes a moment to start: sample before timing
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.02)
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

def host_cpu():
    """The host's CPU model, sockets and cores (lscpu), and the threads this process may use."""
    info = {"threads_available": os.cpu_count() or 1}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            key, _, value = line.partition(":")
            key, value = key.strip(), value.strip()
            if key == "Model name":
                info["model"] = value
            elif key == "Socket(s)":
                info["sockets"] = int(value)
            elif key == "Core(s) per socket":
                info["cores_per_socket"] = int(value)
            elif key == "Thread(s) per core":
                info["threads_per_core"] = int(value)
    except (OSError, ValueError, subprocess.SubprocessError):
        pass
    return info


class ReferenceStep:
    """The reference's own CPU code for the batched step (oracle/_ref, compiled from the reference
    sources): per instance FindJvCandidatesCpu, then SelectHtTargetEdgeIds and BuildCdScreenTasks +
    ScreenCdTasksCpu for the first 64 targets (neighbourhood 25, degree cap 50,
    active-incompatible), instances on `threads` host threads inside one C++ call. Every
    instance's GraphSnapshot is built before any timing. Without the compiled reference it falls
    back to the C restatement (oracle/_build) over the same instances."""

    def __init__(self, batch, threads: int):
        import oracle
        self.batch, self.threads = batch, threads
        self.kind = "reference" if oracle.reference_available() else "port"
        if self.kind == "reference":
            self.graphs = oracle.Reference().batch_graphs(batch)
        else:
            self.port = oracle.Port()

    def run(self, instances):
        """Screens the given instances; returns (active edges screened, seconds)."""
        instances = list(instances)
        t0 = time.perf_counter()
        if self.kind == "reference":
            edges, _ = self.graphs.step(instances, self.threads)
        else:
            from cudaedgeelimination_b200.api import BatchOptions
            sub = _SubBatch(self.batch, instances)
            self.port.batch_expect(sub, BatchOptions(), self.threads)
            edges = int(sub.graph.active.sum())
        return edges, time.perf_counter() - t0


class _SubBatch:
    """A batch made of some instances of another (the C restatement's batch checker takes a union)."""

    def __init__(self, batch, instances):
        from cudaedgeelimination_b200 import GraphSnapshot
        parts = [batch.instance(i) for i in instances]
        nb = np.cumsum([0] + [g.n for g in parts]).astype(np.int64)
        eb = np.cumsum([0] + [g.m for g in parts]).astype(np.int64)
        self.node_begin, self.edge_begin = nb, eb
        self.graph = GraphSnapshot(int(nb[-1]), parts[0].dist_type, np.concatenate([g.x for g in parts]),
                                   np.concatenate([g.y for g in parts]),
                                   np.concatenate([g.edge_u + nb[i] for i, g in enumerate(parts)]),
                                   np.concatenate([g.edge_v + nb[i] for i, g in enumerate(parts)]),
                                   np.concatenate([g.edge_w for g in parts]), np.concatenate([g.active for g in parts]))


def workload_config(batch, world: int):
    """The bench line's `config`, the same in both arms."""
    g = batch.graph
    return {"workload": f"batching mix: {batch.count} instances, n log-uniform [100,5000], uniform/clustered 50/50, "
                        "10-NN, EUC_2D; per step the JV screen of every active edge plus the HT c,d root screen of "
                        "64 targets per instance (neighbourhood 25, degree cap 50, active-incompatible)",
            "instances": batch.count, "nodes": int(g.n), "edges": int(g.m),
            "l2": "inputs (~1.1 GB) larger than L2, no flush", "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------- our arm -----------------

def spot_check(batch, res, opt):
    """Cheap parity check of a few instances against the CPU oracle (the tests do the full one)."""
    import oracle
    port = oracle.Port()
    for i in range(0, batch.count, max(1, batch.count // 6)):
        inst = batch.instance(i)
        e0, e1, n0 = int(batch.edge_begin[i]), int(batch.edge_begin[i + 1]), int(batch.node_begin[i])
        w = port.jv_screen(inst)
        assert (res.witness[e0:e1] == np.where(w >= 0, w + n0, -1)).all()
        expected = port.ht_targets(inst)[:opt.targets]
        assert (res.target_ids[i, :expected.shape[0]] == expected + e0).all()
        local = int(expected[0])
        u, v = int(inst.edge_u[local]), int(inst.edge_v[local])
        c, d, a = port.cd_tasks(inst, u, v, opt.max_neighborhood, opt.max_candidate_degree)
        assert (res.pair_flags(i, 0) == port.cd_screen(inst, u, v, c, d, a, opt.cd_mode)).all()


def check_batch_full(batch, res, cand, fin_opt):
    """Every instance of the step against the C oracle on host threads: JV witnesses, HT targets,
    c,d neighbourhoods and flag words, and the finalised candidates of the finalised step."""
    import oracle
    t0 = time.perf_counter()
    want = oracle.Port().batch_expect(batch, fin_opt)
    for name in ("witness", "target_ids", "target_count", "nbhd", "flags"):
        assert np.array_equal(getattr(res, name), want[name]), f"batched step differs from the oracle in {name}"
    c, d, product, count = cand
    assert np.array_equal(count, want["cand_count"]), "finalised candidate counts differ from the oracle"
    keep = np.arange(c.shape[2])[None, None, :] < count[:, :, None]
    for got, name in ((c, "cand_c"), (d, "cand_d"), (product, "cand_product")):
        assert np.array_equal(np.where(keep, got, -1), np.where(keep, want[name], -1)), f"{name} differs"
    return {"instances": batch.count, "edges": int(res.witness.shape[0]), "targets": int(count.size),
            "checked": "every JV witness, HT target, c,d neighbourhood, flag word and finalised candidate; "
                       "graph launch, plain launches and the end-to-end call give the same bytes",
            "oracle": "oracle/cee_oracle.c on host threads", "seconds": time.perf_counter() - t0, "ok": True}


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
    if args.part == "serve":
        from cudaedgeelimination_b200 import synth as _synth
        wl = _synth.ServeWorkload(jobs=args.serve_jobs)
        return {"serve": run_serve(args, device, world, wl=wl), "serve_leaf": run_serve(args, device, world, leaf=True, wl=wl)}
    if args.part == "epochs":
        return run_fixed_point(args, device)
    if args.part == "refgpu":
        return run_reference_gpu(args, device)
    if args.part == "replies":
        return run_replies(args, device)
    from cudaedgeelimination_b200.api import BatchOptions
    batch = synth.BatchUnion(args.instances)
    g = batch.graph
    ctx = Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    n, m = g.n, g.m
    opt = BatchOptions()  # 64 targets, neighbourhood 25, degree cap 50, active-incompatible

    # ---- resident timing of the batched launch ----
    ctx.batch_prepare(batch, opt)
    from cudaedgeelimination_b200 import TuningCache
    cache = TuningCache()
    cached = cache.get(cache.key(ctx.sm_count, "batch",
                                 largest_instance=int(np.diff(batch.node_begin).max()), instances=batch.count,
                                 edges=int(g.m))) is not None
    tuning = ctx.batch_autotune(reps=2, cache=cache)
    for _ in range(args.warmup):
        ctx.batch_launch()
    res = ctx.batch_fetch()
    if rank == 0:
        spot_check(batch, res, opt)
    barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        torch.cuda.synchronize(device)
        barrier(world)
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.batch_launch()
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize(device)
        barrier(world)
    ms_step = max_over_ranks(ev0.elapsed_time(ev1), world) / args.steps
    clock_summary = clocks.summary()
    edges_step = int(g.active.sum())
    targets = int(res.target_count.sum())
    sizes = (res.nbhd >= 0).sum(axis=2)
    pairs = int((sizes * (sizes - 1) // 2).sum())
    value = edges_step * world / (ms_step / 1e3)

    # ---- the same step with the c,d candidates finalised (FinalizeCdCandidates, 5 per target) ----
    fin_opt = BatchOptions(max_cd_candidates=5)
    ctx.batch_prepare(batch, fin_opt)
    ctx.set_batch_tuning(tuning.jv_tile, tuning.blocks_per_sm, tuning.chunks)
    for _ in range(args.warmup):
        ctx.batch_launch()
    torch.cuda.synchronize(device)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        ctx.batch_launch()
    f1.record(stream)
    f1.synchronize()
    fin_ms = max_over_ranks(f0.elapsed_time(f1), world) / args.steps
    fin_cand = ctx.batch_fetch_candidates()
    fin_counts = fin_cand[3]
    ctx.batch_prepare(batch, opt)
    ctx.set_batch_tuning(tuning.jv_tile, tuning.blocks_per_sm, tuning.chunks)

    # ---- the same work, one synchronous launch per instance ----
    plain_steps = max(1, min(3, args.steps))
    ctx.batch_launch_plain()
    t0 = time.perf_counter()
    for _ in range(plain_steps):
        ctx.batch_launch_plain()
    plain_ms = max_over_ranks((time.perf_counter() - t0) / plain_steps * 1e3, world)
    plain = ctx.batch_fetch()
    assert (plain.witness == res.witness).all() and (plain.flags == res.flags).all()

    # ---- end to end through the C ABI from pinned host buffers ----
    keep = []
    host = GraphSnapshot.__new__(GraphSnapshot)
    host.n, host.dist_type = g.n, g.dist_type
    for name in ("x", "y", "edge_u", "edge_v", "edge_w", "active", "row_offsets", "neighbors", "csr_edge_ids"):
        t, a = pinned_copy(getattr(g, name))
        keep.append(t)
        setattr(host, name, a)
    hb = type("PinnedBatch", (), {})()
    for name in ("node_begin", "edge_begin"):
        t, a = pinned_copy(getattr(batch, name))
        keep.append(t)
        setattr(hb, name, a)
    from cudaedgeelimination_b200.api import _batch_outputs
    out = _batch_outputs(m, batch.count, opt)
    for name in ("witness", "target_ids", "target_count", "nbhd", "flags"):
        t, a = pinned_copy(getattr(out, name))
        keep.append(t)
        setattr(out, name, a)
    for _ in range(args.warmup):
        _, stats = ctx.batch_screen(hb, opt, graph=host, out=out)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, stats = ctx.batch_screen(hb, opt, graph=host, out=out)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world) / args.steps
    assert (out.witness == res.witness).all() and (out.flags == res.flags).all()
    e2e_value = edges_step * world / e2e_s

    # ---- roofline of the dominant kernel ----
    peak, peak_kind = load_peaks()
    out_bytes = 4 * m + targets * 4 + batch.count * 4 + res.nbhd.nbytes + res.flags.nbytes
    alg_bytes = 12 * n + 33 * m + out_bytes - 4 * m  # the witness write is already in 33 m
    achieved = alg_bytes / (ms_step / 1e3) / 1e9

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded; TSPLIB/ElimTSP inputs not shipped)",
        "config": workload_config(batch, world),
        "launch": "one persistent, CUDA-graph-captured launch per step",
        "tuning": {"jv_tile": tuning.jv_tile, "blocks_per_sm": tuning.blocks_per_sm, "chunks": tuning.chunks,
                   "source": "tuning cache" if cached else "cee_batch_autotune (stored in the tuning cache)"},
        "targets": targets, "cd_tasks": pairs,
        "cd_tasks_per_s": pairs * world / (ms_step / 1e3),
        "with_cd_finalisation": {"ms_per_step": fin_ms, "value": edges_step * world / (fin_ms / 1e3), "unit": UNIT,
                                 "candidates": int(fin_counts.sum()),
                                 "note": "same step plus FinalizeCdCandidates (reply counts, ranking, 5 per target)"},
        "plain": {"ms_per_step": plain_ms, "value": edges_step * world / (plain_ms / 1e3), "unit": UNIT,
                  "launches_per_step": batch.count, "batched_speedup": plain_ms / ms_step,
                  "api": "cee_batch_launch_plain (one synchronous launch per instance)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(stats.h2d_bytes),
                "d2h_bytes_per_step": int(stats.d2h_bytes), "ms_per_step": e2e_s * 1e3,
                "api": "cee_batch_screen (pinned host buffers, chunked copy/compute overlap)"},
        "roofline": {"kernel": "batch_screen_kernel", "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                     **traffic_fields("batch_screen_kernel"),
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "issue": issue_roofline("batch_screen_kernel", ms_step, clock_summary.get("sm_mhz"), device),
                     "note": "the screen is instruction-issue bound (integer and FP32 exact-distance work, warp "
                             "sorts and shuffles), not memory bound: see issue and distance_evals_per_s"},
        "clocks": clock_summary,
        "gpu_launches": args.steps,
    }

    # algorithmic exact-distance evaluations of the JV part (sequential CPU count) on a sample
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
        result["roofline"]["jv_distance_evals_per_edge"] = per_edge
        result["roofline"]["distance_evals_per_s"] = (per_edge * edges_step + 351 * targets) / (ms_step / 1e3)

    parity = {}
    if not args.no_kopt and args.part == "all":
        result["kopt"] = run_kopt(args, ctx, stream, device, world, parity if rank == 0 else None)
    if not args.no_serve and args.part == "all":
        from cudaedgeelimination_b200 import synth as _synth
        wl = _synth.ServeWorkload(jobs=args.serve_jobs)
        result["serve"] = run_serve(args, device, world, parity if rank == 0 else None, wl=wl)
        result["serve_leaf"] = run_serve(args, device, world, parity if rank == 0 else None, leaf=True, wl=wl)
    if not args.no_epochs and args.part == "all" and rank == 0:
        result["jv_fixed_point"] = run_fixed_point(args, device)
    if not args.no_refgpu and args.part == "all" and rank == 0:
        result["reference_gpu"] = run_reference_gpu(args, device)

    if rank == 0:
        # the reference's CPU code on the same step: every instance, one pass, all host threads
        threads = os.cpu_count() or 1
        step = ReferenceStep(batch, threads)
        cpu_edges, cpu_s = step.run(range(batch.count))
        result["cpu_baseline"] = {
            "value": cpu_edges / cpu_s, "unit": UNIT, "cores": threads, "kind": step.kind,
            "sample": f"all {batch.count} instances ({cpu_edges} edges, JV screen + 64 c,d root screens each) in "
                      f"{cpu_s:.1f} s, one C++ call on {threads} host threads, snapshots built before timing"}
        if step.kind == "reference":
            # the two parts apart on one core (FindJvCandidatesCpu; BuildCdScreenTasks + ScreenCdTasksCpu),
            # on every 16th instance
            sample = list(range(0, batch.count, 16))
            jv_s, cd_s, e1, t1 = step.graphs.parts_1core(sample)
            result["cpu_baseline"]["parts_1core"] = {
                "jv_edges_per_s": e1 / jv_s, "cd_tasks_per_s": t1 / cd_s, "cores": 1,
                "sample": f"every 16th instance ({len(sample)} instances, {e1} edges, {t1} c,d tasks): "
                          f"JV {jv_s:.2f} s, c,d {cd_s:.2f} s on one thread",
                "api": "FindJvCandidatesCpu; SelectHtTargetEdgeIds + BuildCdScreenTasks + ScreenCdTasksCpu"}
        result["host_cpu"] = host_cpu()
        # full-size parity: every instance of the timed step against the C oracle
        parity["batch"] = check_batch_full(batch, res, fin_cand, fin_opt)
        result["parity"] = parity
    ctx.close()
    return result


OMP_ENV = {"OMP_DYNAMIC": "FALSE", "OMP_PROC_BIND": "spread", "OMP_PLACES": "cores"}


def cpu_leg(name: str, timeout_s: float = 600.0):
    """Runs one CPU-baseline leg (`bench.py --cpu-leg name`) in a child process with the reference
    benchmarks' OpenMP settings, which bind threads and so stay out of this (GPU-driving) process."""
    env = dict(os.environ, **OMP_ENV)
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--cpu-leg", name], capture_output=True, text=True,
                          env=env, timeout=timeout_s)
    if proc.returncode != 0:
        raise RuntimeError(f"CPU baseline leg {name} failed:\n{proc.stdout}\n{proc.stderr}")
    return json.loads(proc.stdout.strip().splitlines()[-1])


def cpu_leg_kopt():
    """EvaluateKOptTemplateCosts(kCpu) -- the reference's OpenMP cost-matrix path
    (src/cpu/kopt_search.cpp:1069-1089, at most kKOptCpuMaxThreads = 8 threads) -- on the 200,000-row
    matrix, k = 3, 4, 5 one call each, at 1 and at 8 threads: the median of 3 repetitions after one
    warm-up, as benchmarks/kopt_cost_benchmark.cpp:53-64 times it."""
    import oracle
    from cudaedgeelimination_b200 import synth
    ref = oracle.Reference()
    g, tasks = synth.kopt_instance()
    rg = ref.graph(g)
    cells = sum(t.shape[0] * {3: 4, 4: 25, 5: 208}[k] for k, t in tasks.items())
    out = {}
    for threads in (1, 8):
        ref.set_omp_threads(threads)
        used = 0
        for k, t in tasks.items():
            used = max(used, int(rg.kopt_costs(k, t, 1)[1][0]))
        samples = []
        for _ in range(3):
            t0 = time.perf_counter()
            for k, t in tasks.items():
                rg.kopt_costs(k, t, 1)
            samples.append(time.perf_counter() - t0)
        sec = float(np.median(samples))
        out[f"threads_{threads}"] = {"value": cells / sec, "unit": "cells/s", "ms": sec * 1e3, "threads_used": used}
    return {"value": out["threads_8"]["value"], "unit": "cells/s", "cores": out["threads_8"]["threads_used"],
            "kind": "reference", "one_thread": out["threads_1"],
            "sample": f"the whole 200,000-row matrix ({cells} cells), k = 3/4/5 one call each, median of 3 after a "
                      "warm-up; EvaluateKOptTemplateCosts(kCpu), OMP_DYNAMIC=FALSE OMP_PROC_BIND=spread OMP_PLACES=cores",
            "host_cpu": host_cpu()}


def run_kopt(args, ctx, stream, device, world, parity=None):
    import torch
    from cudaedgeelimination_b200 import synth
    from cudaedgeelimination_b200.api import KOPT_TEMPLATE_COUNTS

    g, tasks = synth.kopt_instance()
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    rows = sum(t.shape[0] for t in lists)
    cells = sum(t.shape[0] * KOPT_TEMPLATE_COUNTS[k] for k, t in zip(ks, lists))
    ctx.kopt_prepare_multi(g, ks, lists)
    from cudaedgeelimination_b200 import TuningCache
    ktune = ctx.kopt_autotune(reps=3, cache=TuningCache())
    kname = "kopt_rows_kernel" if ktune.kernel == 1 else "kopt_cost_kernel"
    for _ in range(args.warmup):
        ctx.kopt_launch()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    total = 0.0
    with ClockSampler(device) as clocks, torch.cuda.stream(stream):
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
    clock_summary = clocks.summary()
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
    # fused leaf consume: improving-template masks only (the 126 MB matrix never crosses PCIe)
    masks, firsts, _, lstats = ctx.kopt_improving_multi(g, ks, ptasks)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        masks, firsts, _, lstats = ctx.kopt_improving_multi(g, ks, ptasks)
    leaf_s = max_over_ranks((time.perf_counter() - t0) / args.steps, world)
    improving_rows = int(sum(int((f >= 0).sum()) for f in firsts))
    peak, peak_kind = load_peaks()
    alg_bytes = rows * 48 + cells * 8 + 8 * g.n
    achieved = alg_bytes / (ms / 1e3) / 1e9
    large = run_kopt_large(args, ctx, stream, device, world, g, parity, kname)
    extra = {}
    if parity is not None:
        import oracle
        port = oracle.Port()
        t0 = time.perf_counter()
        for k, t, got, m, f in zip(ks, lists, outs, masks, firsts):
            want = port.kopt_costs_parallel(g, k, t)
            assert np.array_equal(got, want), f"k-opt matrix differs from the oracle (k={k})"
            better = want < t["deleted_cost"][:, None]
            words = np.zeros_like(m)
            for j in range(want.shape[1]):
                words[:, j // 32] |= better[:, j].astype(np.uint32) << np.uint32(j % 32)
            assert np.array_equal(m, words), f"improving masks differ from the oracle (k={k})"
            assert np.array_equal(f, np.where(better.any(axis=1), better.argmax(axis=1), -1)), "first improving"
        parity["kopt"] = {"rows": rows, "cells": cells, "checked": "every cell of the resident and end-to-end "
                          "matrices, every improving-template mask and first improving template",
                          "oracle": "oracle/cee_oracle.c on host threads", "seconds": time.perf_counter() - t0,
                          "ok": True}
        extra["cpu_baseline"] = cpu_leg("kopt")
        extra["vs_cpu_8_threads"] = (cells / (ms / 1e3)) / extra["cpu_baseline"]["value"]
    return {"metric": "k-opt cost cells/s", "value": cells * world / (ms / 1e3), "unit": "cells/s",
            "ms_per_step": ms, "rows": rows, "cells": cells,
            "tuning": {"kernel": "rows" if ktune.kernel == 1 else "tiled", "rows_per_tile": list(ktune.rows_per_tile),
                       "api": "cee_kopt_autotune through the tuning cache"},
            "config": "15,000-node CEIL_2D instance in [0,1e6)^2, 200,000 rows k=3/4/5 in thirds, one launch; "
                      "L2 flushed (256 MB write) between timed launches",
            "e2e": {"value": cells * world / e2e_s, "unit": "cells/s", "ms_per_step": e2e_s * 1e3,
                    "h2d_bytes_per_step": int(stats.h2d_bytes), "d2h_bytes_per_step": int(stats.d2h_bytes),
                    "api": "cee_kopt_costs_multi (host buffers)"},
            "leaf_consume": {"value": cells * world / leaf_s, "unit": "cells/s", "ms_per_step": leaf_s * 1e3,
                             "kernel_ms": lstats.kernel_ms, "d2h_bytes_per_step": int(lstats.d2h_bytes),
                             "rows_with_improving_template": improving_rows,
                             "api": "cee_kopt_improving_multi (host rows in, improving-template masks out)"},
            "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         **traffic_fields(f"{kname}_200k"),
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "issue": issue_roofline(f"{kname}_200k", ms, clock_summary.get("sm_mhz"), device),
                         "note": "the 126 MB output about fills L2, so part of it is still in L2 when the launch "
                                 "ends; larger_than_l2 is the DRAM-bound figure"},
            "clocks": clock_summary, "larger_than_l2": large, **extra}


def run_kopt_large(args, ctx, stream, device, world, g, parity, kname):
    """The same kernel on 1,000,000 rows (k = 3/4/5 in thirds, 632 MB of output, five times L2), so
    that the cells it writes must reach DRAM within the timed launch."""
    import torch
    from cudaedgeelimination_b200 import synth
    from cudaedgeelimination_b200.api import KOPT_TEMPLATE_COUNTS
    big_g, tasks = synth.kopt_instance(rows=1_000_000)
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    rows = sum(t.shape[0] for t in lists)
    cells = sum(t.shape[0] * KOPT_TEMPLATE_COUNTS[k] for k, t in zip(ks, lists))
    ctx.kopt_prepare_multi(big_g, ks, lists)
    for _ in range(args.warmup):
        ctx.kopt_launch()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.kopt_launch()
    e1.record(stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    peak, peak_kind = load_peaks()
    alg_bytes = rows * 48 + cells * 8 + 8 * big_g.n
    out = {"rows": rows, "cells": cells, "ms_per_launch": ms, "value": cells * world / (ms / 1e3), "unit": "cells/s",
           "roofline": {"kernel": kname, "bound": "hbm", "achieved": alg_bytes / (ms / 1e3) / 1e9,
                        "peak": peak, "unit": "GB/s", "frac": alg_bytes / (ms / 1e3) / 1e9 / peak,
                        "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg_bytes,
                        **traffic_fields(f"{kname}_1m")},
           "config": "1,000,000 rows of the same 15,000-node CEIL_2D instance's walks, back-to-back launches (the "
                     "632 MB output is five times L2, so every launch writes DRAM)"}
    if parity is not None:
        import oracle
        port = oracle.Port()
        outs = [np.empty((t.shape[0], KOPT_TEMPLATE_COUNTS[k]), np.int64) for k, t in zip(ks, lists)]
        ctx.kopt_fetch(outs)
        t0 = time.perf_counter()
        for k, t, got in zip(ks, lists, outs):
            assert np.array_equal(got, port.kopt_costs_parallel(big_g, k, t)), f"1M-row matrix differs (k={k})"
        parity["kopt_1m_rows"] = {"rows": rows, "cells": cells, "checked": "every cell",
                                  "seconds": time.perf_counter() - t0, "ok": True}
    return out


def _pinned_pool(count: int, nbytes: int):
    """`count` page-locked host buffers of `nbytes` each (uint8 numpy views) and their owners."""
    import torch
    owners = [torch.empty(nbytes, dtype=torch.uint8).pin_memory() for _ in range(count)]
    return owners, [t.numpy() for t in owners]


def _job_outputs(wl, job, buf, leaf: bool = False):
    """Output arrays of `job` carved from one pinned buffer: a witness array, the k-opt cost
    matrices, or with `leaf` the improving-template masks and first improving templates."""
    if job[0] == "jv":
        return buf[:4 * wl.jv[job[1]].m].view(np.int32)
    outs, at = [], 0
    if leaf:
        masks, firsts = [], []
        for (c, _), t in zip(job[2], (4, 25, 208)):
            w = (t + 31) // 32
            masks.append(buf[at:at + 4 * c * w].view(np.uint32).reshape(c, w))
            at += 4 * c * w
            firsts.append(buf[at:at + 4 * c].view(np.int32))
            at += 4 * c
        return masks, firsts
    for (c, _), t in zip(job[2], (4, 25, 208)):
        outs.append(buf[at:at + 8 * c * t].view(np.int64).reshape(c, t))
        at += 8 * c * t
    return outs


def _job_output_bytes(wl, job, leaf: bool = False) -> int:
    if job[0] == "jv" or not leaf:
        return wl.output_bytes(job)
    return sum(4 * c * ((t + 31) // 32 + 1) for (c, _), t in zip(job[2], (4, 25, 208)))


def _copy_result(res):
    if isinstance(res, tuple):
        return tuple([a.copy() for a in part] for part in res)
    return np.array(res, copy=True) if not isinstance(res, list) else [r.copy() for r in res]


def _latency_summary(lat_s):
    ms = np.asarray(lat_s) * 1e3
    return {"p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
            "mean_ms": float(ms.mean()), "max_ms": float(ms.max())}


def serve_drive(ctx, wl, sids, ksids, arrivals, buffers, keep_every: int, leaf: bool = False):
    """Feeds the jobs into the serving loop at their arrival times (admitting while it accepts
    them), polls completions, and returns (completion - arrival latencies, wall seconds, kept
    sample outputs: every keep_every-th job's, none for 0)."""
    n = len(wl.jobs)
    free = list(range(len(buffers)))
    inflight = {}
    latency = np.zeros(n)
    kept = {}
    nxt = done = 0
    t0 = time.perf_counter()
    while done < n:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now and free:
            job = wl.jobs[nxt]
            out = _job_outputs(wl, job, buffers[free[-1]], leaf)
            if job[0] == "jv":
                jid = ctx.serve_submit_jv(sids[job[1]], wl.jv[job[1]].m, nxt, out=out)
            elif leaf:
                jid = ctx.serve_submit_kopt_improving(ksids[job[1]], [3, 4, 5], wl.kopt_tasks(job), nxt, outs=out)
            else:
                jid = ctx.serve_submit_kopt(ksids[job[1]], [3, 4, 5], wl.kopt_tasks(job), nxt, outs=out)
            if jid is None:  # no slot or arena room: poll first
                break
            inflight[jid] = (nxt, free.pop())
            nxt += 1
        for jid, tag, res in ctx.serve_poll():
            idx, b = inflight.pop(jid)
            latency[idx] = time.perf_counter() - t0 - arrivals[idx]
            if keep_every and idx % keep_every == 0:
                kept[idx] = _copy_result(res)
            free.append(b)
            done += 1
    return latency, time.perf_counter() - t0, kept


def plain_drive(ctx, wl, arrivals, buffer, keep_every: int, leaf: bool = False):
    """The same jobs one at a time through the regular entry points (cee_jv_screen,
    cee_kopt_costs_multi, or with `leaf` cee_kopt_improving_multi), each started at
    max(arrival, previous completion)."""
    n = len(wl.jobs)
    latency = np.zeros(n)
    service = np.zeros(n)
    kept = {}
    t0 = time.perf_counter()
    for idx, job in enumerate(wl.jobs):
        while time.perf_counter() - t0 < arrivals[idx]:
            pass
        s0 = time.perf_counter()
        if job[0] == "jv":
            out = _job_outputs(wl, job, buffer)
            ctx.jv_screen(wl.jv[job[1]], out=out)
        elif leaf:
            masks, firsts, _, _ = ctx.kopt_improving_multi(wl.kopt[job[1]][0], [3, 4, 5], wl.kopt_tasks(job))
            out = (masks, firsts)
        else:
            out = _job_outputs(wl, job, buffer)
            ctx.kopt_costs_multi(wl.kopt[job[1]][0], [3, 4, 5], wl.kopt_tasks(job), outs=out)
        end = time.perf_counter()
        service[idx] = end - s0
        latency[idx] = end - t0 - arrivals[idx]
        if keep_every and idx % keep_every == 0:
            kept[idx] = _copy_result(out)
    return latency, service, time.perf_counter() - t0, kept


def cpu_leg_serve(jobs: int, budget_s: float = 12.0):
    """The serving stream's jobs in arrival order, one at a time, on the reference's own CPU code:
    FindJvCandidatesCpu for a JV epoch job, EvaluateKOptTemplateCosts(kCpu) per k for a k-opt job
    (OpenMP as the reference sets it: up to 8 threads). Every snapshot is built before timing; jobs
    run until the budget is spent."""
    import oracle
    from cudaedgeelimination_b200 import synth
    ref = oracle.Reference()
    wl = synth.ServeWorkload(jobs=jobs)
    jv_graphs = [ref.graph(g) for g in wl.jv]
    kopt_graphs = [ref.graph(g) for g, _ in wl.kopt]
    done = {"jv": 0, "kopt": 0}
    t0 = time.perf_counter()
    for job in wl.jobs:
        if time.perf_counter() - t0 > budget_s:
            break
        if job[0] == "jv":
            jv_graphs[job[1]].jv_cpu()
        else:
            for k, t in zip((3, 4, 5), wl.kopt_tasks(job)):
                kopt_graphs[job[1]].kopt_costs(k, t, 1)
        done[job[0]] += 1
    sec = time.perf_counter() - t0
    count = done["jv"] + done["kopt"]
    return {"value": count / sec, "unit": "jobs/s", "cores": min(8, os.cpu_count() or 1), "kind": "reference",
            "sample": f"the first {count} of {len(wl.jobs)} jobs in arrival order ({done['jv']} JV epochs, "
                      f"{done['kopt']} k-opt batches) run one at a time in {sec:.1f} s; FindJvCandidatesCpu (1 thread) "
                      "and EvaluateKOptTemplateCosts(kCpu) (OpenMP, at most 8 threads); snapshots built before timing"}


def pcie_d2h_gbs(device) -> float:
    """Pinned device-to-host bandwidth of this box: 8 copies of 512 MB."""
    import torch
    dev = torch.empty(512 << 20, dtype=torch.uint8, device=device)
    host = torch.empty(512 << 20, dtype=torch.uint8).pin_memory()
    host.copy_(dev, non_blocking=True)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(8):
        host.copy_(dev, non_blocking=True)
    torch.cuda.synchronize(device)
    return 8 * (512 << 20) / (time.perf_counter() - t0) / 1e9


def run_serve(args, device, world, parity=None, leaf: bool = False, wl=None):
    """The serving stream (Poisson arrivals at 0.8 x the loop's measured capacity) through the
    serving loop, and the same jobs run plain-sequentially through the regular entry points. With
    `leaf` the k-opt jobs return improving-template sets (the fused leaf consume) instead of cost
    matrices, in both arms."""
    from cudaedgeelimination_b200 import Context, synth
    from cudaedgeelimination_b200.api import ServeConfig

    base = synth.ServeWorkload(jobs=args.serve_jobs) if wl is None else wl
    wl = synth.ServeWorkload.__new__(synth.ServeWorkload)  # a copy whose row pools this run pins
    wl.__dict__.update(base.__dict__)
    wl.kopt = list(base.kopt)
    pinned_pools = []  # k-opt row pools in page-locked memory, as a serving caller would keep them
    for i, (g, pools) in enumerate(wl.kopt):
        pinned = {}
        for k, rows in pools.items():
            owner, view = pinned_copy(rows)
            pinned_pools.append(owner)
            pinned[k] = view
        wl.kopt[i] = (g, pinned)
    slots = args.serve_slots
    max_bytes = max(_job_output_bytes(wl, j, leaf) for j in wl.jobs)
    owners, buffers = _pinned_pool(slots + 1, max_bytes)
    ctx = Context(device)
    ctx.serve_start(ServeConfig(hbm_budget_bytes=8 << 30, slots=slots, idle_ms=20))
    sids = [ctx.serve_add_snapshot(g) for g in wl.jv]
    ksids = [ctx.serve_add_snapshot(g) for g, _ in wl.kopt]
    assert None not in sids and None not in ksids
    keep_every = max(1, len(wl.jobs) // 100)
    # warm-up on the first jobs, then capacity: every job queued at t = 0 (closed loop); the parity
    # sample is kept from the Poisson run, so the capacity runs of both arms copy no results aside
    warm = synth.ServeWorkload.__new__(synth.ServeWorkload)
    warm.__dict__.update(wl.__dict__)
    warm.jobs = wl.jobs[:min(200, len(wl.jobs))]
    serve_drive(ctx, warm, sids, ksids, np.zeros(len(warm.jobs)), buffers[:slots], 0, leaf)
    _, cap_s, _ = serve_drive(ctx, wl, sids, ksids, np.zeros(len(wl.jobs)), buffers[:slots], 0, leaf)
    capacity = len(wl.jobs) / cap_s
    lam = 0.8 * capacity
    arrivals = np.cumsum(wl.gaps) / lam
    lat, wall, kept = serve_drive(ctx, wl, sids, ksids, arrivals, buffers[:slots], keep_every, leaf)
    ctx.serve_stop()
    ctx.close()

    plain_ctx = Context(device)
    _, service, plain_closed_s, _ = plain_drive(plain_ctx, warm, np.zeros(len(warm.jobs)), buffers[slots], 0, leaf)
    _, service, plain_closed_s, _ = plain_drive(plain_ctx, wl, np.zeros(len(wl.jobs)), buffers[slots], 0, leaf)
    plain_capacity = len(wl.jobs) / plain_closed_s
    plain_lat, _, plain_wall, plain_kept = plain_drive(plain_ctx, wl, arrivals, buffers[slots], keep_every, leaf)
    plain_ctx.close()
    for idx, want in plain_kept.items():  # served results equal the regular entry points' results
        got = kept[idx]
        if isinstance(want, tuple):
            assert all((a == b).all() for g_, w_ in zip(got, want) for a, b in zip(g_, w_)), \
                f"serve/plain mismatch on job {idx}"
        elif isinstance(want, list):
            assert all((a == b).all() for a, b in zip(got, want)), f"serve/plain mismatch on job {idx}"
        else:
            assert (got == want).all(), f"serve/plain mismatch on job {idx}"
    extra = {}
    if parity is not None:  # the same sample against the C oracle
        import oracle
        port = oracle.Port()
        t0 = time.perf_counter()
        for idx, got in kept.items():
            job = wl.jobs[idx]
            if job[0] == "jv":
                assert np.array_equal(got, port.jv_screen(wl.jv[job[1]])), f"served JV job {idx} differs from the oracle"
            else:
                g = wl.kopt[job[1]][0]
                for j, (k, t) in enumerate(zip((3, 4, 5), wl.kopt_tasks(job))):
                    want = port.kopt_costs_parallel(g, k, t)
                    if not leaf:
                        assert np.array_equal(got[j], want), f"served k-opt job {idx} differs"
                        continue
                    better = want < t["deleted_cost"][:, None]
                    words = np.zeros_like(got[0][j])
                    for c in range(want.shape[1]):
                        words[:, c // 32] |= better[:, c].astype(np.uint32) << np.uint32(c % 32)
                    first = np.where(better.any(axis=1), better.argmax(axis=1), -1)
                    assert np.array_equal(got[0][j], words) and np.array_equal(got[1][j], first), \
                        f"served improving sets of job {idx} differ"
        parity["serve_leaf" if leaf else "serve"] = {
            "jobs": len(kept), "of": len(wl.jobs), "checked": "every output of every sampled job "
            "(each 100th of the Poisson run) against the C oracle and the regular entry points",
            "seconds": time.perf_counter() - t0, "ok": True}
        if not leaf:
            extra["cpu_baseline"] = cpu_leg(f"serve:{len(wl.jobs)}")
    kinds = np.array([j[0] == "jv" for j in wl.jobs])
    per_kind = {"jv": _latency_summary(lat[kinds]), "kopt": _latency_summary(lat[~kinds])}
    d2h_bytes = sum(_job_output_bytes(wl, j, leaf) for j in wl.jobs)
    ceiling = pcie_d2h_gbs(device)
    del owners, pinned_pools
    jv_jobs = sum(1 for j in wl.jobs if j[0] == "jv")
    return {
        "metric": "served jobs/s and p50/p99 latency", "jobs": len(wl.jobs), "jv_jobs": jv_jobs,
        "kopt_jobs": len(wl.jobs) - jv_jobs, "seed": wl.seed, "lambda_jobs_per_s": lam,
        "capacity_jobs_per_s": capacity, "jobs_per_s": len(wl.jobs) / wall,
        **_latency_summary(lat),
        "plain": {"capacity_jobs_per_s": plain_capacity, "jobs_per_s": len(wl.jobs) / plain_wall,
                  **_latency_summary(plain_lat), "service_p50_ms": float(np.percentile(service, 50) * 1e3),
                  "service_p99_ms": float(np.percentile(service, 99) * 1e3),
                  "api": "cee_jv_screen / " + ("cee_kopt_improving_multi" if leaf else "cee_kopt_costs_multi") +
                         ", one job at a time"},
        "capacity_speedup": capacity / plain_capacity,
        "per_kind": per_kind,
        "d2h_bytes": int(d2h_bytes),
        "d2h_gb_per_s_at_capacity": d2h_bytes / cap_s / 1e9,
        "pcie_d2h_gb_per_s": ceiling,
        "copy_engine_busy_frac": d2h_bytes / 1e9 / ceiling / cap_s,
        "copy_engine_note": "time the results need at the measured pinned D2H bandwidth (512 MB copies) over the "
                            "capacity run's wall time: near 1 means the loop is bound by PCIe, not by the SMs",
        "config": f"{len(wl.jobs)} jobs, Poisson arrivals at 0.8 x measured serving capacity; 70% JV epochs on "
                  f"{len(wl.jv)} resident instances of the batching mix (n log-uniform [200,20000]), 30% k-opt "
                  f"batches of 1k-50k rows (k = 3/4/5 in thirds) on {len(wl.kopt)} resident CEIL_2D instances, "
                  + ("returning improving-template sets (the fused leaf consume)" if leaf else
                     "returning full cost matrices") + f"; "
                  f"{slots} slots, k-opt rows and results in pinned host buffers; latency = arrival to results "
                  "on the host",
        "checked_jobs": len(plain_kept),
        **extra,
    }


def run_replies(args, device):
    """HT Hamilton replies (cee_ht_replies + fetch) of every other node of the 50,000-node 10-NN
    case as a center, against the oracle's lists: the device span of one call (count pass, offsets,
    write pass) on the context's stream and the host time of the whole call."""
    import torch
    import oracle
    from cudaedgeelimination_b200 import Context, synth
    g = synth.uniform_knn(50_000, 10_000_000, 10, 0, 7)
    e = int(np.flatnonzero(g.active)[0])
    u, v = int(min(g.edge_u[e], g.edge_v[e])), int(max(g.edge_u[e], g.edge_v[e]))
    centers = np.array([c for c in range(g.n) if c not in (u, v)], np.int32)
    ctx = Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    for _ in range(max(args.warmup, 1)):
        offsets, replies = ctx.ht_replies(g, u, v, centers)
    dev_ms, host_ms = [], []
    for _ in range(max(args.steps, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        offsets, replies = ctx.ht_replies(g, u, v, centers)
        e1.record(stream)
        e1.synchronize()
        host_ms.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(e0.elapsed_time(e1))
    ctx.close()
    want_offsets, want = oracle.Port().ht_replies(g, u, v, centers)
    assert np.array_equal(offsets, want_offsets) and np.array_equal(replies, want), "replies differ from the oracle"
    deg = np.diff(g.row_offsets)[centers].astype(np.int64)
    pairs = int((deg * (deg - 1) // 2).sum())
    ms = float(np.median(host_ms))
    return {"metric": "HT Hamilton replies/s", "value": len(replies) / (ms / 1e3), "unit": "replies/s",
            "replies": int(len(replies)), "centers": int(centers.shape[0]), "pairs_tested": pairs,
            "ms_per_call": ms, "device_span_ms": float(np.median(dev_ms)), "pairs_per_s": pairs / (ms / 1e3),
            "parity": "offsets and every reply equal the oracle's (oracle/cee_oracle.c)",
            "config": f"50,000-node uniform 10-NN EUC_2D, target ({u}, {v}), every other node a center; "
                      "snapshot resident (graph_hit), 36 MB of replies copied to host memory per call"}


def run_fixed_point(args, device):
    """JV elimination to a fixed point with every epoch on the device (cee_jv_eliminate), against
    the reference's own RunJvElimination(kCpu) loop (oracle/_ref) on the same instance."""
    import oracle
    from cudaedgeelimination_b200 import Context, synth
    cases = [("3,000-node clustered (8-NN + quadrant neighbours), EUC_2D", synth.jv_clustered()),
             ("50,000-node uniform in [0,10^7)^2, 10-NN, EUC_2D", synth.uniform_knn(50_000, 10_000_000, 10, 0, 7))]
    ctx = Context(device)
    ref = oracle.Reference() if oracle.reference_available() else None
    out = []
    for name, g in cases:
        ctx.jv_eliminate(g)  # warm-up (allocations, module load)
        t0 = time.perf_counter()
        active, witness, epoch, before, committed, stats = ctx.jv_eliminate(g)
        wall = time.perf_counter() - t0
        screened = int(before.sum())
        row = {"workload": name, "nodes": g.n, "edges": g.m, "epochs": int(stats.epochs),
               "eliminated": int(stats.committed), "ms": wall * 1e3, "edges_screened_per_s": screened / wall,
               "api": "cee_jv_eliminate (upload, every epoch on the device, download)"}
        if ref is not None:
            rg = ref.graph(g)
            t0 = time.perf_counter()
            rstats, records, _, _ = rg.run_jv(1)
            rwall = time.perf_counter() - t0
            assert np.array_equal(rg.active(), active) and np.array_equal(rstats[:, 2], committed)
            row["reference_cpu"] = {"ms": rwall * 1e3, "edges_screened_per_s": screened / rwall, "cores": 1,
                                    "api": "RunJvElimination(kCpu): screen, CPU verify, commit, hash per epoch"}
            row["speedup_vs_reference"] = rwall / wall
        out.append(row)
    ctx.close()
    return out


def run_reference_gpu(args, device):
    """The reference's own GPU path on this B200 -- its CUDA units (src/cuda/jv_cuda.cu, kopt_cost.cu,
    ht_cd.cu) compiled for sm_100a by oracle/Makefile into oracle/_ref/libcudaee_refcuda.so -- against
    this project's kernels behind the same reference API (oracle/_ref/libcudaee_dropin.so). Each CUDA
    seam call is timed on the host around the call (its uploads, launch and download included: what
    the reference's callers wait for), and RunJvElimination(kCuda) is timed end to end."""
    import oracle
    from cudaedgeelimination_b200 import synth
    if not (oracle.reference_available(variant="refcuda") and oracle.reference_available(dropin=True)):
        return {"unavailable": "oracle/_ref/libcudaee_refcuda.so or libcudaee_dropin.so is not built"}
    arms = {"reference": oracle.Reference(variant="refcuda"), "ours": oracle.Reference(dropin=True)}
    out = {"api": "the reference's CUDA seam (FindJvCandidatesCuda, detail::EvaluateKOptTemplateCostsCuda, "
                  "detail::ScreenHtCdCandidatesCuda) and RunJvElimination(kCuda); reference = its own CUDA units "
                  "built for sm_100a, ours = the drop-in shim over libcee.so",
           "timing": "host clock around each call, warm calls (caches filled by a first call, reported apart)"}
    reps = 7
    jv = []
    cases = [("3,000-node clustered (8-NN + quadrant neighbours), EUC_2D", synth.jv_clustered()),
             ("50,000-node uniform in [0,10^7)^2, 10-NN, EUC_2D", synth.uniform_knn(50_000, 10_000_000, 10, 0, 7))]
    for name, g in cases:
        row = {"workload": name, "nodes": g.n, "edges": g.m}
        witnesses = {}
        for arm, ref in arms.items():
            ms, w = ref.graph(g).seam_jv_timed(reps)
            warm = float(np.median(ms[1:]))
            row[arm] = {"first_call_ms": float(ms[0]), "ms_per_call": warm, "edges_per_s": g.m / (warm / 1e3)}
            witnesses[arm] = w
        row["same_witnesses"] = bool(np.array_equal(witnesses["reference"], witnesses["ours"]))
        row["speedup"] = row["reference"]["ms_per_call"] / row["ours"]["ms_per_call"]
        jv.append(row)
    out["jv_seam"] = jv
    g = cases[0][1]
    loop = {"workload": cases[0][0]}
    records = {}
    runs = 7  # the arms alternate; each run starts from a fresh snapshot; the first run is a warm-up
    times = {arm: [] for arm in arms}
    for r in range(runs):
        for arm, ref in arms.items():
            rg = ref.graph(g)
            t0 = time.perf_counter()
            stats, rec, _, _ = rg.run_jv(2)
            times[arm].append((time.perf_counter() - t0) * 1e3)
            loop[arm] = {"epochs": int(stats.shape[0])}
            records[arm] = rec
    for arm in arms:
        loop[arm].update({"ms": float(np.median(times[arm][1:])), "first_run_ms": times[arm][0],
                          "runs": runs - 1})
    loop["same_records"] = bool(np.array_equal(records["reference"], records["ours"]))
    loop["speedup"] = loop["reference"]["ms"] / loop["ours"]["ms"]
    loop["api"] = "RunJvElimination(kCuda) to a fixed point: seam screen, CPU verify, commit, hash per epoch"
    out["jv_elimination_loop"] = loop
    kg, tasks = synth.kopt_instance()
    kopt = {"workload": "200,000 rows k = 3/4/5 in thirds, 15,000-node CEIL_2D", "cells": 0}
    mats = {}
    for arm, ref in arms.items():
        rg = ref.graph(kg)
        total = first = 0.0
        mats[arm] = []
        for k in (3, 4, 5):
            ms, costs = rg.seam_kopt_timed(k, tasks[k], 4)
            total += float(np.median(ms[1:]))
            first += float(ms[0])
            mats[arm].append(costs)
        kopt[arm] = {"ms_per_matrix": total, "first_call_ms": first}
    kopt["cells"] = int(sum(m.size for m in mats["ours"]))
    for arm in arms:
        kopt[arm]["cells_per_s"] = kopt["cells"] / (kopt[arm]["ms_per_matrix"] / 1e3)
    kopt["same_cells"] = all(np.array_equal(a, b) for a, b in zip(mats["reference"], mats["ours"]))
    kopt["speedup"] = kopt["reference"]["ms_per_matrix"] / kopt["ours"]["ms_per_matrix"]
    out["kopt_seam"] = kopt
    batch = synth.BatchUnion(256)
    cd = {"workload": "the first 256 instances of the batching mix, their first 64 targets each "
                      "(neighbourhood 25, degree cap 50, active-incompatible); task lists built before timing"}
    flags = {}
    for arm, ref in arms.items():
        rb = ref.batch_graphs(batch)
        sec, count, set_ = rb.seam_cd_timed(list(range(batch.count)))
        cd[arm] = {"seconds": sec, "cd_tasks": count, "cd_tasks_per_s": count / sec}
        flags[arm] = (count, set_)
    cd["same_flags_checksum"] = flags["reference"] == flags["ours"]
    cd["speedup"] = cd["reference"]["seconds"] / cd["ours"]["seconds"]
    out["cd_seam"] = cd
    # detail::EvaluateHtHamiltonRepliesCuda: every other node of the 50,000-node case as a center
    g = cases[1][1]
    e = int(np.flatnonzero(g.active)[0])
    u, v = int(min(g.edge_u[e], g.edge_v[e])), int(max(g.edge_u[e], g.edge_v[e]))
    centers = np.array([c for c in range(g.n) if c not in (u, v)], np.int32)
    replies = {"workload": f"{cases[1][0]}; target ({u}, {v}), {centers.shape[0]:,} centers"}
    totals = {}
    for arm, ref in arms.items():
        ms, totals[arm] = ref.graph(g).seam_ht_replies_timed(u, v, centers, 5)
        replies[arm] = {"first_call_ms": float(ms[0]), "ms_per_call": float(np.median(ms[1:])), "replies": totals[arm]}
    replies["same_total"] = totals["reference"] == totals["ours"]
    replies["speedup"] = replies["reference"]["ms_per_call"] / replies["ours"]["ms_per_call"]
    out["ht_reply_seam"] = replies
    return out


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


def run_reference(args, rank: int, world: int):
    """The reference arm: the reference's own CPU code for the batched step (ReferenceStep) on every
    host thread. A step is a stratified eighth of the batch -- instances s mod 8, s + 8, ... for
    step s -- so eight consecutive steps cover every instance once; value = edges / seconds over
    the timed steps. Under torchrun only rank 0 runs it."""
    if rank != 0:
        return None
    from cudaedgeelimination_b200 import synth
    batch = synth.BatchUnion(args.instances)
    threads = os.cpu_count() or 1
    step = ReferenceStep(batch, threads)
    stride = 8
    for s in range(args.warmup):
        step.run(range(s % stride, batch.count, stride))
    edges = seconds = 0.0
    for s in range(args.steps):
        e, sec = step.run(range(s % stride, batch.count, stride))
        edges += e
        seconds += sec
    value = edges / seconds
    sample = (f"each step every {stride}th instance ({batch.count // stride} of {batch.count}; offsets rotate so "
              f"{stride} steps cover the batch), {int(edges)} edges over {args.steps} steps in {seconds:.1f} s, "
              f"one C++ call per step on {threads} host threads, snapshots built before timing")
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded; TSPLIB/ElimTSP inputs not shipped)", "config": workload_config(batch, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": step.kind, "sample": sample},
            "host_cpu": host_cpu(),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.record_traffic is not None:
        csv_path, key, kernel, profile, capture, scale = args.record_traffic
        record_traffic(csv_path, key, kernel, profile, capture, float(scale))
        return
    if args.cpu_leg is not None:  # a CPU-baseline child process (see cpu_leg)
        name, _, arg = args.cpu_leg.partition(":")
        out = cpu_leg_kopt() if name == "kopt" else cpu_leg_serve(int(arg or 10_000), args.cpu_budget_s)
        print(json.dumps(out), flush=True)
        return
    if args.impl == "reference":
        out = run_reference(args, rank, world)
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
