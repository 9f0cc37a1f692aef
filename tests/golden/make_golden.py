"""Regenerates the golden fixtures in this directory from the reference itself.

    python tests/golden/make_golden.py        (needs oracle/_ref/libcudaee_ref.so, which
                                               oracle/Makefile compiles from the reference sources)

Every expected value below is produced by the reference's own CPU code (ExactIntegerDistance,
IntegerSqrtFloor, BuildKOptReconnectTable, FindJvCandidatesCpu, RunJvElimination,
EvaluateKOptTemplateCosts, BuildCdScreenTasks, ScreenCdTasksCpu, EvaluateHtCdCandidates,
SelectHtTargetEdgeIds). The inputs are seeded synthetic snapshots built here, plus the
reference's 8-node test fixture (tests/data/recursive-point.{tsp,edg} of the reference), read
from the reference tree when this script runs.
"""
from __future__ import annotations

import json
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from cudaedgeelimination_b200 import GraphSnapshot, synth  # noqa: E402

def _reference_dir() -> pathlib.Path:
    """$CEE_REFERENCE_DIR, else the directory the oracle recipe compiles the reference from."""
    env = os.environ.get("CEE_REFERENCE_DIR")
    if env:
        return pathlib.Path(env)
    import subprocess
    out = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref-dir"], capture_output=True, text=True)
    path = pathlib.Path(out.stdout.strip()) if out.returncode == 0 and out.stdout.strip() else None
    if path is None or not (path / "tests" / "data").exists():
        raise SystemExit("make_golden.py reads the reference's test data: set CEE_REFERENCE_DIR to its source tree")
    return path


REFERENCE = _reference_dir()


def snapshot_arrays(g) -> dict:
    return {"n": np.int64(g.n), "dist_type": np.int64(g.dist_type), "x": g.x, "y": g.y, "edge_u": g.edge_u,
            "edge_v": g.edge_v, "edge_w": g.edge_w, "active": g.active}


def distance_kats(ref: oracle.Reference) -> dict:
    rng = np.random.default_rng(0xD157)
    cases = [(0, 0, 3, 4), (0, 0, 1, 1), (0, 0, 0, 0), (5, 5, 5, 6), (-7, 3, 2, -9)]
    for scale in (10, 1000, 10**6, 2**25, 2**29):
        for _ in range(40):
            cases.append(tuple(int(v) for v in rng.integers(-scale, scale, 4)))
    # squared distances just around perfect squares and q^2 + q (the EUC_2D rounding edge)
    for q in (1, 2, 3, 1000, 46340, 10**6, 2**24 + 3):
        for dy in (0, 1, 2):
            cases.append((0, 0, q, dy))
    out = []
    for x1, y1, x2, y2 in cases:
        out.append([x1, y1, x2, y2, ref.distance(x1, y1, x2, y2, 0), ref.distance(x1, y1, x2, y2, 1)])
    isqrt_in = [0, 1, 2, 3, 4, 15, 16, 17, 24, 25, 26, 2**32 - 1, 2**32, 2**52 + 1, 2**62, 2**64 - 1]
    isqrt_in += [int(v) for v in rng.integers(0, 2**62, 64, dtype=np.int64)]
    return {"distances": out, "isqrt": [[v, ref.isqrt(v)] for v in isqrt_in]}


def read_fixture() -> GraphSnapshot:
    tsp = (REFERENCE / "tests/data/recursive-point.tsp").read_text().split("\n")
    start = tsp.index("NODE_COORD_SECTION") + 1
    xs, ys = [], []
    for line in tsp[start:]:
        if line.strip() in ("", "EOF"):
            break
        _, x, y = line.split()
        xs.append(int(x))
        ys.append(int(y))
    edg = (REFERENCE / "tests/data/recursive-point.edg").read_text().split()
    count = int(edg[1])
    rows = np.array(edg[2:2 + 3 * count], np.int64).reshape(count, 3)
    return GraphSnapshot.from_edges(xs, ys, rows[:, :2], 0, weights=rows[:, 2])


def jv_case(ref: oracle.Reference, g) -> dict:
    rg = ref.graph(g)
    witness0 = rg.jv_cpu()
    targets = rg.ht_targets(1)
    stats, records, h0, h1 = rg.run_jv(1)
    return {**snapshot_arrays(g), "witness0": witness0, "epoch_stats": stats, "records": records,
            "initial_hash": np.uint64(h0), "final_hash": np.uint64(h1), "final_active": rg.active(),
            "targets": targets}


def kopt_case(ref: oracle.Reference) -> dict:
    i = np.arange(17)
    xs, ys = (7 * i) % 23, (i * i + 3 * i) % 19
    out = {"x": xs.astype(np.int64), "y": ys.astype(np.int64)}
    from cudaedgeelimination_b200.api import KOPT_TASK_DTYPE
    for k in (3, 4, 5):
        rows = [list(range(2 * k)), [0, 1, 1, 2, 3, 4, 5, 6, 7, 8][:2 * k], [(3 * p + 2) % 17 for p in range(2 * k)],
                [0, 1, 1, 2, 1, 3, 1, 4, 1, 5][:2 * k], [0, 1, 1, 2, 2, 3, 3, 4, 4, 0][:2 * k]]
        tasks = np.zeros(len(rows), KOPT_TASK_DTYPE)
        for r, ports in enumerate(rows):
            tasks[r]["port_nodes"][:len(ports)] = ports
        out[f"tasks{k}"] = tasks.view(np.uint8).reshape(len(rows), 48)
        for t in (0, 1):
            g = GraphSnapshot.from_edges(xs, ys, np.zeros((0, 2), np.int64), t)
            costs, _ = ref.graph(g).kopt_costs(k, tasks, backend=1)
            out[f"costs{k}_{t}"] = costs
        mates, h = ref.kopt_table(k)
        out[f"mates{k}"] = mates
        out[f"hash{k}"] = np.uint64(h)
    return out


def cd_case(ref: oracle.Reference) -> dict:
    i = np.arange(32)
    xs, ys = (37 * i + 11) % 101, (i * i * 13 + 7 * i) % 97
    edges = [(a, b) for a in range(32) for b in range(a + 1, 32) if (a == 0 and b == 1) or (17 * a + 13 * b) % 5 == 0]
    out = {}
    for t in (0, 1):
        g = GraphSnapshot.from_edges(xs, ys, edges, t)
        rg = ref.graph(g)
        c, d, a = rg.cd_tasks(0, 1, 0, 0)
        out.update({f"x": g.x, "y": g.y, "edge_u": g.edge_u, "edge_v": g.edge_v, "edge_w_%d" % t: g.edge_w,
                    f"c_{t}": c, f"d_{t}": d, f"active_{t}": a})
        for mode in (0, 1):
            out[f"flags_{t}_{mode}"] = rg.cd_screen(0, 1, c, d, a, mode)
            out[f"candidates_{t}_{mode}"] = rg.cd_candidates(0, 1, 0, 0, 0, mode, backend=1)
    return out


def ht_replies_case(ref: oracle.Reference) -> dict:
    """EvaluateHtHamiltonReplies / EvaluateHtEndReplies (kCpu) on the recursive-point fixture and on a
    small ceiling instance: every center of a few active target edges, and every (endpoint, internal
    neighbour) direction of the first active edges."""
    out = {}
    i = np.arange(40)
    xs, ys = (29 * i + 5) % 89, (i * i * 7 + 3 * i) % 83
    edges = [(a, b) for a in range(40) for b in range(a + 1, 40) if (11 * a + 7 * b) % 6 == 0 or b == a + 1]
    for name, g in (("point", read_fixture()), ("ceil", GraphSnapshot.from_edges(xs, ys, edges, 1))):
        rg = ref.graph(g)
        out.update({f"{name}_{k}": v for k, v in snapshot_arrays(g).items()})
        active = np.flatnonzero(g.active)
        targets = active[:: max(1, len(active) // 4)][:4]
        for j, e in enumerate(targets):
            u, v = int(min(g.edge_u[e], g.edge_v[e])), int(max(g.edge_u[e], g.edge_v[e]))
            centers = np.array([c for c in range(g.n) if c not in (u, v)], np.int32)
            offsets, replies, _ = rg.ht_hamilton_replies(u, v, centers, backend=1)
            out[f"{name}_target_{j}"] = np.array([u, v], np.int32)
            out[f"{name}_offsets_{j}"] = offsets
            out[f"{name}_replies_{j}"] = replies
        tasks = np.array([(a, b) for e in active[:60] for a, b in ((g.edge_u[e], g.edge_v[e]), (g.edge_v[e], g.edge_u[e]))],
                         np.int32)
        offsets, replies, _ = rg.ht_end_replies(tasks, backend=1)
        out[f"{name}_end_tasks"] = tasks
        out[f"{name}_end_offsets"] = offsets
        out[f"{name}_end_replies"] = replies
    return out


def main() -> None:
    ref = oracle.Reference()
    (HERE / "distance_kats.json").write_text(json.dumps(distance_kats(ref), indent=0))
    np.savez_compressed(HERE / "jv_small_uniform.npz", **jv_case(ref, synth.jv_small()))
    np.savez_compressed(HERE / "jv_recursive_point.npz", **jv_case(ref, read_fixture()))
    np.savez_compressed(HERE / "kopt_small.npz", **kopt_case(ref))
    np.savez_compressed(HERE / "cd_small.npz", **cd_case(ref))
    np.savez_compressed(HERE / "ht_replies.npz", **ht_replies_case(ref))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
