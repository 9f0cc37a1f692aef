"""The CPU oracle (oracle/cee_oracle.c) pinned against the reference: its known-answer tests,
its pinned template hashes, and golden fixtures the reference itself produced
(tests/golden/make_golden.py), plus a live cross-check when the reference library is built."""
import json
import pathlib

import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth
from helpers import knn_graph, random_graph

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# configs/kopt_reconnect_hashes_v1.txt of the reference (also tests/unit/test_kopt.cpp:330-352)
PINNED_TEMPLATES = {3: (4, 0xE58AF5E08D290D04), 4: (25, 0x03179E3CA191CE82), 5: (208, 0x6696DDE548591BCE)}


def load(name):
    return np.load(GOLDEN / name)


def snapshot(d, suffix=""):
    return GraphSnapshot(int(d["n"]), int(d["dist_type"]), d["x"], d["y"], d["edge_u"], d["edge_v"],
                         d["edge_w" + suffix], d["active"])


def test_reference_distance_kats(port):
    # tests/unit/test_core.cpp:44-66
    assert port.distance(0, 0, 3, 4, 0) == 5
    assert port.distance(0, 0, 1, 1, 0) == 1
    assert port.distance(0, 0, 1, 1, 1) == 2
    assert [port.isqrt(v) for v in (0, 15, 16)] == [0, 3, 4]


def test_distance_golden(port):
    kats = json.loads((GOLDEN / "distance_kats.json").read_text())
    for x1, y1, x2, y2, euc, ceil in kats["distances"]:
        assert port.distance(x1, y1, x2, y2, 0) == euc
        assert port.distance(x1, y1, x2, y2, 1) == ceil
    for value, root in kats["isqrt"]:
        assert port.isqrt(value) == root


@pytest.mark.parametrize("k", [3, 4, 5])
def test_template_tables_pinned(port, k):
    mates, h = port.kopt_templates(k)
    assert (mates.shape[0], h) == PINNED_TEMPLATES[k]
    golden = load("kopt_small.npz")
    np.testing.assert_array_equal(mates, golden[f"mates{k}"])
    for m in mates:  # perfect matchings that never re-add a deleted edge
        assert all(m[m[p]] == p and m[p] != p for p in range(2 * k))
        assert all(m[2 * e] != 2 * e + 1 for e in range(k))


@pytest.mark.parametrize("name", ["jv_small_uniform.npz", "jv_recursive_point.npz"])
def test_jv_golden(port, name):
    d = load(name)
    g = snapshot(d)
    np.testing.assert_array_equal(port.jv_screen(g), d["witness0"])
    assert port.content_hash(g) == int(d["initial_hash"])
    active, before, committed, final_hash = port.jv_eliminate(g)
    np.testing.assert_array_equal(before, d["epoch_stats"][:, 0])
    np.testing.assert_array_equal(committed, d["epoch_stats"][:, 2])
    assert final_hash == int(d["final_hash"])
    np.testing.assert_array_equal(active, d["final_active"])
    np.testing.assert_array_equal(port.ht_targets(g), d["targets"])


def test_kopt_golden(port):
    d = load("kopt_small.npz")
    for k in (3, 4, 5):
        tasks = d[f"tasks{k}"].view(np.uint8).reshape(-1, 48).copy()
        from cudaedgeelimination_b200 import KOPT_TASK_DTYPE
        tasks = tasks.view(KOPT_TASK_DTYPE).reshape(-1)
        for t in (0, 1):
            g = GraphSnapshot.from_edges(d["x"], d["y"], np.zeros((0, 2), np.int64), t)
            np.testing.assert_array_equal(port.kopt_costs(g, k, tasks), d[f"costs{k}_{t}"])


def test_cd_golden(port):
    d = load("cd_small.npz")
    for t in (0, 1):
        g = GraphSnapshot(32, t, d["x"], d["y"], d["edge_u"], d["edge_v"], d[f"edge_w_{t}"],
                          np.ones(d["edge_u"].shape[0], np.uint8))
        c, dd, a = port.cd_tasks(g, 0, 1, 0, 0)
        np.testing.assert_array_equal(c, d[f"c_{t}"])
        np.testing.assert_array_equal(dd, d[f"d_{t}"])
        np.testing.assert_array_equal(a, d[f"active_{t}"])
        for mode in (0, 1):
            flags = port.cd_screen(g, 0, 1, c, dd, a, mode)
            np.testing.assert_array_equal(flags, d[f"flags_{t}_{mode}"])
            # FinalizeCdCandidates: ranked by Hamilton reply product (all kept)
            np.testing.assert_array_equal(port.cd_finalize(g, 0, 1, c, dd, flags, 0), d[f"candidates_{t}_{mode}"])


def test_verifier_rejects_tampered_witness(port):
    """A witness replaced by an edge endpoint must be rejected (the reference's tamper test,
    tests/exhaustive/check_small_instances.py:146-165)."""
    g = synth.jv_small()
    w = port.jv_screen(g)
    e = int(np.flatnonzero(w >= 0)[0])
    assert port.jv_verify(g, e, int(w[e]))
    assert not port.jv_verify(g, e, int(g.edge_u[e]))
    assert not port.jv_verify(g, e, -1)


# ---- live cross-check against the reference library compiled from its sources ----------

@pytest.mark.parametrize("seed", range(3))
def test_jv_matches_reference_live(port, ref, seed):
    for g in (knn_graph(250, 7 + seed, seed, dist_type=seed % 2), random_graph(120, 900, seed, shuffle=True,
                                                                                 active_frac=0.85)):
        rg = ref.graph(g)
        np.testing.assert_array_equal(port.jv_screen(g), rg.jv_cpu())
        _, records, _, final_hash = rg.run_jv(1)
        assert port.jv_eliminate(g)[3] == final_hash


def test_kopt_and_cd_match_reference_live(port, ref):
    g, tasks = synth.kopt_instance(rows=900, n=800)
    rg = ref.graph(g)
    for k in (3, 4, 5):
        np.testing.assert_array_equal(port.kopt_costs(g, k, tasks[k]), rg.kopt_costs(k, tasks[k])[0])
    g = synth.jv_small()
    rg = ref.graph(g)
    for t in port.ht_targets(g)[:8]:
        u, v = int(g.edge_u[t]), int(g.edge_v[t])
        c, d, a = port.cd_tasks(g, u, v)
        rc, rd, ra = rg.cd_tasks(u, v)
        np.testing.assert_array_equal(c, rc)
        for mode in (0, 1):
            flags = port.cd_screen(g, u, v, c, d, a, mode)
            np.testing.assert_array_equal(flags, rg.cd_screen(u, v, c, d, a, mode))
            np.testing.assert_array_equal(port.cd_finalize(g, u, v, c, d, flags, 5),
                                          rg.cd_candidates(u, v, 25, 5, 50, mode, backend=1))


def test_ht_replies_golden(port):
    """Hamilton and end reply lists (AppendHtHamiltonRepliesUnchecked / AppendHtEndRepliesUnchecked,
    src/cpu/hamilton_tutte.cpp:230-282) against the reference's own EvaluateHt*Replies(kCpu) output."""
    d = load("ht_replies.npz")
    for name in ("point", "ceil"):
        g = GraphSnapshot(int(d[f"{name}_n"]), int(d[f"{name}_dist_type"]), d[f"{name}_x"], d[f"{name}_y"],
                          d[f"{name}_edge_u"], d[f"{name}_edge_v"], d[f"{name}_edge_w"], d[f"{name}_active"])
        j = 0
        while f"{name}_target_{j}" in d:
            u, v = (int(t) for t in d[f"{name}_target_{j}"])
            centers = [c for c in range(g.n) if c not in (u, v)]
            offsets, replies = port.ht_replies(g, u, v, centers)
            np.testing.assert_array_equal(offsets, d[f"{name}_offsets_{j}"])
            np.testing.assert_array_equal(replies, d[f"{name}_replies_{j}"])
            j += 1
        assert j > 0
        offsets, replies = port.ht_end_replies(g, d[f"{name}_end_tasks"])
        np.testing.assert_array_equal(offsets, d[f"{name}_end_offsets"])
        np.testing.assert_array_equal(replies, d[f"{name}_end_replies"])


def test_ht_replies_match_reference_live(port, ref):
    rng = np.random.default_rng(7)
    for g in (knn_graph(220, 7, seed=3), knn_graph(160, 12, seed=4, dist_type=1), random_graph(90, 500, seed=5)):
        rg = ref.graph(g)
        active = np.flatnonzero(g.active)
        for e in active[rng.integers(len(active), size=3)]:
            u, v = int(min(g.edge_u[e], g.edge_v[e])), int(max(g.edge_u[e], g.edge_v[e]))
            centers = np.array([c for c in rng.integers(0, g.n, 50) if c not in (u, v)], np.int32)
            offsets, replies = port.ht_replies(g, u, v, centers)
            r_offsets, r_replies, used = rg.ht_hamilton_replies(u, v, centers, backend=1)
            assert used == 1
            np.testing.assert_array_equal(offsets, r_offsets)
            np.testing.assert_array_equal(replies, r_replies)
        tasks = np.stack([g.edge_u[active[:40]], g.edge_v[active[:40]]], axis=1)
        offsets, replies = port.ht_end_replies(g, tasks)
        r_offsets, r_replies, _ = rg.ht_end_replies(tasks, backend=1)
        np.testing.assert_array_equal(offsets, r_offsets)
        np.testing.assert_array_equal(replies, r_replies)
