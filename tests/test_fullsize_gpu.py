"""Parity at the full benchmark sizes, against the C oracle on host threads:

  * the 200,000-row k-opt leaf cost matrix (15,000-node CEIL_2D instance, k = 3/4/5 in thirds):
    every one of its 15,799,871 cells, resident and end to end (src/cpu/kopt_search.cpp:962-1042);
  * the 4,096-instance batching mix: every instance's JV witnesses (src/cpu/jv_elimination.cpp:209-224),
    HT targets (src/cpu/ht_scan.cpp:316-345), c,d neighbourhoods and flags
    (src/cpu/hamilton_tutte.cpp:168-228) and finalised candidates (:283-327), through the graph
    launch, the plain per-instance path and the chunked end-to-end call;
  * the serving stream: a mixed sample of its jobs (JV epochs and k-opt batches on resident
    snapshots, all in the loop at once), each against the oracle.
"""
import time

import numpy as np
import pytest

from cudaedgeelimination_b200 import synth
from cudaedgeelimination_b200.api import KOPT_TEMPLATE_COUNTS, BatchOptions, ServeConfig

pytestmark = pytest.mark.gpu


def assert_batch_equal(res, want, what):
    for name in ("witness", "target_ids", "target_count", "nbhd", "flags"):
        got = getattr(res, name)
        bad = np.flatnonzero((got != want[name]).reshape(got.shape[0], -1).any(axis=1)) if got.ndim > 1 else \
            np.flatnonzero(got != want[name])
        assert bad.size == 0, f"{what}: {name} differs at {bad.size} rows, first {bad[:5]}"


def assert_candidates_equal(cand, want):
    c, d, product, count = cand
    np.testing.assert_array_equal(count, want["cand_count"])
    keep = np.arange(c.shape[2])[None, None, :] < count[:, :, None]
    np.testing.assert_array_equal(np.where(keep, c, -1), np.where(keep, want["cand_c"], -1))
    np.testing.assert_array_equal(np.where(keep, d, -1), np.where(keep, want["cand_d"], -1))
    np.testing.assert_array_equal(np.where(keep, product, -1), np.where(keep, want["cand_product"], -1))


@pytest.fixture(scope="module")
def full_batch():
    return synth.BatchUnion(4096)


@pytest.fixture(scope="module")
def full_batch_expected(port, full_batch):
    return port.batch_expect(full_batch, BatchOptions(max_cd_candidates=5))


def test_batch_all_instances(ctx, full_batch, full_batch_expected):
    opt = BatchOptions()
    ctx.batch_prepare(full_batch, opt)
    ctx.batch_launch()
    assert_batch_equal(ctx.batch_fetch(), full_batch_expected, "graph launch")
    res, _ = ctx.batch_screen(full_batch, opt)
    assert_batch_equal(res, full_batch_expected, "end-to-end call")


def test_batch_all_instances_finalised(ctx, full_batch, full_batch_expected):
    opt = BatchOptions(max_cd_candidates=5)
    ctx.batch_prepare(full_batch, opt)
    ctx.batch_launch()
    assert_batch_equal(ctx.batch_fetch(), full_batch_expected, "graph launch, finalised")
    assert_candidates_equal(ctx.batch_fetch_candidates(), full_batch_expected)
    ctx.batch_launch_plain()
    assert_batch_equal(ctx.batch_fetch(), full_batch_expected, "plain per-instance launches")
    assert_candidates_equal(ctx.batch_fetch_candidates(), full_batch_expected)


def test_kopt_matrix_all_cells(ctx, port):
    g, tasks = synth.kopt_instance()
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    assert sum(t.shape[0] * KOPT_TEMPLATE_COUNTS[k] for k, t in zip(ks, lists)) == 15_799_871
    want = [port.kopt_costs_parallel(g, k, t) for k, t in zip(ks, lists)]
    ctx.kopt_prepare_multi(g, ks, lists)
    ctx.kopt_launch()
    outs = [np.empty_like(w) for w in want]
    ctx.kopt_fetch(outs)
    for k, got, exp in zip(ks, outs, want):
        np.testing.assert_array_equal(got, exp, err_msg=f"resident matrix, k={k}")
    e2e, _ = ctx.kopt_costs_multi(g, ks, lists)
    for k, got, exp in zip(ks, e2e, want):
        np.testing.assert_array_equal(got, exp, err_msg=f"end-to-end matrix, k={k}")


def test_kopt_improving_all_rows(ctx, port):
    """Fused leaf consume on the full matrix: the improving-template masks and first improving
    template of every row equal the ones derived from the oracle's cost rows."""
    g, tasks = synth.kopt_instance()
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    masks, firsts, _, _ = ctx.kopt_improving_multi(g, ks, lists)
    for k, t, m, f in zip(ks, lists, masks, firsts):
        costs = port.kopt_costs_parallel(g, k, t)
        improving = costs < t["deleted_cost"][:, None]
        T = costs.shape[1]
        words = np.zeros((t.shape[0], -(-T // 32)), np.uint32)
        for j in range(T):
            words[:, j // 32] |= improving[:, j].astype(np.uint32) << np.uint32(j % 32)
        np.testing.assert_array_equal(m, words, err_msg=f"masks, k={k}")
        first = np.where(improving.any(axis=1), improving.argmax(axis=1), -1)
        np.testing.assert_array_equal(f, first, err_msg=f"first improving template, k={k}")


def test_serve_stream_sample(port):
    """The serving workload's first 240 jobs, submitted as fast as the loop admits them, each
    against the oracle."""
    from cudaedgeelimination_b200 import Context
    wl = synth.ServeWorkload(jobs=240)
    ctx = Context(0)
    try:
        ctx.serve_start(ServeConfig(hbm_budget_bytes=4 << 30, slots=32, idle_ms=20))
        sids = [ctx.serve_add_snapshot(g) for g in wl.jv]
        ksids = [ctx.serve_add_snapshot(g) for g, _ in wl.kopt]
        assert None not in sids and None not in ksids
        results, pending, nxt = {}, {}, 0
        t0 = time.time()
        while len(results) < len(wl.jobs):
            while nxt < len(wl.jobs):
                job = wl.jobs[nxt]
                if job[0] == "jv":
                    jid = ctx.serve_submit_jv(sids[job[1]], wl.jv[job[1]].m, nxt)
                else:
                    jid = ctx.serve_submit_kopt(ksids[job[1]], [3, 4, 5], wl.kopt_tasks(job), nxt)
                if jid is None:
                    break
                pending[jid] = nxt
                nxt += 1
            for jid, tag, res in ctx.serve_poll():
                results[tag] = res
                pending.pop(jid)
            if time.time() - t0 >= 300:
                kinds_left = sorted({wl.jobs[tag][0] for tag in pending.values()})
                pytest.fail(f"serving loop stalled: {len(results)} of {len(wl.jobs)} jobs reported, {nxt} "
                            f"submitted, pending {ctx.serve_pending()} (jobs, arena bytes), kinds still pending "
                            f"{kinds_left}, loop totals {ctx.serve_stats()}")
        ctx.serve_stop()
    finally:
        ctx.close()
    kinds = {"jv": 0, "kopt": 0}
    for idx, job in enumerate(wl.jobs):
        kinds[job[0]] += 1
        if job[0] == "jv":
            np.testing.assert_array_equal(results[idx], port.jv_screen(wl.jv[job[1]]), err_msg=f"job {idx}")
        else:
            g = wl.kopt[job[1]][0]
            for k, t, got in zip((3, 4, 5), wl.kopt_tasks(job), results[idx]):
                np.testing.assert_array_equal(got, port.kopt_costs_parallel(g, k, t), err_msg=f"job {idx} k={k}")
    assert kinds["jv"] > 100 and kinds["kopt"] > 30
