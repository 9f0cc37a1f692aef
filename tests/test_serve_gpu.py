"""Serving loop on the B200: each job's result equals the regular entry point's on the same
snapshot and the same job run alone, whatever other jobs share the persistent kernel; small
cases are also checked against the CPU oracle. Covers slot reuse, the idle exit and relaunch,
HBM-budget admission (CEE_BUSY) and malformed requests."""
import time

import numpy as np
import pytest

from cudaedgeelimination_b200 import KOPT_TASK_DTYPE, Context, synth
from cudaedgeelimination_b200._native import CEE_ERR_INVALID, CEE_ERR_STATE, NativeError
from cudaedgeelimination_b200.api import ServeConfig
from helpers import knn_graph, random_graph

pytestmark = pytest.mark.gpu


def random_tasks(g, k, rows, seed, repeats=False):
    """k-opt rows with random ports (repeated ports when `repeats`), any node ids in range."""
    rng = np.random.default_rng(seed)
    tasks = np.zeros(rows, KOPT_TASK_DTYPE)
    pool = g.n if not repeats else min(g.n, 2 * k - 2)
    base = rng.integers(0, g.n, pool)
    tasks["port_nodes"][:, :2 * k] = base[rng.integers(0, pool, (rows, 2 * k))]
    tasks["deleted_cost"] = rng.integers(0, 1 << 20, rows)
    return tasks


def drain(c, want, limit_s=60.0):
    out = {}
    t0 = time.time()
    while len(out) < want:
        for job, tag, res in c.serve_poll():
            out[tag] = res
        assert time.time() - t0 < limit_s, f"serving loop stalled ({len(out)} of {want} jobs back)"
    return out


def submit(c, fn, *args, **kwargs):
    """Submits, polling the loop while it answers CEE_BUSY; returns the completions seen meanwhile."""
    seen = {}
    t0 = time.time()
    while True:
        job = fn(*args, **kwargs)
        if job is not None:
            return job, seen
        for _, tag, res in c.serve_poll():
            seen[tag] = res
        assert time.time() - t0 < 60.0, "admission never succeeded"


@pytest.fixture(scope="module")
def snapshots():
    wide = knn_graph(400, 8, seed=31, coord=1 << 28)      # coordinate span >= 2^26: wide distance path
    sparse = random_graph(500, 1500, seed=32, active_frac=0.7)
    ceil = knn_graph(300, 6, seed=33, dist_type=1)
    kg, ktasks = synth.kopt_instance(rows=3000, n=2000)
    return {"small": synth.jv_small(), "clustered": synth.jv_clustered(), "wide": wide, "sparse": sparse,
            "ceil": ceil, "kopt": kg, "_ktasks": ktasks}


def job_list(snaps):
    """(tag, snapshot name, kind, payload): JV jobs on every snapshot and k-opt jobs of 1..3 segments."""
    jobs = []
    tag = 1
    for name in ("small", "clustered", "wide", "sparse", "ceil", "kopt"):
        jobs.append((tag, name, "jv", None))
        tag += 1
    kt = snaps["_ktasks"]
    jobs.append((tag, "kopt", "kopt", ([3, 4, 5], [kt[3], kt[4], kt[5]])))
    tag += 1
    jobs.append((tag, "kopt", "kopt", ([5], [kt[5][:777]])))
    tag += 1
    for i, name in enumerate(("wide", "ceil", "small")):
        for k in (3, 4, 5):
            jobs.append((tag, name, "kopt", ([k], [random_tasks(snaps[name], k, 301 + 17 * k, 40 + i * 3 + k,
                                                             repeats=(k + i) % 2 == 0)])))
            tag += 1
    jobs.append((tag, "ceil", "kopt", ([4, 3], [random_tasks(snaps["ceil"], 4, 50, 61, True),
                                              random_tasks(snaps["ceil"], 3, 1, 62)])))
    tag += 1
    # improving-template sets (the fused leaf consume), on walk rows and on random repeated ports
    jobs.append((tag, "kopt", "improving", ([3, 4, 5], [kt[3][:1000], kt[4][:999], kt[5][:1001]])))
    tag += 1
    jobs.append((tag, "wide", "improving", ([5, 4], [random_tasks(snaps["wide"], 5, 130, 71, True),
                                                   random_tasks(snaps["wide"], 4, 77, 72)])))
    return jobs


def run_jobs(c, snaps, ids, jobs):
    results = {}
    for tag, name, kind, payload in jobs:
        if kind == "jv":
            _, seen = submit(c, c.serve_submit_jv, ids[name], snaps[name].m, tag)
        elif kind == "improving":
            _, seen = submit(c, c.serve_submit_kopt_improving, ids[name], payload[0], payload[1], tag)
        else:
            _, seen = submit(c, c.serve_submit_kopt, ids[name], payload[0], payload[1], tag)
        results.update(seen)
    results.update(drain(c, len(jobs) - len(results)))
    return results


def expected(ctx, snaps, job):
    tag, name, kind, payload = job
    g = snaps[name]
    if kind == "jv":
        return ctx.jv_screen(g)[0]
    if kind == "improving":
        masks, firsts, _, _ = ctx.kopt_improving_multi(g, payload[0], payload[1])
        return masks, firsts
    outs, _ = ctx.kopt_costs_multi(g, payload[0], payload[1])
    return outs


def assert_same(kind, got, want):
    if kind == "jv":
        np.testing.assert_array_equal(got, want)
    elif kind == "improving":
        for got_list, want_list in zip(got, want):
            assert len(got_list) == len(want_list)
            for a, b in zip(got_list, want_list):
                np.testing.assert_array_equal(a, b)
    else:
        assert len(got) == len(want)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("slots", [64, 2], ids=["slots64", "slots2"])
def test_mix_matches_regular_and_alone(ctx, snapshots, slots):
    jobs = job_list(snapshots)
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=256 << 20, slots=slots, idle_ms=5))
        ids = {name: c.serve_add_snapshot(g) for name, g in snapshots.items() if not name.startswith("_")}
        assert all(v is not None for v in ids.values())
        mixed = run_jobs(c, snapshots, ids, jobs)
        assert sorted(mixed) == [j[0] for j in jobs]
        for job in jobs:
            assert_same(job[2], mixed[job[0]], expected(ctx, snapshots, job))
        # the same jobs alone, one at a time, with the kernel idle in between
        for job in jobs[::3]:
            alone = run_jobs(c, snapshots, ids, [job])
            assert_same(job[2], alone[job[0]], mixed[job[0]])
        assert c.serve_pending()[0] == 0
        for sid in ids.values():
            c.serve_release_snapshot(sid)
        assert c.serve_pending() == (0, 0)
        c.serve_stop()
    finally:
        c.close()


def test_oracle_small(port, snapshots):
    g = snapshots["small"]
    k_tasks = random_tasks(g, 4, 64, 7, repeats=True)
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=64 << 20, slots=4, idle_ms=5))
        sid = c.serve_add_snapshot(g)
        c.serve_submit_jv(sid, g.m, tag=1)
        c.serve_submit_kopt(sid, [4], [k_tasks], tag=2)
        c.serve_submit_kopt_improving(sid, [4], [k_tasks], tag=3)
        res = drain(c, 3)
        np.testing.assert_array_equal(res[1], port.jv_screen(g))
        costs = port.kopt_costs(g, 4, k_tasks)
        np.testing.assert_array_equal(res[2][0], costs)
        better = costs < k_tasks["deleted_cost"][:, None]  # the reference's consumer's test
        masks, firsts = res[3]
        want = np.zeros_like(masks[0])
        for t in range(costs.shape[1]):
            want[:, t // 32] |= better[:, t].astype(np.uint32) << np.uint32(t % 32)
        np.testing.assert_array_equal(masks[0], want)
        np.testing.assert_array_equal(firsts[0], np.where(better.any(axis=1), better.argmax(axis=1), -1))
        c.serve_stop()
    finally:
        c.close()


def test_idle_exit_and_relaunch(ctx, snapshots):
    g = snapshots["sparse"]
    want = ctx.jv_screen(g)[0]
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=64 << 20, slots=2, idle_ms=1))
        sid = c.serve_add_snapshot(g)
        for i in range(6):
            submit(c, c.serve_submit_jv, sid, g.m, i)
            np.testing.assert_array_equal(drain(c, 1)[i], want)
            time.sleep(0.02)  # the kernel leaves after about 1 ms without work
        c.serve_stop()
    finally:
        c.close()


def test_snapshot_upload_while_jobs_run(ctx, snapshots):
    """Adding a snapshot stops the running kernel and resumes its jobs afterwards."""
    big = synth.uniform_knn(20_000, 1_000_000, 10, 0, 78)
    later = snapshots["ceil"]
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=256 << 20, slots=8, idle_ms=50))
        sid = c.serve_add_snapshot(big)
        for t in range(4):
            c.serve_submit_jv(sid, big.m, tag=t)
        lid = c.serve_add_snapshot(later)  # while the four jobs are on the GPU
        c.serve_submit_jv(lid, later.m, tag=10)
        res = drain(c, 5)
        want = ctx.jv_screen(big)[0]
        for t in range(4):
            np.testing.assert_array_equal(res[t], want)
        np.testing.assert_array_equal(res[10], ctx.jv_screen(later)[0])
        c.serve_stop()
    finally:
        c.close()


def test_admission_and_release(snapshots):
    big, small = synth.uniform_knn(20_000, 1_000_000, 10, 0, 77), snapshots["small"]  # ~4 MB resident
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=1 << 20, slots=8, idle_ms=5))
        assert c.serve_add_snapshot(big) is None          # over the budget: CEE_BUSY
        sid = c.serve_add_snapshot(small)
        assert sid is not None
        used_snapshot = c.serve_pending()[1]
        assert 0 < used_snapshot <= 1 << 20
        jobs = [c.serve_submit_jv(sid, small.m, tag=t) for t in range(8)]
        assert all(j is not None for j in jobs)
        assert c.serve_submit_jv(sid, small.m, tag=99) is None  # every slot taken: CEE_BUSY
        drain(c, 8)
        assert c.serve_pending() == (0, used_snapshot)
        c.serve_release_snapshot(sid)
        assert c.serve_pending() == (0, 0)
        assert c.serve_add_snapshot(big) is None
        c.serve_stop()
    finally:
        c.close()


def test_downloads_start_without_polling(ctx, snapshots):
    """A job's downloads are queued at submission behind a device wait for its completion: jobs left
    alone finish and land in their host buffers with no poll in between, so the first poll after a
    pause returns every one of them, with the regular entry points' results."""
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=64 << 20, slots=8, idle_ms=2000))
        jobs = job_list(snapshots)[:8]
        ids = {name: c.serve_add_snapshot(snapshots[name]) for name in {j[1] for j in jobs}}
        for tag, name, kind, payload in jobs:
            if kind == "jv":
                assert c.serve_submit_jv(ids[name], snapshots[name].m, tag) is not None
            else:
                assert c.serve_submit_kopt(ids[name], payload[0], payload[1], tag) is not None
        time.sleep(2.0)
        first = {tag: res for _, tag, res in c.serve_poll()}
        assert sorted(first) == sorted(j[0] for j in jobs)
        for job in jobs:
            assert_same(job[2], first[job[0]], expected(ctx, snapshots, job))
        c.serve_stop()
    finally:
        c.close()


def test_stop_with_jobs_in_flight(snapshots):
    """cee_serve_stop with jobs still on the GPU returns (their queued downloads are released), and
    the context serves again after a new cee_serve_start."""
    big = synth.uniform_knn(20_000, 1_000_000, 10, 0, 78)
    c = Context(0)
    try:
        for _ in range(2):
            c.serve_start(ServeConfig(hbm_budget_bytes=256 << 20, slots=16, idle_ms=50))
            sid = c.serve_add_snapshot(big)
            for t in range(16):
                assert c.serve_submit_jv(sid, big.m, tag=t) is not None
            t0 = time.monotonic()
            c.serve_stop()
            assert time.monotonic() - t0 < 30
        c.serve_start(ServeConfig(hbm_budget_bytes=64 << 20, slots=4, idle_ms=50))
        sid = c.serve_add_snapshot(snapshots["small"])
        c.serve_submit_jv(sid, snapshots["small"].m, tag=7)
        np.testing.assert_array_equal(drain(c, 1)[7], c.jv_screen(snapshots["small"])[0])
        c.serve_stop()
    finally:
        c.close()


def test_empty_jobs(snapshots):
    g = snapshots["small"].copy()
    g.active[:] = 0
    g.rebuild_csr()
    empty = random_graph(10, 0, seed=5)
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=16 << 20, slots=2, idle_ms=5))
        sid = c.serve_add_snapshot(g)
        eid = c.serve_add_snapshot(empty)
        c.serve_submit_jv(sid, g.m, tag=1)
        c.serve_submit_jv(eid, 0, tag=2)
        c.serve_submit_kopt(sid, [3], [np.zeros(0, KOPT_TASK_DTYPE)], tag=3)
        res = drain(c, 3)
        assert (res[1] == -1).all() and res[2].shape == (0,) and res[3][0].shape == (0, 4)
        c.serve_stop()
    finally:
        c.close()


def test_malformed_requests(snapshots):
    g = snapshots["small"]
    c = Context(0)
    try:
        with pytest.raises(NativeError) as e:
            c.serve_submit_jv(0, g.m)
        assert e.value.code == CEE_ERR_STATE
        c.serve_start(ServeConfig(hbm_budget_bytes=16 << 20, slots=2, idle_ms=5))
        sid = c.serve_add_snapshot(g)
        for bad in (lambda: c.serve_submit_jv(sid + 5, g.m),
                    lambda: c.serve_submit_kopt(sid, [6], [np.zeros(1, KOPT_TASK_DTYPE)]),
                    lambda: c.serve_submit_kopt(sid, [3, 3, 3, 3], [np.zeros(1, KOPT_TASK_DTYPE)] * 4),
                    lambda: c.serve_release_snapshot(sid + 9)):
            with pytest.raises(NativeError) as e:
                bad()
            assert e.value.code == CEE_ERR_INVALID
        # a port node out of range is found by the device bounds checks (the submission reads no
        # row on the host): that job completes with CEE_ERR_INVALID, the next one with CEE_OK
        bad_ports = random_tasks(g, 3, 4, 1)
        bad_ports["port_nodes"][2, 1] = g.n + 3
        bad_id = c.serve_submit_kopt(sid, [3], [bad_ports], tag=1)
        good_id = c.serve_submit_kopt(sid, [3], [random_tasks(g, 3, 4, 2)], tag=2)
        status = {}
        t0 = time.monotonic()
        while len(status) < 2 and time.monotonic() - t0 < 30:
            for job, tag, _, st in c.serve_poll(with_status=True):
                status[job] = st
        assert status == {bad_id: CEE_ERR_INVALID, good_id: 0}
        assert c.serve_pending()[0] == 0
        c.serve_stop()
    finally:
        c.close()


def test_rows_pinned_unaligned_and_pageable(ctx, snapshots):
    """k-opt rows from page-locked memory (16-byte aligned or not) and from pageable memory all give
    the regular entry point's cells; the loop's counters record the jobs and the bytes moved."""
    import torch
    g, kt = snapshots["kopt"], snapshots["_ktasks"]
    rows = np.ascontiguousarray(kt[5][:2000])
    want = ctx.kopt_costs_multi(g, [5], [rows])[0][0]
    nb = rows.nbytes
    owner = torch.empty(nb + 64, dtype=torch.uint8).pin_memory()
    base = owner.numpy()
    aligned = base[:nb].view(KOPT_TASK_DTYPE)
    unaligned = base[4:4 + nb].view(KOPT_TASK_DTYPE)
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=256 << 20, slots=4, idle_ms=20))
        sid = c.serve_add_snapshot(g)
        for tag, arr in ((1, unaligned), (2, aligned), (3, rows.copy())):
            arr[:] = rows
            before = c.serve_stats()
            assert c.serve_submit_kopt(sid, [5], [arr], tag) is not None
            got = drain(c, 1)[tag]
            np.testing.assert_array_equal(got[0], want)
            after = c.serve_stats()
            assert after["rows_bytes"] - before["rows_bytes"] == nb
            assert after["download_bytes"] - before["download_bytes"] == want.nbytes
        assert after["jobs"] == 3
        c.serve_stop()
    finally:
        c.close()


def test_jv_witness_written_in_place(ctx, snapshots):
    """A page-locked witness buffer is written by the kernel in place (no download), a pageable one
    and a page-locked one at an address that is not 4-byte aligned get a copy; all three equal the
    regular entry point's witnesses, and the counters say which path each took."""
    import torch
    g = snapshots["clustered"]
    want = ctx.jv_screen(g)[0]
    nb = 4 * g.m
    owner = torch.empty(nb + 64, dtype=torch.uint8).pin_memory()
    base = owner.numpy()
    in_place = base[:nb].view(np.int32)
    odd = np.frombuffer(base[2:2 + nb].data, dtype=np.int32)
    c = Context(0)
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=64 << 20, slots=4, idle_ms=20))
        sid = c.serve_add_snapshot(g)
        for tag, out, direct in ((1, in_place, True), (2, np.empty(g.m, np.int32), False), (3, odd, False)):
            out[:] = -7
            before = c.serve_stats()
            assert c.serve_submit_jv(sid, g.m, tag, out=out) is not None
            got = drain(c, 1)[tag]
            np.testing.assert_array_equal(got, want)
            np.testing.assert_array_equal(out, want)
            after = c.serve_stats()
            moved = (after["direct_bytes"] - before["direct_bytes"], after["download_bytes"] - before["download_bytes"])
            assert moved == ((nb, 0) if direct else (0, nb)), (tag, moved)
        c.serve_stop()
    finally:
        c.close()


def test_job_errors_stay_with_their_job(ctx, snapshots):
    """Device bounds checks are reported per job. A k-opt job whose pinned rows the caller rewrites
    with an out-of-range node after the submit-time check (the device copies them late) may fail
    with CEE_ERR_INVALID -- but only that job: a job run beside it and the jobs after it return
    CEE_OK with the regular entry point's results, and the loop stops cleanly."""
    import torch
    from cudaedgeelimination_b200._native import CEE_OK
    g, kt = snapshots["kopt"], snapshots["_ktasks"]
    good = kt[4][:500]
    want = ctx.kopt_costs_multi(g, [4], [good])[0][0]
    rows = np.tile(kt[5], 20)[:50_000]
    owner = torch.from_numpy(rows.view(np.uint8).reshape(-1).copy()).pin_memory()
    c = Context(0)
    saw_error = False
    try:
        c.serve_start(ServeConfig(hbm_budget_bytes=256 << 20, slots=4, idle_ms=20))
        sid = c.serve_add_snapshot(g)
        for attempt in range(12):
            pinned = owner.numpy().view(KOPT_TASK_DTYPE)
            pinned[:] = rows
            c.serve_submit_kopt(sid, [5], [pinned], tag=1)
            pinned["port_nodes"][-2000:, 0] = g.n + 7  # after the check, before or after the copy
            c.serve_submit_kopt(sid, [4], [good], tag=2)
            status, out = {}, {}
            t0 = time.time()
            while len(status) < 2:
                for _, tag, res, st in c.serve_poll(with_status=True):
                    status[tag], out[tag] = st, res
                assert time.time() - t0 < 60, "serving loop stalled"
            assert status[2] == CEE_OK
            np.testing.assert_array_equal(out[2][0], want)
            assert status[1] in (CEE_OK, CEE_ERR_INVALID)
            c.serve_submit_kopt(sid, [4], [good], tag=3)  # the job after a failed one
            after = drain(c, 1)
            np.testing.assert_array_equal(after[3][0], want)
            if status[1] == CEE_ERR_INVALID:
                saw_error = True
                break
        c.serve_stop()
    finally:
        c.close()
    if not saw_error:
        pytest.skip("the rewritten rows were always copied before the rewrite; isolation checked on clean jobs only")
