"""k-opt leaf cost matrices on the B200 against the CPU oracle: int64 cells bit-exact."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import KOPT_TASK_DTYPE, BuildKOptReconnectTable, GraphSnapshot, synth
from cudaedgeelimination_b200 import _native
from cudaedgeelimination_b200._native import NativeError

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[(1, 0), (0, 0), (0, 2)], ids=["rows-kernel", "tiled-default", "tiled-small"])
def kc(ctx, request):
    """The context with each k-opt kernel: the one-thread-per-row kernel with the proper templates
    compiled in (the default wherever it applies), then the tiled kernel with its default tiles and
    with small tiles (many partial tiles)."""
    kernel, tile = request.param
    ctx.set_option(_native.OPT_KOPT_KERNEL, kernel)
    for opt, rows in zip((_native.OPT_KOPT_ROWS_K3, _native.OPT_KOPT_ROWS_K4, _native.OPT_KOPT_ROWS_K5),
                         (tile * 4, tile * 3, tile)):
        ctx.set_option(opt, rows)
    yield ctx
    ctx.set_option(_native.OPT_KOPT_KERNEL, 1)
    for opt in (_native.OPT_KOPT_ROWS_K3, _native.OPT_KOPT_ROWS_K4, _native.OPT_KOPT_ROWS_K5):
        ctx.set_option(opt, 0)

INVALID = np.iinfo(np.int64).max


def coords_only(xs, ys, dist_type=0):
    return GraphSnapshot.from_edges(xs, ys, np.zeros((0, 2), np.int64), dist_type)


def make_tasks(g, k, ports_rows):
    tasks = np.zeros(len(ports_rows), KOPT_TASK_DTYPE)
    for r, ports in enumerate(ports_rows):
        tasks[r]["port_nodes"][:len(ports)] = ports
        tasks[r]["deleted_cost"] = sum(g.distance(ports[2 * e], ports[2 * e + 1]) for e in range(k))
    return tasks


def seventeen():
    # the small point set of the reference's matrix test: x = 7i mod 23, y = (i^2 + 3i) mod 19
    i = np.arange(17)
    return (7 * i) % 23, (i * i + 3 * i) % 19


@pytest.mark.parametrize("dist_type", [0, 1])
def test_consecutive_adjacent_and_strided_ports(kc, port, dist_type):
    g = coords_only(*seventeen(), dist_type)
    for k in (3, 4, 5):
        rows = [list(range(2 * k)), [0, 1, 1, 2, 3, 4, 5, 6, 7, 8][:2 * k],
                [(3 * p + 2) % 17 for p in range(2 * k)]]
        tasks = make_tasks(g, k, rows)
        table = BuildKOptReconnectTable(k)
        gpu, _ = kc.kopt_costs(g, table, tasks)
        cpu = port.kopt_costs(g, k, tasks, table.templates)
        np.testing.assert_array_equal(gpu, cpu)
        assert (gpu[1] == INVALID).any()  # shared ports produce invalid cells


def test_repeated_rows(kc, port):
    g = coords_only(*seventeen())
    tasks = make_tasks(g, 5, [list(range(10))] * 40)
    table = BuildKOptReconnectTable(5)
    gpu, _ = kc.kopt_costs(g, table, tasks)
    np.testing.assert_array_equal(gpu, port.kopt_costs(g, 5, tasks))
    assert (gpu == gpu[0]).all()


@pytest.mark.parametrize("dist_type", [0, 1])
def test_walk_rows_all_k(kc, port, dist_type):
    g, tasks = synth.kopt_instance(rows=6001, n=3000)
    if dist_type == 0:
        g = GraphSnapshot(g.n, 0, g.x, g.y, g.edge_u, g.edge_v, g.edge_w, g.active)
    for k in (3, 4, 5):
        table = BuildKOptReconnectTable(k)
        gpu, _ = kc.kopt_costs(g, table, tasks[k])
        np.testing.assert_array_equal(gpu, port.kopt_costs(g, k, tasks[k]))


def test_multi_segment_matches_single(kc, port):
    g, tasks = synth.kopt_instance(rows=3001, n=2000)
    outs, stats = kc.kopt_costs_multi(g, [3, 4, 5], [tasks[3], tasks[4], tasks[5]])
    for k, out in zip((3, 4, 5), outs):
        np.testing.assert_array_equal(out, port.kopt_costs(g, k, tasks[k]))
    # odd row counts and a single row
    outs, _ = kc.kopt_costs_multi(g, [5, 3], [tasks[5][:1], tasks[3][:7]])
    np.testing.assert_array_equal(outs[0], port.kopt_costs(g, 5, tasks[5][:1]))
    np.testing.assert_array_equal(outs[1], port.kopt_costs(g, 3, tasks[3][:7]))


def test_cache_contract(ctx, port):
    """Snapshot / template / workspace hits as the reference's test_kopt.cpp:224-234, 322-324."""
    ctx.clear(2)
    g = coords_only(*seventeen())
    rows = {k: make_tasks(g, k, [list(range(2 * k))] * 3) for k in (3, 4, 5)}
    for k in (3, 4, 5):
        _, s = ctx.kopt_costs(g, BuildKOptReconnectTable(k), rows[k])
        assert s.snapshot_hit == (k != 3) and not s.template_hit and s.resident_bytes > 0
    _, s = ctx.kopt_costs(g, BuildKOptReconnectTable(5), rows[5])
    assert s.snapshot_hit and s.template_hit and s.workspace_hit
    ceil = GraphSnapshot(g.n, 1, g.x, g.y, g.edge_u, g.edge_v, g.edge_w, g.active)
    gpu, s = ctx.kopt_costs(ceil, BuildKOptReconnectTable(5), rows[5])
    np.testing.assert_array_equal(gpu, port.kopt_costs(ceil, 5, rows[5]))
    assert not s.snapshot_hit and s.template_hit and s.workspace_hit


def test_bad_template_rejected(ctx):
    g = coords_only(*seventeen())
    table = BuildKOptReconnectTable(3)
    table.templates = table.templates.copy()
    table.templates[0, 0] = table.templates[0, 1]  # no longer a perfect matching
    with pytest.raises(NativeError):
        ctx.kopt_costs(g, table, make_tasks(g, 3, [list(range(6))]))


def test_caller_templates_readding_deleted_edges(kc, port):
    """A caller table may hold matchings that pair port 2e with 2e+1; every such cell re-adds a
    deleted edge and is invalid, on rows with and without repeated nodes."""
    g = coords_only(*seventeen())
    rng = np.random.default_rng(5)
    for k in (3, 4, 5):
        P = 2 * k
        mates = []
        for _ in range(40):  # random perfect matchings, many of them improper
            perm = rng.permutation(P)
            m = np.full(14, 0xFF, np.uint8)
            for a, b in zip(perm[0::2], perm[1::2]):
                m[a], m[b] = b, a
            mates.append(m)
        table = BuildKOptReconnectTable(k)
        table.templates = np.concatenate([table.templates[:8], np.array(mates, np.uint8)])
        rows = [list(rng.integers(0, 17, P)) for _ in range(60)] + [list(range(P)), list(range(1, P + 1))]
        tasks = make_tasks(g, k, rows)
        gpu, _ = kc.kopt_costs(g, table, tasks)
        np.testing.assert_array_equal(gpu, port.kopt_costs(g, k, tasks, table.templates))


def test_heavily_repeated_ports(kc, port):
    """Nodes shared by several deleted edges: a node in three deleted edges (k=3), a closed
    5-cycle where every node repeats (k=5, the maximum number of duplicate sets), and runs."""
    g = coords_only(*seventeen())
    cases = {3: [[0, 1, 1, 2, 1, 3], [5, 6, 6, 7, 7, 5], [2, 9, 9, 4, 4, 11]],
             4: [[0, 1, 1, 2, 1, 3, 1, 4], [0, 1, 1, 2, 2, 3, 3, 0], [3, 4, 4, 5, 6, 7, 7, 8]],
             5: [[0, 1, 1, 2, 2, 3, 3, 4, 4, 0], [0, 1, 1, 2, 1, 3, 1, 4, 1, 5], [2, 3, 3, 4, 4, 5, 9, 10, 10, 11]]}
    for k, rows in cases.items():
        tasks = make_tasks(g, k, rows)
        table = BuildKOptReconnectTable(k)
        gpu, _ = kc.kopt_costs(g, table, tasks)
        np.testing.assert_array_equal(gpu, port.kopt_costs(g, k, tasks))


def tour_rows(k, rng, n, per_pattern=3):
    """Rows cut from tours: for every gap pattern g (bit e: deleted edges e and e+1 adjacent in the tour,
    bit k-1: the last and the first), `per_pattern` rows of random distinct tour nodes."""
    rows = []
    for g in range(1 << k):
        for _ in range(per_pattern):
            pos, p = [], 0
            for e in range(k):
                pos.append(p)
                p += 1 if (g >> e) & 1 and e < k - 1 else 2 + int(rng.integers(0, 3))
            length = pos[-1] + 1 if (g >> (k - 1)) & 1 else pos[-1] + 2 + int(rng.integers(0, 3))
            tour = rng.choice(n, length, replace=False)
            rows.append([int(tour[q]) for e in range(k) for q in (pos[e], (pos[e] + 1) % length)])
    return rows


@pytest.mark.parametrize("dist_type", [0, 1])
def test_every_gap_pattern(kc, port, dist_type):
    """Tour rows of every gap pattern (the recognised rows whose validity comes from the per-template
    pattern masks), interleaved with rows of other repeats (the class-code path), in the same tiles."""
    rng = np.random.default_rng(17 + dist_type)
    xs, ys = rng.integers(0, 50_000, 400), rng.integers(0, 50_000, 400)
    g = coords_only(xs, ys, dist_type)
    for k in (3, 4, 5):
        rows = tour_rows(k, rng, 400)
        other = [list(rng.integers(0, 12, 2 * k)) for _ in range(len(rows) // 2)]  # arbitrary repeats
        mixed = [r for pair in zip(rows, other + rows[len(other):]) for r in pair]
        tasks = make_tasks(g, k, mixed)
        table = BuildKOptReconnectTable(k)
        gpu, _ = kc.kopt_costs(g, table, tasks)
        np.testing.assert_array_equal(gpu, port.kopt_costs(g, k, tasks))


def expected_improving(costs, deleted):
    """Bit masks and first index of the templates with cost < deleted cost, row by row."""
    better = costs < deleted[:, None]
    words = (costs.shape[1] + 31) // 32
    masks = np.zeros((costs.shape[0], words), np.uint32)
    for t in range(costs.shape[1]):
        masks[:, t // 32] |= (better[:, t].astype(np.uint32) << np.uint32(t % 32))
    first = np.where(better.any(axis=1), better.argmax(axis=1), -1).astype(np.int32)
    return masks, first


@pytest.mark.parametrize("with_costs", [False, True], ids=["masks-only", "with-costs"])
def test_improving_sets(kc, port, with_costs):
    """Fused leaf consume: improving-template masks and first improving template per row equal the
    ones the reference's consumer would try -- templates whose oracle cost is strictly below the
    row's deleted cost (src/cpu/kopt_search.cpp:694-715) -- on walk rows whose deleted costs are
    shifted both ways (kept >= 0, as ValidateKOptCostTask requires, :784-807)."""
    g, rows = synth.kopt_instance(rows=6000, n=3000)
    lists = []
    rng = np.random.default_rng(3)
    for k in (3, 4, 5):
        t = rows[k].copy()
        shifted = t["deleted_cost"] + rng.integers(-2000, 2000, t.shape[0])  # a spread of improving and not
        t["deleted_cost"] = np.maximum(shifted, 0)
        lists.append(t)
    oracle_costs = [port.kopt_costs(g, k, t) for k, t in zip((3, 4, 5), lists)]
    masks, firsts, costs, stats = kc.kopt_improving_multi(g, [3, 4, 5], lists, with_costs=with_costs)
    for seg in range(3):
        want_m, want_f = expected_improving(oracle_costs[seg], lists[seg]["deleted_cost"])
        np.testing.assert_array_equal(masks[seg], want_m)
        np.testing.assert_array_equal(firsts[seg], want_f)
        if with_costs:
            np.testing.assert_array_equal(costs[seg], oracle_costs[seg])
    assert any((f >= 0).any() for f in firsts) and any((f < 0).any() for f in firsts)


def test_autotune_keeps_cells_and_caches_the_shape(ctx, port, tmp_path):
    """cee_kopt_autotune times the row kernel and three tiled shapes on the prepared launch and keeps
    the fastest; the cells are the oracle's under the chosen shape, and a second context applies the
    shape stored in the tuning cache instead of timing."""
    from cudaedgeelimination_b200 import Context, TuningCache
    g, tasks = synth.kopt_instance(rows=6000, n=3000)
    ks = [3, 4, 5]
    lists = [tasks[k] for k in ks]
    cache = TuningCache(tmp_path / "tuning.json")
    try:
        ctx.kopt_prepare_multi(g, ks, lists)
        chosen = ctx.kopt_autotune(reps=2, cache=cache)
        assert chosen.kernel in (0, 1) and chosen.ms > 0
        ctx.kopt_launch()
        outs = [np.empty((t.shape[0], {3: 4, 4: 25, 5: 208}[k]), np.int64) for k, t in zip(ks, lists)]
        ctx.kopt_fetch(outs)
        for k, t, got in zip(ks, lists, outs):
            np.testing.assert_array_equal(got, port.kopt_costs(g, k, t))
        stored = TuningCache(tmp_path / "tuning.json")
        other = Context(0)
        try:
            other.kopt_prepare_multi(g, ks, lists)
            again = other.kopt_autotune(reps=2, cache=stored)
            assert again.kernel == chosen.kernel and list(again.rows_per_tile) == list(chosen.rows_per_tile)
        finally:
            other.close()
    finally:
        ctx.set_kopt_tuning(1, (0, 0, 0))


def test_large_pageable_copies(ctx, port):
    """Matrices and task rows above the staging threshold, in pageable memory, go through the
    context's pinned staging buffers (several 16 MB chunks, host threads, odd sizes): the cells still
    equal the oracle's, for rows uploaded and cells downloaded that way."""
    g, tasks = synth.kopt_instance(rows=360_003, n=5000)
    k5 = np.ascontiguousarray(tasks[5][:120_001])  # 5.8 MB of rows in, 200 MB of cells out
    k3 = np.ascontiguousarray(tasks[3][:1001])
    outs, _ = ctx.kopt_costs_multi(g, [5, 3], [k5, k3])
    assert outs[0].nbytes > (64 << 20)
    np.testing.assert_array_equal(outs[0], port.kopt_costs_parallel(g, 5, k5))
    np.testing.assert_array_equal(outs[1], port.kopt_costs(g, 3, k3))
