"""Batched screen (many instances, one persistent graph-captured launch) against the CPU oracle:
per instance the JV witnesses, the HT targets (SelectHtTargetEdgeIds order), and per target the
c,d task list (BuildCdScreenTasks) and its flags (ScreenCdTasksCpu) -- all exact. The
one-launch-per-instance path and the chunked end-to-end call must give the same bytes."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth
from cudaedgeelimination_b200.api import BatchOptions

pytestmark = pytest.mark.gpu


class TinyBatch:
    """A hand-built batch: instances of varied size including degenerate ones."""

    def __init__(self, graphs):
        nb = np.cumsum([0] + [g.n for g in graphs]).astype(np.int64)
        eb = np.cumsum([0] + [g.m for g in graphs]).astype(np.int64)
        self.node_begin, self.edge_begin, self.count = nb, eb, len(graphs)
        self.graph = GraphSnapshot(int(nb[-1]), graphs[0].dist_type, np.concatenate([g.x for g in graphs]),
                                   np.concatenate([g.y for g in graphs]),
                                   np.concatenate([g.edge_u + nb[i] for i, g in enumerate(graphs)]),
                                   np.concatenate([g.edge_v + nb[i] for i, g in enumerate(graphs)]),
                                   np.concatenate([g.edge_w for g in graphs]), np.concatenate([g.active for g in graphs]))
        self.graphs = graphs

    def instance(self, i):
        return self.graphs[i]


def check_against_oracle(port, batch, res, opt, instances=None):
    g = batch.graph
    np.testing.assert_array_equal(res.witness, port.jv_screen(g))
    T, NB = opt.targets, opt.max_neighborhood
    for i in instances if instances is not None else range(batch.count):
        inst = batch.instance(i)
        n0, e0 = int(batch.node_begin[i]), int(batch.edge_begin[i])
        expected = port.ht_targets(inst)[:T]
        assert res.target_count[i] == expected.shape[0]
        np.testing.assert_array_equal(res.target_ids[i, :expected.shape[0]], expected + e0)
        assert (res.target_ids[i, expected.shape[0]:] == -1).all()
        for t, local in enumerate(expected):
            u, v = int(inst.edge_u[local]), int(inst.edge_v[local])
            c, d, a = port.cd_tasks(inst, u, v, NB, opt.max_candidate_degree)
            hood = res.nbhd[i, t]
            size = int((hood >= 0).sum())
            ii, jj = np.triu_indices(size, 1)
            gc = np.minimum(hood[ii], hood[jj]) - n0
            gd = np.maximum(hood[ii], hood[jj]) - n0
            np.testing.assert_array_equal(gc, c)
            np.testing.assert_array_equal(gd, d)
            np.testing.assert_array_equal(res.pair_flags(i, t), port.cd_screen(inst, u, v, c, d, a, opt.cd_mode))
        for t in range(expected.shape[0], T):
            assert (res.nbhd[i, t] == -1).all() and (res.flags[i, t] == 0).all()


@pytest.fixture(scope="module")
def small_batch():
    return synth.BatchUnion(48)


@pytest.mark.parametrize("opt", [BatchOptions(), BatchOptions(10, 8, 0, 1), BatchOptions(40, 32, 50, 0)],
                         ids=["defaults", "t10-nb8-nocap-missing", "t40-nb32"])
def test_batch_graph_launch(ctx, port, small_batch, opt):
    ctx.batch_prepare(small_batch, opt)
    ctx.batch_launch()
    res = ctx.batch_fetch()
    check_against_oracle(port, small_batch, res, opt, instances=range(0, 48, 5))


def test_plain_e2e_and_autotune_agree(ctx, small_batch):
    opt = BatchOptions()
    ctx.batch_prepare(small_batch, opt)
    ctx.batch_launch()
    graph_res = ctx.batch_fetch()
    ctx.batch_launch_plain()
    plain_res = ctx.batch_fetch()
    for chunks in (1, 3, 8):
        ctx.set_batch_tuning(64, 0, chunks)
        e2e_res, stats = ctx.batch_screen(small_batch, opt)
        assert stats.h2d_bytes > 0 and stats.d2h_bytes > 0
        for a, b in ((graph_res, plain_res), (graph_res, e2e_res)):
            for name in ("witness", "target_ids", "target_count", "nbhd", "flags"):
                np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
    chosen = ctx.batch_autotune(reps=1)
    assert chosen.jv_tile > 0
    ctx.batch_launch()
    tuned = ctx.batch_fetch()
    np.testing.assert_array_equal(tuned.witness, graph_res.witness)
    np.testing.assert_array_equal(tuned.flags, graph_res.flags)


def test_degenerate_instances(ctx, port):
    from helpers import complete_graph
    graphs = [GraphSnapshot.from_edges([0, 5, 9, 20], [0, 3, 1, 4], [(0, 1), (1, 2), (2, 3)]),  # no eligible target
              complete_graph([0, 10, 0, 10, 5], [0, 0, 10, 10, 5]),                             # 5 nodes < nb
              synth.batch_instance(3), complete_graph(list(range(0, 90, 9)), [(7 * i) % 31 for i in range(10)])]
    batch = TinyBatch(graphs)
    for opt in (BatchOptions(), BatchOptions(64, 4, 0, 1)):
        ctx.batch_prepare(batch, opt)
        ctx.batch_launch()
        check_against_oracle(port, batch, ctx.batch_fetch(), opt)
        res, _ = ctx.batch_screen(batch, opt)
        check_against_oracle(port, batch, res, opt)


def grid_knn(side, k, seed, copies=1):
    """Points of a side x side integer grid (each repeated `copies` times at the same place), shuffled:
    many equal doubled-midpoint distances, so the neighbourhood order hinges on the node-id ties."""
    rng = np.random.default_rng(seed)
    xs = np.repeat(np.tile(np.arange(side) * 7, side), copies)
    ys = np.repeat(np.repeat(np.arange(side) * 7, side), copies)
    order = rng.permutation(xs.shape[0])
    xs, ys = xs[order], ys[order]
    n = xs.shape[0]
    d2 = (xs[:, None] - xs[None, :]) ** 2 + (ys[:, None] - ys[None, :]) ** 2
    np.fill_diagonal(d2, np.iinfo(np.int64).max)
    edges = set()
    for i in range(n):
        for j in np.lexsort((np.arange(n), d2[i]))[:k]:
            edges.add((min(i, int(j)), max(i, int(j))))
    return GraphSnapshot.from_edges(xs, ys, sorted(edges), 0)


def test_spatial_chunks_ties_caps_and_large(ctx, port):
    """The chunked neighbourhood search (instances up to 8,192 nodes) against the oracle's full scan:
    grids with equal distances and co-located nodes (ties by node id), a degree cap that leaves few
    eligible nodes, and an instance above the chunked size (full scan)."""
    from helpers import knn_graph
    graphs = [grid_knn(24, 8, seed=1), grid_knn(12, 6, seed=2, copies=3), knn_graph(600, 10, seed=3),
              synth.uniform_knn(9000, 200_000, 6, 0, 4)]
    batch = TinyBatch(graphs)
    for opt in (BatchOptions(), BatchOptions(16, 25, 9, 0), BatchOptions(8, 32, 0, 1)):
        ctx.batch_prepare(batch, opt)
        ctx.batch_launch()
        check_against_oracle(port, batch, ctx.batch_fetch(), opt)
        res, _ = ctx.batch_screen(batch, opt)
        check_against_oracle(port, batch, res, opt)


def test_e2e_weight_range(ctx):
    """The end-to-end call narrows weights to int32 on the host: weights outside [0, 2^31) fail with
    CEE_ERR_RANGE, as in the resident prepare."""
    from cudaedgeelimination_b200._native import CEE_ERR_RANGE, NativeError
    batch = TinyBatch([synth.batch_instance(0), synth.batch_instance(1)])
    for bad in (-1, 1 << 31):
        g = batch.graph.copy()
        g.edge_w = g.edge_w.copy()
        g.edge_w[g.m - 3] = bad
        with pytest.raises(NativeError) as err:
            ctx.batch_screen(batch, BatchOptions(), graph=g)
        assert err.value.code == CEE_ERR_RANGE
        with pytest.raises(NativeError) as err:
            ctx.batch_prepare(batch, BatchOptions(), graph=g)
        assert err.value.code == CEE_ERR_RANGE
    res, _ = ctx.batch_screen(batch, BatchOptions())  # the context stays usable
    assert res.witness.shape == (batch.graph.m,)


def test_unsorted_instance_rejected(ctx):
    g = synth.batch_instance(0)
    swapped = GraphSnapshot(g.n, 0, g.x, g.y, g.edge_u[::-1].copy(), g.edge_v[::-1].copy(), g.edge_w[::-1].copy(),
                            g.active)
    batch = TinyBatch([swapped])
    from cudaedgeelimination_b200._native import NativeError
    with pytest.raises(NativeError):
        ctx.batch_prepare(batch, BatchOptions())
    with pytest.raises(NativeError):
        ctx.batch_screen(batch, BatchOptions())


def test_upper_ends_out_of_order_rejected(ctx):
    """Two edges with the same lower end, their upper ends swapped: the end-to-end call checks the
    lower ends on host threads and the upper ends on the device; both paths reject the list."""
    from cudaedgeelimination_b200._native import CEE_ERR_INVALID, NativeError
    g = synth.batch_instance(0, n_lo=300, n_hi=300)
    e = int(np.flatnonzero(g.edge_u[:-1] == g.edge_u[1:])[0])
    u, v, w = g.edge_u.copy(), g.edge_v.copy(), g.edge_w.copy()
    v[[e, e + 1]] = v[[e + 1, e]]
    w[[e, e + 1]] = w[[e + 1, e]]
    batch = TinyBatch([synth.batch_instance(1, n_lo=300, n_hi=300), GraphSnapshot(g.n, g.dist_type, g.x, g.y, u, v, w,
                                                                                   g.active)])
    with pytest.raises(NativeError) as err:
        ctx.batch_screen(batch, BatchOptions())
    assert err.value.code == CEE_ERR_INVALID
    with pytest.raises(NativeError):
        ctx.batch_prepare(batch, BatchOptions())
    res, _ = ctx.batch_screen(TinyBatch([g]), BatchOptions())  # the context stays usable
    assert res.witness.shape == (g.m,)


def test_csr_row_leaving_its_instance(ctx):
    """Every instance here has at most 8,192 nodes, so the screen keys candidates by node id relative
    to the edge's endpoint; a CSR row that names a node of another instance more than 8,191 ids away
    fails the neighbour bounds test (CEE_ERR_INVALID), resident and end to end, and the context stays
    usable."""
    from cudaedgeelimination_b200._native import CEE_ERR_INVALID, NativeError
    batch = TinyBatch([synth.batch_instance(0, n_lo=300, n_hi=300), synth.batch_instance(1, n_lo=8000, n_hi=8000),
                       synth.batch_instance(2, n_lo=300, n_hi=300)])
    g = batch.graph.copy()
    g.neighbors = g.neighbors.copy()
    far = int(batch.node_begin[3]) - 1  # the last node of the third instance
    for x in range(0, 300, 37):  # the last slot of a few rows of the first instance (rows stay ascending)
        g.neighbors[g.row_offsets[x + 1] - 1] = far
    with pytest.raises(NativeError) as err:
        ctx.batch_prepare(batch, BatchOptions(), graph=g)
        ctx.batch_launch()
        ctx.batch_fetch()
    assert err.value.code == CEE_ERR_INVALID
    with pytest.raises(NativeError) as err:
        ctx.batch_screen(batch, BatchOptions(), graph=g)
    assert err.value.code == CEE_ERR_INVALID
    res, _ = ctx.batch_screen(batch, BatchOptions())
    assert res.witness.shape == (batch.graph.m,)


def check_candidates(port, batch, opt, cand, instances):
    """Finalised c,d candidates equal FinalizeCdCandidates over the oracle's tasks and flags."""
    c, d, product, count = cand
    K = opt.max_cd_candidates
    for i in instances:
        inst = batch.instance(i)
        n0 = int(batch.node_begin[i])
        for t, local in enumerate(port.ht_targets(inst)[:opt.targets]):
            u, v = int(inst.edge_u[local]), int(inst.edge_v[local])
            tc, td, ta = port.cd_tasks(inst, u, v, opt.max_neighborhood, opt.max_candidate_degree)
            flags = port.cd_screen(inst, u, v, tc, td, ta, opt.cd_mode)
            want = port.cd_finalize(inst, u, v, tc, td, flags, K)
            k = int(count[i, t])
            assert k == want.shape[0]
            np.testing.assert_array_equal(c[i, t, :k] - n0, want[:, 0])
            np.testing.assert_array_equal(d[i, t, :k] - n0, want[:, 1])
            np.testing.assert_array_equal(product[i, t, :k], want[:, 2])


@pytest.mark.parametrize("opt", [BatchOptions(max_cd_candidates=5), BatchOptions(targets=8, cd_mode=1, max_cd_candidates=32),
                                 BatchOptions(targets=16, max_neighborhood=32, max_candidate_degree=0, max_cd_candidates=3)],
                         ids=["default-5", "missing-or-incompatible-32", "nb32-nocap-3"])
def test_finalised_candidates(ctx, port, small_batch, opt):
    ctx.batch_prepare(small_batch, opt)
    ctx.batch_launch()
    res = ctx.batch_fetch()
    check_against_oracle(port, small_batch, res, opt, instances=range(0, small_batch.count, 6))
    cand = ctx.batch_fetch_candidates()
    check_candidates(port, small_batch, opt, cand, range(small_batch.count))
    assert (cand[3] > 0).any()


def test_finalised_candidates_match_reference(ctx, ref, small_batch):
    opt = BatchOptions(max_cd_candidates=5)
    ctx.batch_prepare(small_batch, opt)
    ctx.batch_launch()
    res = ctx.batch_fetch()
    c, d, product, count = ctx.batch_fetch_candidates()
    for i in range(0, small_batch.count, 8):
        inst = small_batch.instance(i)
        rg = ref.graph(inst)
        n0 = int(small_batch.node_begin[i])
        for t in range(int(res.target_count[i])):
            local = int(res.target_ids[i, t] - small_batch.edge_begin[i])
            u, v = int(inst.edge_u[local]), int(inst.edge_v[local])
            want = rg.cd_candidates(u, v, 25, 5, 50, 0, backend=1)
            k = int(count[i, t])
            got = np.stack([c[i, t, :k] - n0, d[i, t, :k] - n0, product[i, t, :k]], 1)
            np.testing.assert_array_equal(got, want)


def hub_graph(n, k, hub_degrees, seed):
    """A k-nearest-neighbour graph whose hubs, the nodes nearest node 0, are joined to their nearest
    hub_degrees[h] nodes: the first targets (node 0's edges) get neighbourhood nodes with rows
    longer than a warp and than the pair table."""
    from helpers import knn_graph
    g = knn_graph(n, k, seed=seed)
    edges = set(zip(g.edge_u.tolist(), g.edge_v.tolist()))
    d2 = (g.x[:, None] - g.x[None, :]) ** 2 + (g.y[:, None] - g.y[None, :]) ** 2
    hubs = np.lexsort((np.arange(n), d2[0]))[1:len(hub_degrees) + 1]
    for h, deg in zip(hubs, hub_degrees):
        for j in np.lexsort((np.arange(n), d2[h]))[1:deg + 1]:
            edges.add((min(int(h), int(j)), max(int(h), int(j))))
    return GraphSnapshot.from_edges(g.x, g.y, sorted(edges), 0)


def test_finalised_candidates_long_rows(ctx, port):
    # reply counts at centers of degree 20 to 140: one neighbour per lane up to 32, the shared pair
    # table up to 64, the closed-form pair index beyond
    graphs = [hub_graph(400, 6, [33, 64, 65, 140], seed=4), hub_graph(300, 8, [31, 32, 63, 100], seed=5)]
    batch = TinyBatch(graphs)
    for opt in (BatchOptions(targets=64, max_candidate_degree=0, max_cd_candidates=8),
                BatchOptions(targets=32, max_neighborhood=32, max_candidate_degree=0, cd_mode=1, max_cd_candidates=32)):
        ctx.batch_prepare(batch, opt)
        ctx.batch_launch()
        check_against_oracle(port, batch, ctx.batch_fetch(), opt)
        cand = ctx.batch_fetch_candidates()
        check_candidates(port, batch, opt, cand, range(batch.count))
        assert (cand[3] > 0).any()
