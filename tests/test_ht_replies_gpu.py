"""HT Hamilton and end replies on the B200 (cee_ht_replies / cee_ht_end_replies) against the CPU
oracle: offsets and lists identical, in the reference's order; the reference's own batch entry
points run them through the drop-in seam and compare them with their CPU lists themselves."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth
from cudaedgeelimination_b200._native import CEE_ERR_INVALID, NativeError
from helpers import complete_graph, knn_graph, random_graph

pytestmark = pytest.mark.gpu


def graphs():
    return [knn_graph(300, 6, seed=11), knn_graph(200, 10, seed=12, dist_type=1), synth.jv_clustered(),
            random_graph(150, 700, seed=13, active_frac=0.8), knn_graph(120, 40, seed=14),  # rows > 32
            knn_graph(400, 8, seed=15, coord=1 << 28)]  # wide coordinate span


def targets(g, rng, k):
    active = np.flatnonzero(g.active)
    for e in active[rng.integers(len(active), size=k)]:
        yield int(min(g.edge_u[e], g.edge_v[e])), int(max(g.edge_u[e], g.edge_v[e]))


@pytest.mark.parametrize("index", range(6))
def test_hamilton_replies_match_oracle(ctx, port, index):
    g = graphs()[index]
    rng = np.random.default_rng(index)
    for u, v in targets(g, rng, 4):
        centers = np.array([c for c in rng.integers(0, g.n, 300) if c not in (u, v)], np.int32)  # repeats too
        offsets, replies = ctx.ht_replies(g, u, v, centers)
        want_offsets, want = port.ht_replies(g, u, v, centers)
        np.testing.assert_array_equal(offsets, want_offsets)
        np.testing.assert_array_equal(replies, want)
    every = np.array([c for c in range(g.n) if c not in (u, v)], np.int32)
    offsets, replies = ctx.ht_replies(g, u, v, every)
    want_offsets, want = port.ht_replies(g, u, v, every)
    np.testing.assert_array_equal(offsets, want_offsets)
    np.testing.assert_array_equal(replies, want)


@pytest.mark.parametrize("index", range(6))
def test_end_replies_match_oracle(ctx, port, index):
    g = graphs()[index]
    active = np.flatnonzero(g.active)
    tasks = np.concatenate([np.stack([g.edge_u[active], g.edge_v[active]], axis=1),
                            np.stack([g.edge_v[active], g.edge_u[active]], axis=1)])
    offsets, replies = ctx.ht_end_replies(g, tasks)
    want_offsets, want = port.ht_end_replies(g, tasks)
    np.testing.assert_array_equal(offsets, want_offsets)
    np.testing.assert_array_equal(replies, want)


def test_complete_graph_and_empty_lists(ctx, port):
    i = np.arange(40)
    g = complete_graph((37 * i) % 101, (53 * i + 7) % 97)
    offsets, replies = ctx.ht_replies(g, 0, 1, np.arange(2, 40, dtype=np.int32))
    want_offsets, want = port.ht_replies(g, 0, 1, range(2, 40))
    np.testing.assert_array_equal(offsets, want_offsets)
    np.testing.assert_array_equal(replies, want)
    offsets, replies = ctx.ht_replies(g, 0, 1, np.zeros(0, np.int32))
    assert offsets.tolist() == [0] and replies.shape == (0, 3)
    offsets, replies = ctx.ht_end_replies(g, np.zeros((0, 2), np.int32))
    assert offsets.tolist() == [0] and replies.shape == (0, 2)


def test_graph_cache_and_validation(ctx):
    g = knn_graph(200, 6, seed=21)
    u, v = next(targets(g, np.random.default_rng(0), 1))
    centers = np.array([c for c in range(20) if c not in (u, v)], np.int32)
    ctx.clear(64)
    ctx.ht_replies(g, u, v, centers)
    assert not ctx.last_reply_stats.graph_hit
    ctx.ht_replies(g, u, v, centers)
    assert ctx.last_reply_stats.graph_hit and ctx.last_reply_stats.workspace_hit
    with pytest.raises(NativeError) as err:  # a center on the target
        ctx.ht_replies(g, u, v, np.array([u], np.int32))
    assert err.value.code == CEE_ERR_INVALID
    row = set(g.neighbors[g.row_offsets[0]:g.row_offsets[1]].tolist())
    missing = (0, next(b for b in range(1, g.n) if b not in row))
    with pytest.raises(NativeError) as err:  # the target is not an edge
        ctx.ht_replies(g, missing[0], missing[1], centers[:1])
    assert err.value.code == CEE_ERR_INVALID
    with pytest.raises(NativeError) as err:  # the task's internal neighbour is not adjacent
        ctx.ht_end_replies(g, np.array([missing], np.int32))
    assert err.value.code == CEE_ERR_INVALID
    g2 = g.copy()
    g2.active[int(np.flatnonzero(g.active)[0])] = 0  # the CSR still holds that edge: not the active edges
    with pytest.raises(NativeError) as err:
        ctx.ht_replies(g2, u, v, centers[:1])
    assert err.value.code == CEE_ERR_INVALID


def test_reference_batches_through_the_dropin(port):
    """EvaluateHtHamiltonReplies / EvaluateHtEndReplies (kCuda) of the reference, linked with this
    project's seam: the reference compares the device lists with its CPU lists and throws on any
    difference; the result must come from the CUDA seam and equal the oracle's."""
    import oracle
    if not oracle.reference_available(dropin=True):
        pytest.skip("oracle/_ref/libcudaee_dropin.so not built")
    ref = oracle.Reference(dropin=True)
    rng = np.random.default_rng(5)
    for g in graphs()[:4]:
        rg = ref.graph(g)
        for u, v in targets(g, rng, 2):
            centers = np.array([c for c in rng.integers(0, g.n, 80) if c not in (u, v)], np.int32)
            for dedup in (True, False):
                offsets, replies, used = rg.ht_hamilton_replies(u, v, centers, backend=2, dedup=dedup)
                assert used == 2
                want_offsets, want = port.ht_replies(g, u, v, centers)
                np.testing.assert_array_equal(offsets, want_offsets)
                np.testing.assert_array_equal(replies, want)
        active = np.flatnonzero(g.active)[:50]
        tasks = np.stack([g.edge_u[active], g.edge_v[active]], axis=1)
        offsets, replies, used = rg.ht_end_replies(tasks, backend=2)
        assert used == 2
        np.testing.assert_array_equal(replies, port.ht_end_replies(g, tasks)[1])


def test_python_seam_mirrors(port):
    import cudaedgeelimination_b200 as cee
    ok, _ = cee.HtHamiltonReplyCudaAvailable()
    assert ok and cee.HtEndReplyCudaAvailable()[0]
    g = knn_graph(250, 8, seed=31)
    u, v = next(targets(g, np.random.default_rng(1), 1))
    centers = np.array([c for c in range(g.n) if c not in (u, v)], np.int32)
    offsets, replies = cee.EvaluateHtHamiltonRepliesCuda(g, (u, v), centers)
    want_offsets, want = port.ht_replies(g, u, v, centers)
    np.testing.assert_array_equal(offsets, want_offsets)
    np.testing.assert_array_equal(replies, want)
    tasks = np.array([[u, v], [v, u]], np.int32)
    np.testing.assert_array_equal(cee.EvaluateHtEndRepliesCuda(g, tasks)[1], port.ht_end_replies(g, tasks)[1])
    cee.ClearHtReplyCudaCache()
