"""JV screen on the B200 against the CPU oracle: witness arrays must be identical (bit-exact
integer work), epoch after epoch, including the reference's edge cases."""
import ctypes

import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth
from cudaedgeelimination_b200 import _native
from cudaedgeelimination_b200._native import NativeError, CEE_ERR_RANGE
from helpers import commit, complete_graph, knn_graph, random_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[0, 1], ids=["thread", "warp"])
def jv(ctx, request):
    """The context with the JV screen mapped one thread per edge, then one warp per edge."""
    ctx.set_option(_native.OPT_JV_KERNEL, request.param)
    yield ctx
    ctx.set_option(_native.OPT_JV_KERNEL, 1)


def check_epochs(ctx, port, g, max_rounds=100):
    """Runs the fixed-point loop with the GPU screen, comparing every epoch to the oracle."""
    epochs = 0
    for _ in range(max_rounds):
        gpu, stats = ctx.jv_screen(g)
        cpu = port.jv_screen(g)
        np.testing.assert_array_equal(gpu, cpu)
        assert stats.edges_screened == int(g.active.sum())
        for e in np.flatnonzero(gpu >= 0)[:50]:
            assert port.jv_verify(g, int(e), int(gpu[e]))
        epochs += 1
        g, committed = commit(port, g, gpu)
        if committed == 0:
            break
    return g, epochs


def test_small_uniform_fixed_point(jv, port):
    g = synth.jv_small()
    final, epochs = check_epochs(jv, port, g)
    active, before, committed, final_hash = port.jv_eliminate(g)
    np.testing.assert_array_equal(final.active, active)
    assert epochs == len(before)


def test_clustered_multi_epoch(jv, port):
    g = synth.jv_clustered()
    final, epochs = check_epochs(jv, port, g)
    assert epochs >= 2
    assert port.content_hash(final) == port.jv_eliminate(g)[3]


@pytest.mark.parametrize("seed", range(4))
def test_random_knn(jv, port, seed):
    check_epochs(jv, port, knn_graph(400, 6 + 2 * seed, seed, dist_type=seed % 2))


@pytest.mark.parametrize("seed", range(3))
def test_dense_rows_multi_pass(jv, port, seed):
    # degrees well above 32: several scoring passes and long witness scans
    g = random_graph(90, 1800, 100 + seed)
    assert g.degree().max() > 32
    check_epochs(jv, port, g, max_rounds=3)


def test_unsorted_edges_and_inactive(jv, port):
    g = random_graph(300, 2500, 7, shuffle=True, active_frac=0.8)
    check_epochs(jv, port, g, max_rounds=3)


def test_k4_and_complete_graphs(jv, port):
    k4 = complete_graph([0, 10, 0, 10], [0, 0, 10, 10])
    gpu, _ = jv.jv_screen(k4)
    np.testing.assert_array_equal(gpu, port.jv_screen(k4))
    rng = np.random.default_rng(3)
    for n in (5, 9, 12):
        g = complete_graph(rng.permutation(1000)[:n], rng.permutation(1000)[:n], dist_type=n % 2)
        check_epochs(jv, port, g)


def test_low_degree_gate_and_empty(jv, port):
    # a path: every degree <= 2, so no edge is screened
    g = GraphSnapshot.from_edges([0, 5, 9, 20], [0, 3, 1, 4], [(0, 1), (1, 2), (2, 3)])
    gpu, _ = jv.jv_screen(g)
    assert (gpu == -1).all()
    empty = GraphSnapshot.from_edges([0, 1, 2], [0, 1, 2], np.zeros((0, 2), np.int64))
    gpu, _ = jv.jv_screen(empty)
    assert gpu.shape == (0,)


def test_large_coordinates_exact(jv, port):
    # spans close to 2^30: squared distances near 2^61 exercise the FP64 root + integer fix-up
    rng = np.random.default_rng(11)
    span = (1 << 30) - 1
    xs = rng.integers(0, span, 64)
    ys = rng.integers(0, span, 64)
    xs[0], ys[0], xs[1], ys[1] = 0, 0, span, span
    for t in (0, 1):
        g = GraphSnapshot.from_edges(xs + (1 << 40), ys - (1 << 35),
                                     [(i, j) for i in range(64) for j in range(i + 1, 64) if (i * 7 + j) % 5 < 2],
                                     dist_type=t)
        gpu, _ = jv.jv_screen(g)
        np.testing.assert_array_equal(gpu, port.jv_screen(g))


def test_range_error(ctx):
    g = GraphSnapshot.from_edges([0, 1 << 31, 5, 7], [0, 0, 9, 2], [(0, 1), (1, 2), (2, 3), (0, 3), (0, 2)])
    with pytest.raises(NativeError) as err:
        ctx.jv_screen(g)
    assert err.value.code == CEE_ERR_RANGE


def test_cache_contract(ctx, port):
    """JV resident-cache hit/miss semantics (the reference pins them in tests/unit/test_core.cpp:167-229)."""
    ctx.clear(1)
    g = synth.jv_small()
    first, s1 = ctx.jv_screen(g)
    assert not s1.static_hit and not s1.workspace_hit and s1.resident_bytes > 0
    second, s2 = ctx.jv_screen(g)
    np.testing.assert_array_equal(first, second)
    assert s2.static_hit and s2.workspace_hit and s2.resident_bytes == s1.resident_bytes
    g2 = g.copy()
    g2.active[0] = 0
    g2.rebuild_csr()
    w, s3 = ctx.jv_screen(g2)
    np.testing.assert_array_equal(w, port.jv_screen(g2))
    assert s3.static_hit and s3.workspace_hit
    g3 = g.copy()
    g3.x[0] += 1000
    g3.edge_w = np.array([g3.distance(int(a), int(b)) for a, b in zip(g3.edge_u, g3.edge_v)], np.int64)
    g3.rebuild_csr()
    w, s4 = ctx.jv_screen(g3)
    np.testing.assert_array_equal(w, port.jv_screen(g3))
    assert not s4.static_hit and s4.workspace_hit
    for s in (s1, s2, s3, s4):
        assert np.isfinite(s.h2d_ms) and s.h2d_ms >= 0 and s.kernel_ms >= 0 and s.d2h_ms >= 0


def test_static_unchanged_hint(ctx, port):
    """cee_jv_screen_ex's CEE_JV_STATIC_UNCHANGED: with the cached static data the witnesses equal the
    oracle's and the cache is hit without comparing; a snapshot of other sizes, or a cleared cache,
    makes the hint do nothing; unknown flag bits fail."""
    ctx.clear(1)
    g = synth.jv_small()
    first, s1 = ctx.jv_screen(g, static_unchanged=True)  # nothing cached yet: a full upload
    assert not s1.static_hit
    np.testing.assert_array_equal(first, port.jv_screen(g))
    g2 = g.copy()
    g2.active[: g2.m // 3] = 0
    g2.rebuild_csr()
    w, s2 = ctx.jv_screen(g2, static_unchanged=True)  # same static arrays, fewer active edges
    assert s2.static_hit
    np.testing.assert_array_equal(w, port.jv_screen(g2))
    other = synth.jv_clustered()
    w, s3 = ctx.jv_screen(other, static_unchanged=True)  # other sizes: the hint is not taken
    assert not s3.static_hit
    np.testing.assert_array_equal(w, port.jv_screen(other))
    ctx.clear(1)
    w, s4 = ctx.jv_screen(other, static_unchanged=True)
    assert not s4.static_hit
    np.testing.assert_array_equal(w, port.jv_screen(other))
    out = np.empty(other.m, np.int32)
    view = other.view()
    rc = _native.lib().cee_jv_screen_ex(ctx.handle, ctypes.byref(view), out.ctypes.data_as(_native.c_i32p), None, 2)
    assert rc == _native.CEE_ERR_INVALID
