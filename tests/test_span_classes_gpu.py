"""The three exact-distance routines (span classes small < 2^21 <= narrow < 2^26 <= wide < 2^30)
against the oracle's integer-square-root distance (src/common/distance.cpp:9-52): directly, on
pairs chosen at the rounding and fix-up boundaries up to each class's largest squared distance,
and through the JV, k-opt and c,d screens on instances of each class."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import KOPT_TASK_DTYPE, BuildKOptReconnectTable, CD_TASK_DTYPE
from helpers import knn_graph

pytestmark = pytest.mark.gpu

SMALL, NARROW, WIDE = 0, 1, 2


def boundary_pairs(span, count, seed):
    """Point pairs inside [0, span]^2 whose squared distance s sits next to the decision points of
    the integer root: q^2 (perfect squares), q^2 + q and q^2 + q + 1 (EUC_2D rounding), just
    below (q + 1)^2 (a root estimate that lands one high), plus uniformly random pairs. The two
    corners (0, 0) and (span, span) pin the bounding box and hence the span class."""
    rng = np.random.default_rng(seed)
    xs, ys = [0, span], [0, span]
    q = np.concatenate([rng.integers(1, span + 1, count // 2),
                        np.maximum(1, span - rng.integers(0, 4096, count // 2))])
    rq = np.floor(np.sqrt(q.astype(np.float64))).astype(np.int64)
    r2q = np.floor(np.sqrt(2.0 * q.astype(np.float64))).astype(np.int64)
    kind = rng.integers(0, 6, q.shape[0])
    # dy with s = q^2 + dy^2: 0 (square), ~sqrt(q) (EUC boundary), ~sqrt(2q) (just below (q+1)^2)
    dy = np.choose(kind, [np.zeros_like(q), rq, rq + 1, r2q, np.maximum(r2q - 1, 0),
                          rng.integers(0, span + 1, q.shape[0])])
    dy = np.minimum(dy, span)
    x0 = rng.integers(0, span - q + 1)
    y0 = rng.integers(0, span - dy + 1)
    flip = rng.integers(0, 2, q.shape[0]).astype(bool)  # swap the axes on half of the pairs
    ax, ay = np.where(flip, y0, x0), np.where(flip, x0, y0)
    bx, by = np.where(flip, y0 + dy, x0 + q), np.where(flip, x0 + q, y0 + dy)
    rand = rng.integers(0, span + 1, (count, 4))
    xs = np.concatenate([xs, ax, rand[:, 0], bx, rand[:, 2]])
    ys = np.concatenate([ys, ay, rand[:, 1], by, rand[:, 3]])
    half = q.shape[0] + count
    pi = 2 + np.arange(half)
    pj = 2 + half + np.arange(half)
    swap = rng.integers(0, 2, half).astype(bool)  # both point orders (negative dx, dy)
    return xs, ys, np.where(swap, pj, pi), np.where(swap, pi, pj)


@pytest.mark.parametrize("span,cls", [((1 << 21) - 1, SMALL), (1 << 21, NARROW), ((1 << 26) - 1, NARROW),
                                      (1 << 26, WIDE), ((1 << 30) - 1, WIDE), (1000, SMALL)])
@pytest.mark.parametrize("dist_type", [0, 1])
def test_exact_distances_at_boundaries(ctx, port, span, cls, dist_type):
    xs, ys, pi, pj = boundary_pairs(span, 100_000, seed=span % 9973 + dist_type)
    offset = -(1 << 40)  # absolute coordinates far from the origin: only offsets reach the device
    gpu, got = ctx.exact_distances(xs + offset, ys - offset, dist_type, pi, pj)
    assert got == cls
    np.testing.assert_array_equal(gpu.astype(np.int64), port.distance_pairs(xs, ys, dist_type, pi, pj))


def test_sqrt_estimate_error_bound(ctx):
    # the small class rounds an FP32 root estimate and corrects it by one step with an exact
    # residual: exact while the estimate's relative error stays below 2^-21.6 on every float the
    # class can produce; the B200 measures 2^-23.25
    err = ctx.sqrt_estimate_error()
    assert 0.0 < err <= 2.0 ** -22, err


def test_small_span_all_short_vectors(ctx, port):
    # every (dx, dy) with 0 <= dx, dy < 512 from one point, both distance types
    d = np.arange(512)
    dx, dy = np.meshgrid(d, d)
    xs = np.concatenate([[0], dx.ravel()])
    ys = np.concatenate([[0], dy.ravel()])
    pj = np.arange(1, xs.shape[0], dtype=np.int32)
    pi = np.zeros_like(pj)
    for t in (0, 1):
        gpu, cls = ctx.exact_distances(xs, ys, t, pi, pj)
        assert cls == SMALL
        np.testing.assert_array_equal(gpu.astype(np.int64), port.distance_pairs(xs, ys, t, pi, pj))


def random_kopt_rows(g, k, rows, seed):
    rng = np.random.default_rng(seed)
    tasks = np.zeros(rows, KOPT_TASK_DTYPE)
    for r in range(rows):
        ports = rng.choice(g.n, 2 * k, replace=False)
        tasks[r]["port_nodes"][:2 * k] = ports
        tasks[r]["deleted_cost"] = sum(g.distance(int(ports[2 * e]), int(ports[2 * e + 1])) for e in range(k))
    return tasks


@pytest.mark.parametrize("coord,cls", [(1 << 21, SMALL), (1 << 24, NARROW), (1 << 28, WIDE)])
@pytest.mark.parametrize("dist_type", [0, 1])
def test_screens_per_class(ctx, port, coord, cls, dist_type):
    g = knn_graph(400, 8, seed=coord % 977 + dist_type, coord=coord, dist_type=dist_type)
    _, got = ctx.exact_distances(g.x, g.y, dist_type, [0], [1])
    assert got == cls
    # JV screen (warp per edge)
    witness, _ = ctx.jv_screen(g)
    np.testing.assert_array_equal(witness, port.jv_screen(g))
    # k-opt leaf costs
    for k in (3, 4, 5):
        tasks = random_kopt_rows(g, k, 300, seed=k)
        gpu, _ = ctx.kopt_costs(g, BuildKOptReconnectTable(k), tasks)
        np.testing.assert_array_equal(gpu, port.kopt_costs(g, k, tasks))
    # c,d root screens of the first HT targets
    for t in port.ht_targets(g)[:8]:
        u, v = int(g.edge_u[t]), int(g.edge_v[t])
        c, d, a = port.cd_tasks(g, u, v)
        tasks = np.zeros(c.shape[0], CD_TASK_DTYPE)
        tasks["c"], tasks["d"], tasks["active"] = c, d, a
        for mode in (0, 1):
            np.testing.assert_array_equal(ctx.cd_screen(g, (u, v), tasks, mode), port.cd_screen(g, u, v, c, d, a, mode))
    # device-resident elimination to a fixed point
    active, _, _, before, committed, _ = ctx.jv_eliminate(g)
    o_active, o_before, o_committed, _ = port.jv_eliminate(g)
    np.testing.assert_array_equal(active, o_active)
    np.testing.assert_array_equal(committed, o_committed)
