"""HT c,d root screen on the B200 against the CPU oracle: flags identical."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import CD_TASK_DTYPE, GraphSnapshot, synth
from cudaedgeelimination_b200._native import NativeError

pytestmark = pytest.mark.gpu


def tasks_of(c, d, a):
    t = np.zeros(c.shape[0], CD_TASK_DTYPE)
    t["c"], t["d"], t["active"] = c, d, a
    return t


def thirty_two(dist_type):
    # the sparse 32-node construction of the reference's c,d test
    i = np.arange(32)
    xs, ys = (37 * i + 11) % 101, (i * i * 13 + 7 * i) % 97
    edges = [(a, b) for a in range(32) for b in range(a + 1, 32) if (a == 0 and b == 1) or (17 * a + 13 * b) % 5 == 0]
    return GraphSnapshot.from_edges(xs, ys, edges, dist_type)


@pytest.mark.parametrize("dist_type", [0, 1])
@pytest.mark.parametrize("mode", [0, 1])
def test_all_pairs_small(ctx, port, dist_type, mode):
    g = thirty_two(dist_type)
    c, d, a = port.cd_tasks(g, 0, 1, max_neighborhood=0, max_degree=0)
    flags = ctx.cd_screen(g, (0, 1), tasks_of(c, d, a), mode)
    np.testing.assert_array_equal(flags, port.cd_screen(g, 0, 1, c, d, a, mode))


def test_clustered_targets(ctx, port):
    g = synth.jv_clustered()
    for t in port.ht_targets(g)[:64]:
        u, v = int(g.edge_u[t]), int(g.edge_v[t])
        c, d, a = port.cd_tasks(g, u, v)
        assert c.shape[0] == 300
        for mode in (0, 1):
            np.testing.assert_array_equal(ctx.cd_screen(g, (u, v), tasks_of(c, d, a), mode),
                                          port.cd_screen(g, u, v, c, d, a, mode))


def test_inconsistent_active_bit_rejected(ctx, port):
    g = thirty_two(0)
    c, d, a = port.cd_tasks(g, 0, 1, max_neighborhood=0, max_degree=0)
    a = a.copy()
    a[0] ^= 1
    with pytest.raises(NativeError):
        ctx.cd_screen(g, (0, 1), tasks_of(c, d, a), 0)
