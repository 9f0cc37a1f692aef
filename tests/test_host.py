"""Host-side logic: the snapshot's CSR equals the reference rule, seeded generators are
deterministic, the batch union is consistent with its instances."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth
from helpers import random_graph


@pytest.mark.parametrize("shuffle,active", [(False, 1.0), (True, 1.0), (True, 0.7), (False, 0.5)])
def test_csr_matches_oracle(port, shuffle, active):
    g = random_graph(200, 1500, 5, shuffle=shuffle, active_frac=active)
    ro, nb, ids, ws = port.csr(g.n, g.edge_u, g.edge_v, g.edge_w, g.active)
    np.testing.assert_array_equal(g.row_offsets, ro)
    np.testing.assert_array_equal(g.neighbors, nb)
    np.testing.assert_array_equal(g.csr_edge_ids, ids)
    np.testing.assert_array_equal(g.csr_weights, ws)
    for row in range(g.n):  # rows ascending (the HasActiveEdge binary-search precondition)
        seg = g.neighbors[g.row_offsets[row]:g.row_offsets[row + 1]]
        assert (np.diff(seg) > 0).all()


def test_generators_are_deterministic():
    a, b = synth.jv_clustered(), synth.jv_clustered()
    for name in ("x", "y", "edge_u", "edge_v", "edge_w"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
    g1, t1 = synth.kopt_instance(rows=300, n=500)
    g2, t2 = synth.kopt_instance(rows=300, n=500)
    for k in (3, 4, 5):
        np.testing.assert_array_equal(t1[k].view(np.uint8), t2[k].view(np.uint8))
    assert synth.jv_small().m > 1500


def test_generated_snapshots_are_canonical_knn(port):
    g = synth.jv_small()
    assert (g.edge_u < g.edge_v).all()
    assert (np.lexsort((g.edge_v, g.edge_u)) == np.arange(g.m)).all()
    for e in range(0, g.m, 97):
        assert port.distance(int(g.x[g.edge_u[e]]), int(g.y[g.edge_u[e]]), int(g.x[g.edge_v[e]]),
                             int(g.y[g.edge_v[e]]), g.dist_type) == g.edge_w[e]
    assert len({(int(x), int(y)) for x, y in zip(g.x, g.y)}) == g.n  # de-duplicated points


def test_kopt_rows_follow_the_task_rules():
    g, tasks = synth.kopt_instance(rows=600, n=700)
    for k in (3, 4, 5):
        for row in tasks[k][:100]:
            ports = row["port_nodes"][:2 * k]
            edges = {tuple(sorted((int(ports[2 * e]), int(ports[2 * e + 1])))) for e in range(k)}
            assert len(edges) == k and all(a != b for a, b in edges)  # ValidateKOptCostTask
            assert row["deleted_cost"] == sum(g.distance(int(ports[2 * e]), int(ports[2 * e + 1])) for e in range(k))


def test_batch_union_matches_instances(port):
    b = synth.BatchUnion(24)
    g = b.graph
    h = GraphSnapshot(g.n, g.dist_type, g.x, g.y, g.edge_u, g.edge_v, g.edge_w, g.active)
    np.testing.assert_array_equal(h.row_offsets, g.row_offsets)
    np.testing.assert_array_equal(h.neighbors, g.neighbors)
    np.testing.assert_array_equal(h.csr_edge_ids, g.csr_edge_ids)
    for i in (0, 7, 23):
        inst = b.instance(i)
        ref = synth.batch_instance(i)
        np.testing.assert_array_equal(inst.x, ref.x)
        np.testing.assert_array_equal(inst.edge_v, ref.edge_v)
        # the union screen restricted to an instance is the instance's screen
        w_union = port.jv_screen(h, first=int(b.edge_begin[i]), last=int(b.edge_begin[i + 1]))
        w_inst = port.jv_screen(inst)
        seg = w_union[int(b.edge_begin[i]):int(b.edge_begin[i + 1])]
        np.testing.assert_array_equal(seg, np.where(w_inst >= 0, w_inst + int(b.node_begin[i]), -1))


def test_tuning_cache_roundtrip(tmp_path):
    """Autotuned shapes persist in a JSON file keyed by SM count and power-of-two size buckets."""
    from cudaedgeelimination_b200 import TuningCache
    path = tmp_path / "tuning.json"
    cache = TuningCache(path)
    key = cache.key(148, "batch", largest_instance=5000, instances=4096, edges=30_775_204)
    assert key == "sm148/batch/edges=33554432,instances=4096,largest_instance=8192"
    assert cache.key(148, "batch", largest_instance=4100, instances=4000, edges=17_000_000) == key
    assert cache.key(132, "batch", largest_instance=5000, instances=4096, edges=30_775_204) != key
    assert cache.get(key) is None
    cache.put(key, {"jv_tile": 64, "blocks_per_sm": 8, "chunks": 8})
    again = TuningCache(path)
    assert again.get(key) == {"jv_tile": 64, "blocks_per_sm": 8, "chunks": 8}
    path.write_text('{"version": 0, "entries": {"x": 1}}')  # another format: ignored, not an error
    assert TuningCache(path).get("x") is None


def test_traffic_digest_ignores_comments_only():
    """The digest that ties a recorded ncu traffic figure to its kernel's sources changes with the
    code and not with its comments; string and character literals count as code."""
    import bench
    src = 'int a = 1; // one\n/* block\n comment */ const char* s = "//x"; char c = \'/\';\n'
    assert bench.strip_comments(src) == 'int a = 1;\n const char* s = "//x"; char c = \'/\';'
    assert bench.strip_comments(src.replace("// one", "// other")) == bench.strip_comments(src)
    assert bench.strip_comments(src.replace('"//x"', '"//y"')) != bench.strip_comments(src)
    for kernel in bench.KERNEL_SOURCES:
        assert len(bench.source_digest(kernel)) == 64
