"""Device-resident JV elimination to a fixed point (cee_jv_eliminate) against the CPU oracle's
epoch loop and, when the reference library is built, the reference's own RunJvElimination(kCpu):
final active sets, per-epoch edges and commits, and every (epoch, edge, witness) record identical."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import GraphSnapshot, synth, write_active_edges
from cudaedgeelimination_b200._native import CEE_ERR_INVALID, NativeError
from helpers import knn_graph, random_graph

pytestmark = pytest.mark.gpu


def records_of(witness, epoch):
    """(epoch, edge, witness) records in the reference's proof order: by epoch, then (u, v), i.e.
    ascending edge id for canonically sorted edge lists."""
    ids = np.flatnonzero(epoch >= 0)
    return sorted((int(epoch[e]), int(e), int(witness[e])) for e in ids)


def check(ctx, port, g, max_rounds=100):
    active, witness, epoch, before, committed, stats = ctx.jv_eliminate(g, max_rounds)
    o_active, o_before, o_committed, _ = port.jv_eliminate(g, max_rounds)
    np.testing.assert_array_equal(active, o_active)
    np.testing.assert_array_equal(before, o_before)
    np.testing.assert_array_equal(committed, o_committed)
    assert stats.epochs == len(o_before) and stats.committed == int(o_committed.sum())
    eliminated = (g.active != 0) & (active == 0)
    assert ((epoch >= 0) == eliminated).all() and ((witness >= 0) == eliminated).all()
    for e in np.flatnonzero(eliminated)[:64]:  # every witness is a JV witness in its epoch's snapshot
        assert witness[e] != g.edge_u[e] and witness[e] != g.edge_v[e]
    return active, witness, epoch, before, committed


def test_small_uniform(ctx, port):
    check(ctx, port, synth.jv_small())


def test_clustered_multi_epoch(ctx, port):
    _, _, _, before, _ = check(ctx, port, synth.jv_clustered())
    assert len(before) >= 2


@pytest.mark.parametrize("seed", range(4))
def test_random_knn(ctx, port, seed):
    check(ctx, port, knn_graph(500, 6 + 2 * seed, seed, dist_type=seed % 2))


def test_unsorted_and_inactive(ctx, port):
    check(ctx, port, random_graph(400, 2400, seed=11, shuffle=True, active_frac=0.8))


def test_wide_coordinates(ctx, port):
    check(ctx, port, knn_graph(300, 8, seed=12, coord=1 << 28))


def test_max_rounds_stops_early(ctx, port):
    g = synth.jv_clustered()
    _, _, epoch, before, _ = check(ctx, port, g, max_rounds=1)
    assert len(before) == 1 and epoch.max() == 0


def test_batch_instance_large(ctx, port):
    check(ctx, port, synth.batch_instance(3, n_lo=4000, n_hi=5000))


def test_matches_reference_records(ctx, ref):
    g = synth.jv_clustered()
    active, witness, epoch, before, committed, _ = ctx.jv_eliminate(g)
    rg = ref.graph(g)
    stats, records, _, _ = rg.run_jv(1)  # columns: edges before, proposed, committed
    np.testing.assert_array_equal(before, stats[:, 0])
    np.testing.assert_array_equal(committed, stats[:, 2])
    assert records_of(witness, epoch) == sorted(tuple(int(v) for v in r) for r in records)
    np.testing.assert_array_equal(active, rg.active())


def test_no_edges_and_errors(ctx):
    empty = random_graph(10, 0, seed=5)
    active, witness, epoch, before, committed, stats = ctx.jv_eliminate(empty)
    assert active.shape == (0,) and stats.epochs == 1 and committed.tolist() == [0]
    g = synth.jv_small()
    dup = GraphSnapshot.from_edges(g.x, g.y, np.concatenate([np.stack([g.edge_u, g.edge_v], 1)[:5]] * 2), 0)
    with pytest.raises(NativeError) as e:
        ctx.jv_eliminate(dup)
    assert e.value.code == CEE_ERR_INVALID
    with pytest.raises(NativeError):
        ctx.jv_eliminate(g, 0)


@pytest.mark.parametrize("which", ["clustered", "batch3"])
def test_device_proof_replays_in_the_reference(ctx, ref, tmp_path, which):
    """The proof file of a device elimination (records with every epoch's snapshot hash) is accepted
    by the reference's ReadProof + ReplayProof, and its records, hashes and per-epoch counts equal
    the reference's own RunJvElimination(kCpu) proof."""
    g = synth.jv_clustered() if which == "clustered" else synth.batch_instance(3, n_lo=4000, n_hi=5000)
    path, ref_path = tmp_path / "device.proof", tmp_path / "reference.proof"
    _, _, _, _, committed, _, records = ctx.jv_eliminate_with_proof(g, path)
    assert ref.graph(g).replay_proof_file(path) == len(records) == int(committed.sum())
    ref.graph(g).write_proof_cpu(ref_path)

    def fields(p):
        lines = open(p).read().splitlines()
        kept = [ln for ln in lines if ln.startswith(("record ", "initial_hash ", "final_hash "))]
        counts = [ln.split()[1:7] for ln in lines if ln.startswith("metrics ")]  # epoch .. committed
        return kept, counts

    assert fields(path) == fields(ref_path)


def test_device_final_edge_file_matches_reference(ctx, ref, tmp_path):
    """The .edg file of the device elimination's final active edges equals the one the reference writes
    after its own RunJvElimination(kCpu)."""
    g = synth.jv_clustered()
    active, *_ = ctx.jv_eliminate(g)
    write_active_edges(tmp_path / "device.edg", g, active)
    rg = ref.graph(g)
    rg.write_proof_cpu(tmp_path / "reference.proof")
    rg.write_active_edges(tmp_path / "reference.edg")
    assert open(tmp_path / "device.edg").read() == open(tmp_path / "reference.edg").read()
