"""JV proof log and edge file on the host (cee_content_hash, cee_jv_proof, cee_jv_write_proof,
cee_write_active_edges) against the oracle's and the reference's own ContentHash, WriteProof, ReplayProof
and WriteActiveEdges. No device work: the records are rebuilt
from an elimination's per-edge epochs and witnesses, which these tests take from the reference's CPU run."""
import numpy as np
import pytest

from cudaedgeelimination_b200 import (JV_EPOCH_METRICS_DTYPE, content_hash, jv_proof, synth, write_active_edges,
                                      write_jv_proof)
from cudaedgeelimination_b200._native import CEE_ERR_INVALID, NativeError
from helpers import knn_graph, random_graph


def graphs():
    return {"small": synth.jv_small(), "clustered": synth.jv_clustered(),
            "shuffled": random_graph(400, 2400, seed=11, shuffle=True, active_frac=0.8),
            "ceil": knn_graph(300, 8, seed=3, dist_type=1)}


@pytest.mark.parametrize("name", ["small", "clustered", "shuffled", "ceil"])
def test_content_hash_matches_oracle_and_reference(port, ref, name):
    g = graphs()[name]
    h = content_hash(g)
    assert h == port.content_hash(g)
    assert h == ref.graph(g).content_hash()


def parse_proof(path):
    """(record lines, metrics rows of ints and floats, initial and final hash lines) of a V1 proof."""
    lines = open(path).read().splitlines()
    assert lines[0] == "CUDAEE_PROOF_V1" and lines[-1] == "END"
    records = [ln for ln in lines if ln.startswith("record ")]
    metrics = [ln.split()[1:] for ln in lines if ln.startswith("metrics ")]
    hashes = [ln for ln in lines if ln.startswith(("initial_hash ", "final_hash "))]
    return records, metrics, hashes


def reference_run(ref, g, path):
    """The reference's RunJvElimination(kCpu) proof file for g, and per-edge epoch / witness arrays."""
    epochs = ref.graph(g).write_proof_cpu(path)
    records, _, _ = parse_proof(path)
    edge_epoch = np.full(g.m, -1, np.int32)
    witness = np.full(g.m, -1, np.int32)
    for ln in records:
        f = ln.split()
        edge_epoch[int(f[3])] = int(f[1])
        witness[int(f[3])] = int(f[7])
    return epochs, edge_epoch, witness


@pytest.mark.parametrize("name", ["small", "clustered", "shuffled", "ceil"])
def test_proof_file_matches_reference_and_replays(ref, tmp_path, name):
    g = graphs()[name]
    ref_path, our_path = tmp_path / "reference.proof", tmp_path / "ours.proof"
    epochs, edge_epoch, witness = reference_run(ref, g, ref_path)
    records, hashes = jv_proof(g, epochs, edge_epoch, witness)
    ref_records, ref_metrics, ref_hashes = parse_proof(ref_path)
    metrics = np.zeros(epochs, JV_EPOCH_METRICS_DTYPE)
    for e, row in enumerate(ref_metrics):
        for i, field in enumerate(("epoch", "edges_before", "proposed", "verified", "rejected", "committed")):
            metrics[field][e] = int(row[i])
        metrics["propose_ms"][e], metrics["verify_ms"][e] = float(row[6]), float(row[7])
    write_jv_proof(our_path, "cpu", records, hashes, metrics)
    ours, our_metrics, our_hashes = parse_proof(our_path)
    assert ours == ref_records  # every record line byte for byte: epoch, snapshot hash, edge, u, v, JV, witness
    assert our_hashes == ref_hashes
    assert [row[:6] for row in our_metrics] == [row[:6] for row in ref_metrics]
    assert open(our_path).read() == open(ref_path).read()  # same metrics times given: the whole file
    assert ref.graph(g).replay_proof_file(our_path) == len(records)


def test_tampered_proof_is_rejected_by_the_reference(ref, tmp_path):
    g = synth.jv_clustered()
    epochs, edge_epoch, witness = reference_run(ref, g, tmp_path / "reference.proof")
    records, hashes = jv_proof(g, epochs, edge_epoch, witness)
    metrics = np.zeros(epochs, JV_EPOCH_METRICS_DTYPE)
    bad = records.copy()
    bad["snapshot_hash"][0] ^= 1
    write_jv_proof(tmp_path / "bad.proof", "cpu", bad, hashes, metrics)
    with pytest.raises(RuntimeError):
        ref.graph(g).replay_proof_file(tmp_path / "bad.proof")


def test_hashes_follow_the_epochs(port):
    # hashes[k] is the content hash with every edge eliminated before epoch k inactive
    g = synth.jv_clustered()
    rng = np.random.default_rng(5)
    edge_epoch = np.where(rng.random(g.m) < 0.3, rng.integers(0, 3, g.m), -1).astype(np.int32)
    witness = np.where(edge_epoch >= 0, 0, -1).astype(np.int32)
    records, hashes = jv_proof(g, 3, edge_epoch, witness)
    for k in range(4):
        h = g.copy()
        h.active = ((g.active != 0) & ~((edge_epoch >= 0) & (edge_epoch < k))).astype(np.uint8)
        assert int(hashes[k]) == port.content_hash(h)
    assert (np.diff(records["epoch"].astype(np.int64)) >= 0).all()
    for r in records:
        assert int(r["snapshot_hash"]) == int(hashes[r["epoch"]])


def test_bad_inputs(tmp_path):
    g = synth.jv_small()
    edge_epoch = np.full(g.m, -1, np.int32)
    witness = np.full(g.m, -1, np.int32)
    edge_epoch[0], witness[0] = 2, 1
    with pytest.raises(NativeError) as err:  # epoch beyond the run
        jv_proof(g, 2, edge_epoch, witness)
    assert err.value.code == CEE_ERR_INVALID
    edge_epoch[0], witness[0] = 0, g.n  # witness not a node
    with pytest.raises(NativeError):
        jv_proof(g, 1, edge_epoch, witness)
    records, hashes = jv_proof(g, 1, np.full(g.m, -1, np.int32), witness)
    assert records.shape == (0,) and hashes.shape == (2,) and hashes[0] == hashes[1] == content_hash(g)
    with pytest.raises(NativeError):  # the backend must be one token
        write_jv_proof(tmp_path / "p", "two words", records, hashes, np.zeros(1, JV_EPOCH_METRICS_DTYPE))


@pytest.mark.parametrize("name", ["small", "shuffled", "ceil"])
def test_active_edge_file_matches_reference(ref, tmp_path, name):
    g = graphs()[name]
    write_active_edges(tmp_path / "ours.edg", g)
    rg = ref.graph(g)
    rg.write_active_edges(tmp_path / "reference.edg")
    assert open(tmp_path / "ours.edg").read() == open(tmp_path / "reference.edg").read()
    # with other flags: the final flags of the reference's own elimination
    rg.write_proof_cpu(tmp_path / "run.proof")
    rg.write_active_edges(tmp_path / "reference_final.edg")
    write_active_edges(tmp_path / "ours_final.edg", g, rg.active())
    assert open(tmp_path / "ours_final.edg").read() == open(tmp_path / "reference_final.edg").read()
