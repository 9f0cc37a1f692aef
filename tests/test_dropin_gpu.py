"""The reference's own CPU code driving the B200 kernels through the C++ shim
(oracle/_ref/libcudaee_dropin.so = the reference sources + cudaedgeelimination_b200/shim).

The reference's callers certify our results in situ: RunJvElimination re-verifies every CUDA
candidate and throws on a rejection (src/cpu/jv_elimination.cpp:296-303), EvaluateKOptTemplateCosts
compares every cell with its CPU matrix (src/cpu/kopt_search.cpp:1462-1473), and
EvaluateHtCdCandidates compares GPU and CPU flags (src/cpu/hamilton_tutte.cpp:691-695)."""
import numpy as np
import pytest

import oracle
from cudaedgeelimination_b200 import synth
from helpers import knn_graph, random_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin():
    if not oracle.reference_available(dropin=True):
        pytest.skip("oracle/_ref/libcudaee_dropin.so not built (needs the reference sources)")
    return oracle.Reference(dropin=True)


@pytest.mark.parametrize("make", [synth.jv_small, synth.jv_clustered,
                                  lambda: random_graph(300, 2500, 7, shuffle=True, active_frac=0.8),
                                  lambda: knn_graph(500, 9, 3, dist_type=1)])
def test_run_jv_elimination_cuda_equals_cpu(dropin, make):
    g = make()
    cpu = dropin.graph(g).run_jv(1)
    gpu = dropin.graph(g).run_jv(2)
    np.testing.assert_array_equal(cpu[0], gpu[0])  # per-epoch edges_before / proposed / committed
    np.testing.assert_array_equal(cpu[1], gpu[1])  # proof records (epoch, edge, witness)
    assert cpu[2] == gpu[2] and cpu[3] == gpu[3]   # initial and final content hash


def test_jv_cache_usage_contract(dropin):
    """Hit/miss semantics of the reference's tests/unit/test_core.cpp:167-229."""
    g = synth.jv_small()
    rg = dropin.graph(g)
    dropin.L.ref_jv_clear_cuda_cache()
    w1, u1, r1 = rg.jv_cuda()
    np.testing.assert_array_equal(w1, rg.jv_cpu())
    assert u1[0] == 0 and u1[1] == 0 and u1[2] >= 0 and r1 > 0
    w2, u2, r2 = rg.jv_cuda()
    np.testing.assert_array_equal(w1, w2)
    assert u2[0] == 1 and u2[1] == 1 and r2 == r1
    active = rg.active()
    active[0] = 0
    rg.set_active(active)
    w3, u3, _ = rg.jv_cuda()
    np.testing.assert_array_equal(w3, rg.jv_cpu())
    assert u3[0] == 1 and u3[1] == 1
    dropin.L.ref_jv_clear_cuda_cache()


@pytest.mark.parametrize("k", [3, 4, 5])
def test_kopt_costs_certified_by_reference(dropin, k):
    g, tasks = synth.kopt_instance(rows=3000, n=2000)
    rg = dropin.graph(g)
    cpu, _ = rg.kopt_costs(k, tasks[k], backend=1)
    gpu, meta = rg.kopt_costs(k, tasks[k], backend=2)  # throws unless every cell matches
    np.testing.assert_array_equal(cpu, gpu)
    assert meta[1] >= 0


@pytest.mark.parametrize("mode", [0, 1])
def test_cd_candidates_certified_by_reference(dropin, port, mode):
    g = synth.jv_clustered()
    rg = dropin.graph(g)
    for t in port.ht_targets(g)[:16]:
        u, v = int(g.edge_u[t]), int(g.edge_v[t])
        cpu = rg.cd_candidates(u, v, mode=mode, backend=1)
        gpu = rg.cd_candidates(u, v, mode=mode, backend=2)  # throws unless the flags match
        np.testing.assert_array_equal(cpu, gpu)
