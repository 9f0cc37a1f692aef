"""The reference's own unit tests (tests/unit/test_core.cpp, test_hamilton_tutte.cpp, test_kopt.cpp of
the reference, compiled from its sources by `make -C oracle unit`):

  * on the CPU, built against the reference's CPU library (its CUDA seam = its own stubs): they pass
    as they do in the reference's CPU-only build, which checks the build recipe and the driver;
  * on the GPU (marked gpu), built with CUDAEE_HAS_CUDA against the reference with this project's
    seam dropped in: the reference's own CPU/CUDA parity, cache-contract and proof-byte checks then
    run on the B200 kernels -- JV candidates and their resident cache (test_core.cpp:167-229), the
    k-opt matrix and its cache hits (test_kopt.cpp:158-328), the leaf cursor batcher's proof-byte
    invariance over CUDA cost batches (:608-897), and c,d candidates (test_hamilton_tutte.cpp:404-442).

test_kopt runs through oracle/ref_kopt_unit.cpp, which leaves out the one test that needs the
un-vendored ElimTSP swap oracle; the drop-in test_hamilton_tutte runs through oracle/ref_ht_unit.cpp,
which leaves out TestRecursivePointProof, whose CUDA part drives the HT prover's own CUDA units
(wavefront, path append, replies) -- reference stubs here, outside this project's scope."""
import pathlib
import subprocess

import pytest

UNIT = pathlib.Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "unit"
NAMES = ["test_core", "test_hamilton_tutte", "test_kopt"]
PASSED = {"test_core": "unit tests passed", "test_hamilton_tutte": "Hamilton-Tutte tests passed",
          "test_kopt": "k-opt tests passed"}


def run(variant, name, tmp_path):
    binary = UNIT / variant / name
    if not binary.exists():
        pytest.skip(f"{binary} not built (make -C oracle unit needs the reference sources)")
    env = {"CEE_REF_UNIT_TMP": str(tmp_path), "PATH": "/usr/bin:/bin"}
    proc = subprocess.run([str(binary)], capture_output=True, text=True, timeout=900, env=env, cwd=tmp_path)
    assert proc.returncode == 0, f"{variant}/{name} failed:\n{proc.stdout[-3000:]}\n{proc.stderr[-3000:]}"
    assert PASSED[name] in proc.stdout
    return proc.stdout


@pytest.mark.parametrize("name", NAMES)
def test_reference_unit_cpu(name, tmp_path):
    run("cpu", name, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_reference_unit_dropin(name, tmp_path):
    out = run("dropin", name, tmp_path)
    # the CUDA sections ran on the device (each prints "... skipped: <reason>" when no backend answers)
    assert "CUDA k-opt cost skipped" not in out and "CUDA HT c,d skipped" not in out
