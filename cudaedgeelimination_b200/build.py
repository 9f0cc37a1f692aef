"""In-tree build of the native libraries (nvcc for sm_100a, g++ for host-only parts).

    python -m cudaedgeelimination_b200.build          # libcee.so + libcee_synth.so
    python -m cudaedgeelimination_b200.build --all    # + the oracle and the reference drop-in

Outputs stay inside the repository tree (cudaedgeelimination_b200/*.so, oracle/_build,
oracle/_ref) so that they travel with the repository snapshot to the GPU host.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
INCLUDE = ROOT / "include"
ORACLE = ROOT / "oracle"


def reference_dir() -> pathlib.Path | None:
    """The reference source tree: $CEE_REFERENCE_DIR, else the oracle recipe's default location
    (`make -C oracle ref-dir`); None when neither holds the reference sources."""
    env = os.environ.get("CEE_REFERENCE_DIR")
    if env:
        path = pathlib.Path(env)
    else:
        proc = subprocess.run(["make", "-s", "-C", str(ORACLE), "ref-dir"], capture_output=True, text=True)
        if proc.returncode != 0 or not proc.stdout.strip():
            return None
        path = pathlib.Path(proc.stdout.strip())
    return path if (path / "src" / "cpu" / "jv_elimination.cpp").exists() else None

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", f"-I{INCLUDE}", f"-I{CSRC}"]
CUDA_SOURCES = ["cee_api.cu", "batch.cu", "noalloc.cu", "serve.cu", "epoch.cu", "proof.cu", "host_copy.cu", "ht_replies.cu"]


def _host_cxx() -> str:
    for candidate in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(candidate):
            return candidate
    return "g++"


def _nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return found


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(d.stat().st_mtime > mtime for d in deps)


def build_cee(force: bool = False, verbose_ptxas: bool = False) -> pathlib.Path:
    """Compiles every CUDA source for sm_100a and links libcee.so."""
    OBJ.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [INCLUDE / "cee.h"]
    nvcc = _nvcc()
    objects = []
    jobs = []
    for src in CUDA_SOURCES:
        obj = OBJ / (src + ".o")
        objects.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-ccbin", _host_cxx(), "-c", str(CSRC / src), "-o", str(obj)]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as pool:
        for fut in [pool.submit(_run, cmd) for cmd in jobs]:
            fut.result()
    lib = PKG / "libcee.so"
    if force or jobs or _stale(lib, objects):
        _run([nvcc, *ARCH, "-shared", "-ccbin", _host_cxx(), *map(str, objects), "-o", str(lib), "-lcudart"])
    return lib


def build_synth(force: bool = False) -> pathlib.Path:
    lib = PKG / "libcee_synth.so"
    src = CSRC / "synth.cpp"
    if force or _stale(lib, [src]):
        _run([_host_cxx(), "-std=c++20", "-O2", "-fPIC", "-fopenmp", "-shared", str(src), "-o", str(lib)])
    return lib


def build_oracle(force: bool = False) -> None:
    """The plain-C oracle; plus, when the reference tree is present, the reference library
    compiled from its own sources, the reference with this project's shim dropped in, the
    reference with its own CUDA units built for sm_100a (the GPU comparison arm), and the
    reference's own unit tests built against the first two."""
    reference = reference_dir()
    make = ["make", "-C", str(ORACLE)] + ([f"REF={reference}"] if reference is not None else [])
    if force:
        _run(make + ["clean"])
    _run(make + ["port"])
    if reference is not None:
        _run(make + ["-j8", "ref", "dropin", "refcuda"])
        _run(make + ["-j8", "unit"])
    else:
        print("reference sources not found (set CEE_REFERENCE_DIR): the reference library is not rebuilt",
              file=sys.stderr)


def build_all(force: bool = False) -> None:
    build_cee(force)
    build_synth(force)
    build_oracle(force)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--all", action="store_true")
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--ptxas", action="store_true", help="print ptxas register/spill report")
    args = parser.parse_args()
    build_cee(args.force, args.ptxas)
    build_synth(args.force)
    if args.all:
        build_oracle(args.force)
    print("built", file=sys.stderr)


if __name__ == "__main__":
    main()
