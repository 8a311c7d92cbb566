"""Build recipes for the native parts of axon_b200 (in-tree, no JIT cache).

- ``libaxon_b200.so``: the CUDA engine (sm_100a) behind include/axon_capi.h.
- ``axon``: the C++ command-line drop-in for the reference's ``build/axon``.
- ``oracle/_build``: the CPU oracle used by the tests (built with its own Makefile).

Everything is compiled with nvcc/g++ directly; outputs go to ``axon_b200/_build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = OUT / "libaxon_b200.so"
CLI = OUT / "axon"
ORACLE_DIR = ROOT / "oracle"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
LIB_SOURCES = ["plain.cu", "batch.cu", "multi.cu", "serve.cu", "serve_batched.cu", "engine.cu", "recall.cu", "multi_host.cu", "serve_host.cu",
               "capi.cu", "static_present.cu", "checkpoint.cu"]
CLI_SOURCES = ["cli_main.cpp", "protocol.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str], cwd: Path | None = None) -> None:
    proc = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_lib(force: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in LIB_SOURCES if (CSRC / s).exists()]
    deps = srcs + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "axon_capi.h"]
    if force or _stale(LIB, deps):
        _run([_nvcc(), *ARCH, *NVCC_FLAGS, "-shared", "-o", str(LIB), *map(str, srcs)])
    return LIB


def build_cli(force: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in CLI_SOURCES if (CSRC / s).exists()]
    if not srcs:
        return CLI
    deps = srcs + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "axon_capi.h", LIB]
    if force or _stale(CLI, deps):
        cxx = os.environ.get("CXX", "g++")
        _run([cxx, "-O2", "-std=c++17", "-Wall", "-pthread", "-I", str(ROOT / "include"), "-o", str(CLI),
              *map(str, srcs), "-L", str(OUT), "-laxon_b200", f"-Wl,-rpath,$ORIGIN"])
    return CLI


def build_oracle() -> None:
    """Compile the CPU oracle (test infrastructure) with its Makefile."""
    _run(["make", "-s", "-C", str(ORACLE_DIR)])


def build_all(force: bool = False) -> None:
    build_lib(force)
    build_cli(force)
    build_oracle()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(f"built {LIB} and {CLI}")
