"""Builds the engine's shared library for sm_100a.

`nvcc` compiles the kernels and the C ABI into g4go_b200/_lib/libg4b.so
(CUDA runtime linked statically). The kernels are compiled with -fmad=false
and the host files with -ffp-contract=off: the engine writes every fused
multiply-add it wants as fma, so its results can be compared bit for bit with
the CPU oracle.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
LIB_DIR = PACKAGE / "_lib"
LIBRARY = LIB_DIR / "libg4b.so"
SOURCES = [
    PACKAGE / "csrc" / "transport_kernels.cu",
    PACKAGE / "csrc" / "engine.cpp",
    PACKAGE / "csrc" / "scheduler.cpp",
]
HEADERS = [
    PACKAGE / "csrc" / "g4b_device.cuh",
    PACKAGE / "csrc" / "g4b_dual.cuh",
    PACKAGE / "csrc" / "engine_layout.h",
    PACKAGE / "csrc" / "kernels.h",
    PACKAGE.parent / "include" / "g4b.h",
    PACKAGE.parent / "include" / "g4b_scheduler.h",
]
# The seeded genstep source that stands in for Geant4 in tests and the
# benchmark: host code only, in a library of its own, so that neither the
# engine carries it nor a CPU-only run (the oracle's timing) loads the engine.
SYNTH_LIBRARY = LIB_DIR / "libg4b_synth.so"
SYNTH_SOURCES = [PACKAGE / "csrc" / "synth.cpp"]
SYNTH_HEADERS = [PACKAGE.parent / "include" / "g4b_synth.h", PACKAGE.parent / "include" / "g4b.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    candidate = Path("/usr/local/cuda/bin/nvcc")
    if candidate.exists():
        return str(candidate)
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the engine")


def needs_build(library: Path = LIBRARY, inputs=None) -> bool:
    if not library.exists():
        return True
    built = library.stat().st_mtime
    inputs = SOURCES + HEADERS if inputs is None else inputs
    return any(path.stat().st_mtime > built for path in list(inputs) + [Path(__file__)])


def build_synth(force: bool = False) -> Path:
    """libg4b_synth.so from synth.cpp with the host compiler (no CUDA)."""
    if not force and not needs_build(SYNTH_LIBRARY, SYNTH_SOURCES + SYNTH_HEADERS):
        return SYNTH_LIBRARY
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    temporary = SYNTH_LIBRARY.with_suffix(".so.tmp")
    command = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-shared",
               "-o", str(temporary), *map(str, SYNTH_SOURCES), "-lpthread"]
    subprocess.run(command, check=True, cwd=PACKAGE)
    os.replace(temporary, SYNTH_LIBRARY)
    return SYNTH_LIBRARY


def build(force: bool = False, verbose: bool = False) -> Path:
    build_synth(force=force)
    if not force and not needs_build():
        return LIBRARY
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    temporary = LIBRARY.with_suffix(".so.tmp")
    command = [
        nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-shared", "-o", str(temporary), *map(str, SOURCES), "-lpthread",
    ]
    if verbose:
        command.insert(1, "-Xptxas=-v")
        print(" ".join(command), file=sys.stderr)
    subprocess.run(command, check=True, cwd=PACKAGE)
    os.replace(temporary, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
