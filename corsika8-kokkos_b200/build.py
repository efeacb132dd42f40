"""Builds libc8radio.so in-tree for sm_100a with nvcc.

FP64 device arithmetic is compiled with -fmad=false and host code with
-ffp-contract=off, so every expression that decides a time bin or a branch is
evaluated with the IEEE operations of the reference's x86-64 build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIBRARY = HERE / "libc8radio.so"
SOURCES = ["radio_kernels.cu", "accumulator.cu", "probes.cu", "no_alloc.cu", "server.cu",
           "precision_study.cu", "spool.cu", "snapshot.cu", "tuning.cu"]
HEADERS = ["radio_device.cuh", "radio_kernels.cuh", "host_setup.hpp", "status.hpp"]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
]
OBJECTS = HERE / "_build"


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(found):
        raise RuntimeError("nvcc not found: the radio library needs the CUDA toolkit")
    return found


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = [CSRC / s for s in SOURCES + HEADERS] + [HERE.parent / "include" / "c8radio.h",
                                                       Path(__file__)]
    return any(p.exists() and p.stat().st_mtime > built for p in inputs)


def _compile(source: Path, verbose: bool) -> Path:
    obj = OBJECTS / (source.stem + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, "-c", "-o", str(obj), str(source)]
    if verbose:
        print(" ".join(cmd), flush=True)
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError(f"nvcc failed to compile {source.name}")
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the library if a source is newer than it; returns its path.
    Each source compiles to an object in parallel; one nvcc call links them."""
    if not force and not _stale():
        return LIBRARY
    from concurrent.futures import ThreadPoolExecutor

    OBJECTS.mkdir(exist_ok=True)
    sources = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    with ThreadPoolExecutor(max_workers=min(len(sources), os.cpu_count() or 1)) as pool:
        objects = list(pool.map(lambda src: _compile(src, verbose), sources))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp),
           *map(str, objects)]
    if verbose:
        print(" ".join(cmd), flush=True)
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("nvcc failed to link libc8radio.so")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
