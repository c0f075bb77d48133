"""Build the native library in-tree: ``paracfd_b200/libparacfd_b200.so`` (sm_100a only).

Usage: ``python -m paracfd_b200.build`` or ``paracfd_b200.build.build()``.  Objects go to
``paracfd_b200/_build/`` and are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
TARGET = os.path.join(HERE, "libparacfd_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"),
]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    host_sources = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.h"))) + [os.path.join(ROOT, "include", "paracfd_b200.h")]
    flags = NVCC_FLAGS + (extra_flags or [])
    jobs = []
    objects = []
    for src in sources:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objects.append(obj)
        if _newer(obj, [src] + headers):
            jobs.append([NVCC] + flags + ["-c", src, "-o", obj])
    for src in host_sources:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objects.append(obj)
        if _newer(obj, [src] + headers):
            jobs.append([os.environ.get("CXX", "g++"), "-std=c++17", "-O3", "-fPIC", "-I" + os.path.join(ROOT, "include"),
                         "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as pool:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        list(pool.map(_run, jobs))
    if jobs or _newer(TARGET, objects):
        _run([NVCC, "-shared", "-o", TARGET] + objects + ["-lcudart"])
    return TARGET


if __name__ == "__main__":
    print(build(verbose=True))
