"""Build step of the engine: compiles csrc/ into the in-tree libtbgpu.so.

    python -m tb8gen_b200.build

nvcc targets sm_100a only (-gencode arch=compute_100a,code=sm_100a); the
shared library lands next to this file so that it travels with the
repository to the GPU host and is the one Python loads.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtbgpu.so")
SOURCES = ["tbg_api.cu", "tbg_noalloc.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-diag-suppress", "550",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def newest_input_mtime() -> float:
    t = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


HOST_SRC = os.path.join(HERE, "host", "tbgen.c")
HOST_OUT = os.path.join(HERE, "tbgen")


def build_host(force: bool = False) -> str:
    """The C host driver (host/tbgen.c), linked against libtbgpu.so."""
    if not force and os.path.exists(HOST_OUT) and \
            os.path.getmtime(HOST_OUT) >= max(os.path.getmtime(HOST_SRC), os.path.getmtime(OUT)):
        return HOST_OUT
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-o", HOST_OUT, HOST_SRC, "-L" + HERE, "-ltbgpu",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("gcc failed building tbgen")
    return HOST_OUT


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest_input_mtime():
        build_host()
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libtbgpu.so")
    if verbose:
        sys.stderr.write(r.stderr)
    build_host(force=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
