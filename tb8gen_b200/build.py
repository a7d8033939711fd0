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
SOURCES = ["tbg_api.cu", "tbg_persist_block.cu", "tbg_persist_warp.cu", "tbg_noalloc.cu",
           "tbg_probe_api.cu", "tbg_table.cpp", "tbg_subtable.cu"]
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
           "-ldl", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("gcc failed building tbgen")
    return HOST_OUT


OBJ_DIR = os.path.join(HERE, "_build")
COMPILE_FLAGS = [f for f in NVCC_FLAGS if f != "-shared"]


def _obj_current(obj: str) -> bool:
    """True when obj exists and is newer than every input its .d file lists."""
    dep = obj + ".d"
    if not (os.path.exists(obj) and os.path.exists(dep)):
        return False
    t = os.path.getmtime(obj)
    with open(dep) as f:
        text = f.read().replace("\\\n", " ")
    inputs = text.split(":", 1)[1].split() if ":" in text else []
    return all(os.path.exists(i) and os.path.getmtime(i) <= t for i in inputs)


def _compile(src: str, verbose: bool, force: bool):
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    if not force and _obj_current(obj):
        return obj, None
    cmd = [nvcc(), *COMPILE_FLAGS, "-MD", "-MF", obj + ".d", "-c", "-o", obj,
           os.path.join(CSRC, src)]
    if verbose and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    return obj, subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source of csrc/ to an object (in parallel, each only
    when a file it includes is newer) and links libtbgpu.so."""
    objs = [os.path.join(OBJ_DIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    if not force and not all(os.path.exists(o) for o in objs) and os.path.exists(OUT) and \
            os.path.getmtime(OUT) >= newest_input_mtime():
        build_host()  # a library built elsewhere, shipped without its objects
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, force), SOURCES))
    compiled = False
    for (obj, r), src in zip(results, SOURCES):
        if r is None:
            continue
        compiled = True
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed compiling {src}")
        if verbose:
            sys.stderr.write(r.stderr)
    if not compiled and os.path.exists(OUT) and \
            os.path.getmtime(OUT) >= max(os.path.getmtime(o) for o in objs):
        build_host()
        return OUT
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT,
           *[obj for obj, _ in results]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libtbgpu.so")
    build_host(force=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
