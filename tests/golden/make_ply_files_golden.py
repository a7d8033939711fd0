"""Digests of the reference program's per-ply files (tests/golden/ply_files.json).

The unmodified reference program, built in place under oracle/_ref
(oracle/Makefile: tb8gen, and tb8gen_stub with the 7-piece probe replaced by
the seeded stub, seed and modulus from the environment), runs a material
in a temporary directory and writes its per-ply files: write_data's zstd
frames (util.c:272-343) under <material>/<n>/<W|L>/<w|b>/<wk><bk>
(kslice.c:306-315), the mates under 0/L and the final "wins" under 0/wins.
Each half-ply directory is recorded as the SHA-256 of its 462 decompressed
slice bitmaps concatenated in file-name order, so that a test can compare
the engine's files with the reference's without the reference's long,
file-bound run.  CPU only; run from the repository root:

    python tests/golden/make_ply_files_golden.py
"""
import ctypes
import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

CASES = [("KRvK", None, None), ("KRvKN", 7, 5)]


def zstd():
    z = ctypes.CDLL("libzstd.so.1")
    z.ZSTD_decompress.restype = ctypes.c_size_t
    z.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p,
                                  ctypes.c_size_t]
    z.ZSTD_isError.restype = ctypes.c_uint
    z.ZSTD_isError.argtypes = [ctypes.c_size_t]
    return z


def read_slice_file(z, path):
    """read_data (util.c:316-343): frames {compressed size, chunk size,
    offset} as three size_t, then the zstd data, in any order; returns the
    bitmap bytes."""
    data = open(path, "rb").read()
    parts, pos = {}, 0
    while pos < len(data):
        c, chunk, idx = struct.unpack_from("<QQQ", data, pos)
        pos += 24
        buf = ctypes.create_string_buffer(chunk)
        r = z.ZSTD_decompress(buf, chunk, data[pos:pos + c], c)
        if z.ZSTD_isError(r) or r != chunk:
            raise ValueError(f"bad frame in {path}")
        parts[idx] = buf.raw
        pos += c
    out, at = b"", 0
    for idx in sorted(parts):
        if idx != at:
            raise ValueError(f"gap in {path}")
        out += parts[idx]
        at += len(parts[idx])
    return out


def digests(z, root):
    """{"<n>/<name>/<c>": sha256 of the directory's slices} for the W and L
    directories of every ply and for 0/L and 0/wins."""
    out = {}
    for n in sorted(os.listdir(root), key=lambda x: (not x.isdigit(), x)):
        if not n.isdigit():
            continue
        names = ("L", "wins") if n == "0" else ("W", "L")
        for name in names:
            for c in "wb":
                d = os.path.join(root, n, name, c)
                if not os.path.isdir(d):
                    continue
                h = hashlib.sha256()
                files = sorted(os.listdir(d))
                for f in files:
                    h.update(read_slice_file(z, os.path.join(d, f)))
                out[f"{n}/{name}/{c}"] = [len(files), h.hexdigest()]
    return out


def run(case, z):
    mat, seed, mod = case
    exe = os.path.join(REF, "tb8gen" if seed is None else "tb8gen_stub")
    env = dict(os.environ)
    if seed is not None:
        env["TB8GEN_STUB_SEED"], env["TB8GEN_STUB_MOD"] = str(seed), str(mod)
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([exe, "-t", str(os.cpu_count() or 8), mat], cwd=d, env=env,
                       stdout=subprocess.DEVNULL, check=True)
        return {"seed": seed, "mod": mod, "dirs": digests(z, os.path.join(d, mat))}


def main():
    z = zstd()
    res = {c[0]: run(c, z) for c in CASES}
    with open(os.path.join(HERE, "ply_files.json"), "w") as f:
        json.dump(res, f, indent=0, sort_keys=True)
    print({m: len(v["dirs"]) for m, v in res.items()})


if __name__ == "__main__":
    sys.exit(main())
