"""Digests of the reference program's per-ply files for the fixpoint
material (tests/golden/fixpoint_KQRvKRR.json).

The unmodified reference program with the seeded 7-piece stub
(oracle/_ref/tb8gen_stub, seed 1, values mod 3 -- the stub the fixpoint
bench gives tbgen) runs the whole generation of KQRvKRR (462 king slices of
6,727,980 positions per side, 101 plies) on the host cores and writes its
per-ply files; every W and L directory of every ply, the mates (0/L) and the
final "wins" (0/wins) are recorded as the SHA-256 of their 462 decompressed
slices, as tests/golden/make_ply_files_golden.py records KRvK and KRvKN.
The program's per-ply count lines ("w12_b = 345", tb8gen.c:1024, 1082) are
recorded as "counts".  The reference's run is long (over an hour on 8 host
cores, gigabytes of files), so the digests are made once and committed.

    python tests/golden/make_fixpoint_golden.py [--dir DIR]

With --dir, the files of a finished run in DIR/KQRvKRR are digested instead
of running the program again, and the count lines of its standard output,
if saved to DIR/stdout.
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
MATERIAL, SEED, MOD = "KQRvKRR", 1, 3

_spec = importlib.util.spec_from_file_location("ply_files_golden",
                                               os.path.join(HERE, "make_ply_files_golden.py"))
_g = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_g)


def count_lines(text):
    return [l.strip() for l in text.splitlines()
            if " = " in l and not l.startswith("number of threads")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dir", default=None, help="a finished run's working directory")
    a = ap.parse_args()
    z = _g.zstd()
    counts = []
    if a.dir:
        dirs = _g.digests(z, os.path.join(a.dir, MATERIAL))
        if os.path.exists(os.path.join(a.dir, "stdout")):
            counts = count_lines(open(os.path.join(a.dir, "stdout")).read())
    else:
        env = dict(os.environ, TB8GEN_STUB_SEED=str(SEED), TB8GEN_STUB_MOD=str(MOD))
        with tempfile.TemporaryDirectory() as d:
            r = subprocess.run([os.path.join(REF, "tb8gen_stub"), "-t",
                                str(os.cpu_count() or 8), MATERIAL], cwd=d, env=env,
                               stdout=subprocess.PIPE, text=True, check=True)
            counts = count_lines(r.stdout)
            dirs = _g.digests(z, os.path.join(d, MATERIAL))
    out = {"material": MATERIAL, "seed": SEED, "mod": MOD, "dirs": dirs, "counts": counts}
    with open(os.path.join(HERE, f"fixpoint_{MATERIAL}.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(len(dirs), "directories", len(counts), "count lines")


if __name__ == "__main__":
    sys.exit(main())
