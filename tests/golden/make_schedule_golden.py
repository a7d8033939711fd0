"""Regenerates tests/golden/schedule_counts.json: the per-ply counts printed
by the unmodified reference program (oracle/_ref/tb8gen, built from the
reference sources by `make -C oracle refbin refstub`) for whole generations
of small materials.  Materials with captures into 4+ pieces run the
reference program with probe_wdl replaced by the seeded stub
(oracle/_ref/tb8gen_stub, seed and modulus from the environment).  Each run
writes the reference's slice files into a temporary directory.

    python -m tests.golden.make_schedule_golden [--jobs N]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "..", "oracle", "_ref")

# material, stub seed, stub modulus (None: the plain reference program)
CASES = [("KRvK", None, None), ("KQvK", None, None), ("KRRvK", 1, 3),
         ("KRvKR", 1, 3), ("KRvKN", 7, 5), ("KQvKR", 1, 3), ("KRRvKR", 1, 3)]


def count_lines(text: str) -> list[str]:
    keep = ("broken_", "l", "w")
    out = []
    for line in text.splitlines():
        line = line.strip()
        if " = " in line and line.startswith(keep) and not line.startswith("number"):
            out.append(line)
    return out


def run(case):
    mat, seed, mod = case
    exe = os.path.join(REF, "tb8gen" if seed is None else "tb8gen_stub")
    env = dict(os.environ)
    if seed is not None:
        env["TB8GEN_STUB_SEED"], env["TB8GEN_STUB_MOD"] = str(seed), str(mod)
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([exe, "-t", "8", mat], cwd=d, env=env, capture_output=True,
                           text=True, check=True)
    return mat, {"seed": seed, "mod": mod, "lines": count_lines(r.stdout)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=4)
    a = ap.parse_args()
    with ThreadPoolExecutor(a.jobs) as ex:
        res = dict(ex.map(run, CASES))
    with open(os.path.join(HERE, "schedule_counts.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print({m: len(v["lines"]) for m, v in res.items()})


if __name__ == "__main__":
    main()
