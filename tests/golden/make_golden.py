"""Regenerates tests/golden/ply_golden.json from the reference's own workers
(oracle/_ref/libtbref.so, built by `make -C oracle ref` from the reference
sources).  Run from the repository root:  python -m tests.golden.make_golden
"""
from __future__ import annotations

import json
import os

from oracle import oracle as orc
from tests.golden.scenarios import MATERIALS, run_material
from tests.parity import OracleSide

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if not orc.ref_available():
        raise SystemExit("oracle/_ref/libtbref.so not built")
    out = {"source": "reference workers (tb8gen.c via oracle/_ref/libtbref.so)"}
    for m in MATERIALS:
        out.update(run_material(OracleSide(orc.Ref(m, 8)), m))
    with open(os.path.join(HERE, "ply_golden.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(len(out), "entries")


if __name__ == "__main__":
    main()
