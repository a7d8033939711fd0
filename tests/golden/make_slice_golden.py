"""Regenerates tests/golden/slice_ply.json: the outputs of whole slice-plies
(W step + epilogue + L step + verify, tb8gen.c:519-527, 1072-1077, 653-661)
computed by the reference's own workers (oracle/_ref/libtbref.so, built by
`make -C oracle ref` from the reference sources) on the seeded inputs that
tb8gen_b200.plyjob.SlicePly builds on the device.

Per case it records the counts (|W(s)|, |L(s)|) and the SHA-256 of every
bitmap the step writes: W(s), wins(s), L(s) and the king-move marks into
each neighbour slice (T(t), X(t)).  The first case is the KRRRvKRRR slice-ply
the ply bench times (king slice 96, sources Bernoulli(0.01), seed 1).

Run from the repository root (all host cores; a few minutes for KRRRvKRRR,
longer for the 96 slices of --mix):
    python -m tests.golden.make_slice_golden [--only KEY] [--mix]
"""
from __future__ import annotations

import argparse
import json
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "slice_ply.json")

# (material, slice, p, seed): the bench's slice-ply first, then slices of the
# uneven mix's materials (a diagonal slice among them)
CASES = [
    ("KRRRvKRRR", 96, 0.01, 1),
]


def key(material, s, p, seed, shared=False):
    return f"{material}/{s}/{p}/{seed}" + ("/shared" if shared else "")


def mix_spec():
    """The uneven mix of the ply bench (96 slices, seed 2; neighbours in
    per-material shared buffers), as bench.workload_spec("mix") draws it."""
    import numpy as np

    rng = np.random.default_rng(2)
    mats = ["KRRRvKRRR", "KQRvKRRR", "KQRRvKRR"]
    ps = [0.001, 0.01, 0.05]
    return [(mats[j % 3], int(rng.integers(0, 462)), ps[(j // 3) % 3], 2) for j in range(96)]


def main():
    from oracle import oracle as orc
    from oracle.plyjob_cpu import CpuSlicePly, inputs_from_oracle
    from tb8gen_b200.plyjob import output_digests

    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--mix", action="store_true",
                    help="the 96 slices of the uneven mix (counts and W/L digests per slice)")
    a = ap.parse_args()
    if not orc.ref_available():
        raise SystemExit("oracle/_ref/libtbref.so not built (make -C oracle ref)")
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    out["source"] = ("reference workers (tb8gen.c predecessors, kslice epilogue, "
                     "check_successors via oracle/_ref/libtbref.so), seeded stub seed 1 mod 3")
    cores = os.cpu_count() or 1
    if a.mix:
        mix = {}
        for c in mix_spec():
            k = key(*c, shared=True)
            if k in mix:
                continue
            O = orc.Ref(c[0], cores)
            O.set_stub(1, 3)
            ply = CpuSlicePly(O, inputs_from_oracle(O, *c, shared=True), 1.0)
            ply.step()
            mix[k] = {"counts": list(ply.counts()), "sha256": output_digests(ply.outputs())}
            print(k, mix[k]["counts"], flush=True)
        out["mix"] = mix
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
        return
    for c in CASES:
        k = key(*c)
        if a.only and a.only != k:
            continue
        t0 = time.time()
        O = orc.Ref(c[0], cores)
        O.set_stub(1, 3)
        inputs = inputs_from_oracle(O, *c)
        ply = CpuSlicePly(O, inputs, 1.0)
        ply.step()
        out[k] = {"counts": list(ply.counts()), "sha256": output_digests(ply.outputs()),
                  "N": inputs["N"]}
        print(k, out[k]["counts"], f"{time.time() - t0:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
