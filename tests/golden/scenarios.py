"""Scenarios of the golden fixtures: each runs one reference worker on
seeded inputs through an oracle side (tests.parity.OracleSide) and returns
a digest of every output buffer.  make_golden.py records the digests of
the reference's own workers (oracle/_ref); test_golden.py replays the same
scenarios on the C restatement."""
from __future__ import annotations

import hashlib

import numpy as np

from oracle import oracle as orc
from tests.parity import OracleSide, verify_inputs

MATERIALS = ["KRRvKR", "KQRvKRR", "KNBvKB", "KRvKNN"]
SLICES = [0, 96, 300, 440, 441, 452, 461]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:32]


def popcount(a: np.ndarray) -> int:
    return int(np.unpackbits(a).sum())


def run_material(side: OracleSide, material: str) -> dict:
    out = {}
    side.set_stub(7, 3)
    for s in SLICES:
        for stm in (0, 1):
            src = orc.gen_bitmap(side.size, side.bytes, 11, orc.bitmap_tag(0, stm ^ 1, s), 0.05)
            T = side.predecessors(stm, s, src)
            out[f"{material}/pred/{stm}/{s}"] = {str(t): [digest(v), popcount(v)] for t, v in T.items()}
            for legality in (0, 1):
                sub = orc.gen_bitmap(side.sub_bytes * 8, side.sub_bytes, 5,
                                     orc.bitmap_tag(2, stm ^ 1, s), 0.1)
                T = side.predecessors_sub(stm, s, legality, sub)
                out[f"{material}/psub/{stm}/{s}/{legality}"] = {
                    str(t): [digest(v), popcount(v)] for t, v in T.items()}
            cand, wins, subs = verify_inputs(side, stm, s, 0.3, 0.9)
            x = side.check_successors(stm, s, cand, wins, subs)
            out[f"{material}/verify/{stm}/{s}"] = [digest(x), popcount(x)]
            for mod in (3, 5):
                side.set_stub(1234, mod)
                cls = side.calc_sub(stm, s)
                out[f"{material}/sub/{stm}/{s}/{mod}"] = [[digest(c), popcount(c)] for c in cls]
            side.set_stub(7, 3)
        ill = side.calc_illegal(s)
        out[f"{material}/illegal/{s}"] = [[digest(c), popcount(c)] for c in ill]
        mate = side.calc_mate(s, *ill)
        out[f"{material}/mate/{s}"] = [[digest(c), popcount(c)] for c in mate]
    T = orc.gen_bitmap(side.size, side.bytes, 3, 1, 0.3)
    W = orc.gen_bitmap(side.size, side.bytes, 3, 2, 0.4)
    c, t, w = side.epilogue_W(T, W)
    out[f"{material}/epilogue"] = [c, digest(t), digest(w)]
    return out
