"""Shared drivers for the parity tests: run one reference worker on the CUDA
engine (through the C ABI) and on a CPU oracle with the same inputs.

Scenario layout follows the reference's calls: a per-slice worker reads the
scratch slot (slice -1) and the slices its king moves reach, all of which
must be bound (kslice_get_address asserts it, kslice.h:57-61).
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import bitmap_tag, gen_bitmap, king_targets


class GpuSide:
    """The engine through tb8gen_b200 (ctypes over libtbgpu.so)."""

    def __init__(self, material: str):
        import torch

        import tb8gen_b200 as tbg

        self.torch = torch
        self.tbg = tbg
        tbg.init()
        self.m = tbg.Material(material).select()
        self.size, self.bytes, self.sub_bytes = self.m.size, self.m.bytes, self.m.sub_bytes
        self._keep = {}

    def dev(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def set_stub(self, seed, modulus=3):
        self.tbg.set_stub(seed, modulus)

    def predecessors(self, stm, s, src):
        tbg = self.tbg
        self.m.select()
        tbg.unbind_all()
        tg = [s] + king_targets(stm, s)
        T = {t: self.torch.zeros(self.bytes, dtype=self.torch.uint8, device="cuda") for t in tg}
        sd = self.dev(src)
        tbg.bind(-1, sd)
        for t in tg:
            tbg.bind(t, T[t])
        tbg.predecessors(stm, s)
        tbg.sync()
        return {t: T[t].cpu().numpy() for t in tg}

    def predecessors_sub(self, stm, s, legality, sub):
        tbg = self.tbg
        self.m.select()
        tbg.unbind_all()
        tg = [s] + king_targets(stm, s)
        T = {t: self.torch.zeros(self.bytes, dtype=self.torch.uint8, device="cuda") for t in tg}
        sd = self.dev(sub)
        for t in tg:
            tbg.bind(t, T[t])
        tbg.bind_sub(s, sd)
        tbg.predecessors_sub(stm, s, legality)
        tbg.sync()
        return {t: T[t].cpu().numpy() for t in tg}

    def check_successors(self, stm, s, cand, wins, subs):
        tbg = self.tbg
        self.m.select()
        tbg.unbind_all()
        x = self.dev(cand)
        tbg.bind(-1, x)
        keep = [x]
        for t in wins:
            w, sb = self.dev(wins[t]), self.dev(subs[t])
            keep += [w, sb]
            tbg.bind(t, w)
            tbg.bind_sub(t, sb)
        tbg.check_successors(stm, s)
        tbg.sync()
        return x.cpu().numpy()

    def calc_sub(self, stm, s):
        self.m.select()
        cls = [self.torch.zeros(self.sub_bytes, dtype=self.torch.uint8, device="cuda") for _ in range(5)]
        self.tbg.calc_sub(stm, s, cls)
        self.tbg.sync()
        return [c.cpu().numpy() for c in cls]

    def calc_illegal(self, s):
        self.m.select()
        w = self.torch.full((self.bytes,), 0xAB, dtype=self.torch.uint8, device="cuda")
        b = self.torch.full((self.bytes,), 0xCD, dtype=self.torch.uint8, device="cuda")
        self.tbg.calc_illegal(s, w, b)
        self.tbg.sync()
        return w.cpu().numpy(), b.cpu().numpy()

    def calc_mate(self, s, ill_w, ill_b):
        self.m.select()
        iw, ib = self.dev(ill_w), self.dev(ill_b)
        mw = self.torch.full((self.bytes,), 0x5A, dtype=self.torch.uint8, device="cuda")
        mb = self.torch.full((self.bytes,), 0xA5, dtype=self.torch.uint8, device="cuda")
        self.tbg.calc_mate(s, iw, ib, mw, mb)
        self.tbg.sync()
        return mw.cpu().numpy(), mb.cpu().numpy()

    def epilogue_W(self, T, wins):
        self.m.select()
        self.tbg.unbind_all()
        t, w = self.dev(T), self.dev(wins)
        self.tbg.bind(0, t)
        self.tbg.bind(-1, w)
        c = self.tbg.epilogue_W(0, -1)
        return c, t.cpu().numpy(), w.cpu().numpy()


class OracleSide:
    """A CPU oracle (oracle.Port or oracle.Ref) driven the same way."""

    def __init__(self, O):
        self.O = O
        self.size, self.bytes, self.sub_bytes = O.size, O.bytes, O.sub_bytes

    def set_stub(self, seed, modulus=3):
        self.O.set_stub(seed, modulus)

    def predecessors(self, stm, s, src):
        O = self.O
        O.unbind_all()
        tg = [s] + king_targets(stm, s)
        T = {t: np.zeros(self.bytes, np.uint8) for t in tg}
        O.bind(-1, src.copy())
        for t in tg:
            O.bind(t, T[t], np.zeros(self.sub_bytes, np.uint8))
        O.predecessors(stm, s)
        return T

    def predecessors_sub(self, stm, s, legality, sub):
        O = self.O
        O.unbind_all()
        tg = [s] + king_targets(stm, s)
        T = {t: np.zeros(self.bytes, np.uint8) for t in tg}
        O.bind(-1, np.zeros(self.bytes, np.uint8))
        for t in tg:
            O.bind(t, T[t], sub.copy() if t == s else np.zeros(self.sub_bytes, np.uint8))
        O.predecessors_sub(stm, s, legality)
        return T

    def check_successors(self, stm, s, cand, wins, subs):
        O = self.O
        O.unbind_all()
        x = cand.copy()
        O.bind(-1, x)
        for t in wins:
            O.bind(t, wins[t].copy(), subs[t].copy())
        O.check_successors(stm, s)
        return x

    def calc_sub(self, stm, s):
        cls = [np.zeros(self.sub_bytes, np.uint8) for _ in range(5)]
        self.O.calc_sub(stm, s, cls)
        return cls

    def calc_illegal(self, s):
        w = np.zeros(self.bytes, np.uint8)
        b = np.zeros(self.bytes, np.uint8)
        self.O.calc_illegal(s, w, b)
        return w, b

    def calc_mate(self, s, ill_w, ill_b):
        mw = np.zeros(self.bytes, np.uint8)
        mb = np.zeros(self.bytes, np.uint8)
        self.O.calc_mate(s, ill_w, ill_b, mw, mb)
        return mw, mb

    def epilogue_W(self, T, wins):
        t, w = T.copy(), wins.copy()
        c = self.O.epilogue_W(t, w)
        return c, t, w


def verify_inputs(side, stm, s, cand_p, wins_p, seed=3):
    """Candidates of (stm, s) and, for s and its king-move slices, the
    opponent's wins (illegal mask | Bernoulli) and sub/win bitmaps -- the
    buffers calc_L_n loads before check_successors (tb8gen.c:1002-1011).
    The illegal masks and sub bitmaps come from `side` itself (an oracle)."""
    size, nbytes = side.size, side.bytes
    cand = gen_bitmap(size, nbytes, seed, bitmap_tag(1, stm, s), cand_p)
    wins, subs = {}, {}
    for t in [s] + king_targets(stm, s):
        ill = side.calc_illegal(t)[stm ^ 1]
        wins[t] = ill | gen_bitmap(size, nbytes, seed, bitmap_tag(5, stm ^ 1, t), wins_p)
        subs[t] = side.calc_sub(stm ^ 1, t)[4]
    return cand, wins, subs


def diff_report(a: dict, b: dict) -> str:
    out = []
    for k in a:
        if not np.array_equal(a[k], b[k]):
            d = np.flatnonzero(a[k] != b[k])
            out.append(f"slice {k}: {d.size} bytes differ, first at {d[0]}")
    return "; ".join(out)
