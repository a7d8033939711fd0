"""One slice-ply job on the engine: the W step and the L step of calc_W_n /
calc_L_n (tb8gen.c:943-1084) for one king slice, with every bitmap resident
in HBM.

For slice s, white to move in the W step (black in the L step):

  W step  clear T(s); predecessors(WHITE, s) from L_prev = L^b_{n-1}(s)
          (marks into s and its white-king slices, tb8gen.c:1051-1054);
          epilogue: W(s) = T(s) & ~wins_in, wins_out = wins_in | W(s)
          (tb8gen.c:1072-1077).
  L step  clear X(s); candidates(BLACK, s) from W_prev = W^w_{n-1}(s)
          (predecessors() of tb8gen.c:972-975, less the predecessors a
          slider step takes out of white's wins(s), which the verify would
          clear; filtered=False: predecessors() itself);
          check_successors(BLACK, s) against white's "wins" of s and its
          black-king slices and white's sub/win (tb8gen.c:1000-1017); X(s)
          then holds L(s).

Inputs are seeded: L_prev and W_prev are Bernoulli(p) bitmaps with the
positions illegal for their side to move cleared, wins_in(s) and the
neighbours' wins are white's illegal masks (the initial "wins",
tb8gen.c:749-750), sub/win comes from the capture stub.  The inputs stay
unchanged by a step, so every step does the same work.

Neighbour targets: with ``shared_neighbours`` every king-move mark into a
slice other than s goes to one per-material bitmap (and the verify reads
one per-material neighbour "wins"/sub bitmap), so that many jobs fit in
HBM at once; otherwise each neighbour slice gets its own buffers.  Only
T(s) and X(s) are cleared by a step: a neighbour's clear belongs to the
neighbour's own ply.
"""
from __future__ import annotations

import torch

import tb8gen_b200 as tbg

WHITE, BLACK = 0, 1
GAMMA = 0x9E3779B97F4A7C15


def bern_threshold(p: float) -> int:
    return (1 << 64) - 1 if p >= 1.0 else int(p * float(1 << 64))


def tag(bitmap_id: int, stm: int, s: int) -> int:
    return (bitmap_id << 32) | (stm << 16) | (s & 0xFFFF)


_KING_TABLES = None


def _king_tables():
    """KKSquare / KKMap / FlipTest / MirrorMask as generated in the engine's
    host code, restated here for the job layout (probe.c:441-539,
    tb8gen.c:69-89)."""
    global _KING_TABLES
    if _KING_TABLES is not None:
        return _KING_TABLES
    tri = [1, 2, 3, 10, 11, 19, 0, 9, 18, 27]

    def touching(a, b):
        return abs((a & 7) - (b & 7)) <= 1 and abs((a >> 3) - (b >> 3)) <= 1

    kkidx = [[-1] * 64 for _ in range(10)]
    nxt, nd = 0, 441
    for t in range(10):
        for sq in range(64):
            if touching(tri[t], sq):
                continue
            if t >= 6:
                if (sq & 7) < (sq >> 3):
                    continue
                if (sq & 7) == (sq >> 3):
                    kkidx[t][sq] = nd
                    nd += 1
                    continue
            kkidx[t][sq] = nxt
            nxt += 1
    kksq = [None] * 462
    for t in range(10):
        for sq in range(64):
            if kkidx[t][sq] >= 0:
                kksq[kkidx[t][sq]] = (tri[t], sq)
    triangle = [0] * 64
    for sq in range(64):
        f, r = sq & 7, sq >> 3
        f, r = (7 - f if f > 3 else f), (7 - r if r > 3 else r)
        if r > f:
            f, r = r, f
        triangle[sq] = tri.index(r * 8 + f)
    mirror = [(0x07 if (sq & 7) >= 4 else 0) | (0x38 if (sq >> 3) >= 4 else 0) for sq in range(64)]
    flipd = [((sq & 7) << 3) | (sq >> 3) for sq in range(64)]
    kkmap = [[-1] * 64 for _ in range(64)]
    for i in range(64):
        for j in range(64):
            s1, s2 = i ^ mirror[i], j ^ mirror[i]
            tri_ok = (s1 & 7) <= 3 and (s1 >> 3) <= (s1 & 7)
            diag = tri_ok and (s1 & 7) == (s1 >> 3)
            lower = (s2 & 7) >= (s2 >> 3)
            if (not tri_ok) or (diag and not lower):
                s1, s2 = flipd[s1], flipd[s2]
            kkmap[i][j] = kkidx[triangle[s1]][s2]
    _KING_TABLES = (kksq, kkmap)
    return _KING_TABLES


def king_attacks(sq: int) -> int:
    b = 0
    for df in (-1, 0, 1):
        for dr in (-1, 0, 1):
            f, r = (sq & 7) + df, (sq >> 3) + dr
            if (df or dr) and 0 <= f < 8 and 0 <= r < 8:
                b |= 1 << (r * 8 + f)
    return b


def king_slices(stm: int, s: int) -> list[int]:
    """Slices other than s reached by a king move of side stm from slice s."""
    kksq, kkmap = _king_tables()
    ks = list(kksq[s])
    me, opp = ks[stm], ks[stm ^ 1]
    b = king_attacks(me) & ~king_attacks(opp) & ~(1 << opp)
    out = set()
    for to in range(64):
        if b >> to & 1:
            k2 = list(ks)
            k2[stm] = to
            out.add(kkmap[k2[0]][k2[1]])
    out.discard(s)
    return sorted(out)


class MaterialPool:
    """Per-material shared buffers (neighbour sinks and neighbour inputs)."""

    def __init__(self, name: str, seed: int, wins_p: float = 0.0):
        self.m = tbg.Material(name)
        self.name = name
        self.seed = seed
        dev = "cuda"
        B, SB = self.m.bytes, self.m.sub_bytes
        self.t_sink = torch.zeros(B, dtype=torch.uint8, device=dev)
        self.x_sink = torch.zeros(B, dtype=torch.uint8, device=dev)
        # neighbour "wins" and sub/win: white's illegal mask and sub/win of one
        # fixed slice (0), standing for every neighbour of every job.
        self.m.select()
        iw = torch.empty(B, dtype=torch.uint8, device=dev)
        ib = torch.empty(B, dtype=torch.uint8, device=dev)
        tbg.calc_illegal(0, iw, ib)
        self.wins_nbr = iw
        del ib
        cls = [torch.empty(SB, dtype=torch.uint8, device=dev) for _ in range(5)]
        tbg.calc_sub(WHITE, 0, cls)
        self.sub_nbr = cls[4]
        del cls


class SlicePly:
    """Buffers and step of one slice-ply job (see module docstring)."""

    def __init__(self, material: str, s: int, p: float, seed: int,
                 pool: MaterialPool | None = None, filtered: bool = True):
        self.material, self.s, self.p, self.seed = material, s, p, seed
        self.filtered = filtered
        self.pool = pool
        self.m = pool.m if pool is not None else tbg.Material(material)
        self.m.select()
        self.N, self.B, self.SB = self.m.size, self.m.bytes, self.m.sub_bytes
        dev = "cuda"
        z = lambda n=None: torch.zeros(n or self.B, dtype=torch.uint8, device=dev)
        B = self.B
        self.wk = king_slices(WHITE, s)
        self.bk = king_slices(BLACK, s)
        # illegal masks of s
        ill_w, ill_b = z(), z()
        tbg.calc_illegal(s, ill_w, ill_b)
        # inputs
        self.L_prev = z()
        tbg.gen_bernoulli(self.L_prev, self.N, seed, tag(0, BLACK, s), bern_threshold(p))
        self.L_prev &= ~ill_b
        self.W_prev = z()
        tbg.gen_bernoulli(self.W_prev, self.N, seed, tag(3, WHITE, s), bern_threshold(p))
        self.W_prev &= ~ill_w
        self.wins_in = ill_w
        del ill_b
        cls = [z(self.SB) for _ in range(5)]
        tbg.calc_sub(WHITE, s, cls)
        self.sub_win = cls[4]
        del cls
        # outputs
        self.T = z()
        self.X = z()
        self.wins = z()
        if pool is None:
            self.T_nbr = {t: z() for t in self.wk}
            self.X_nbr = {t: z() for t in self.bk}
            self.wins_nbr, self.sub_nbr = {}, {}
            for t in self.bk:
                iw, ib = z(), z()
                tbg.calc_illegal(t, iw, ib)
                self.wins_nbr[t] = iw
                del ib
                c = [z(self.SB) for _ in range(5)]
                tbg.calc_sub(WHITE, t, c)
                self.sub_nbr[t] = c[4]
        else:
            self.T_nbr = {t: pool.t_sink for t in self.wk}
            self.X_nbr = {t: pool.x_sink for t in self.bk}
            self.wins_nbr = {t: pool.wins_nbr for t in self.bk}
            self.sub_nbr = {t: pool.sub_nbr for t in self.bk}
        self.positions = self.N

    # ---- the step, as per-slice calls through the C ABI -------------------
    def w_scatter(self):
        self.m.select()
        tbg.unbind_all()
        tbg.bind(-1, self.L_prev)
        tbg.bind(self.s, self.T)
        for t, buf in self.T_nbr.items():
            tbg.bind(t, buf)
        tbg.clear(self.s)
        tbg.predecessors(WHITE, self.s)

    def w_epilogue(self):
        self.m.select()
        tbg.unbind_all()
        tbg.bind(self.s, self.T)
        tbg.epilogue_W_to(self.s, self.wins_in, self.wins, count=False)

    def l_scatter(self):
        self.m.select()
        tbg.unbind_all()
        tbg.bind(-1, self.W_prev)
        tbg.bind(self.s, self.X)
        for t, buf in self.X_nbr.items():
            tbg.bind(t, buf)
        tbg.clear(self.s)
        if self.filtered:
            # candidates that a slider step leaves in white's wins(s) only:
            # l_verify clears the others anyway
            tbg.candidates(BLACK, self.s, self.wins)
        else:
            tbg.predecessors(BLACK, self.s)

    def l_verify(self):
        self.m.select()
        tbg.unbind_all()
        tbg.bind(-1, self.X)
        tbg.bind(self.s, self.wins)
        tbg.bind_sub(self.s, self.sub_win)
        for t in self.bk:
            tbg.bind(t, self.wins_nbr[t])
            tbg.bind_sub(t, self.sub_nbr[t])
        tbg.check_successors(BLACK, self.s)

    PHASES = ("w_scatter", "w_epilogue", "l_scatter", "l_verify")

    def step(self):
        self.w_scatter()
        self.w_epilogue()
        self.l_scatter()
        self.l_verify()

    def outputs(self) -> dict:
        """Every bitmap a step writes (device tensors): W(s), the new
        wins(s), L(s) and, with per-neighbour buffers, the king-move marks
        into the neighbour slices (T(t) for white's, X(t) for black's)."""
        out = {"W(s)": self.T, "wins(s)": self.wins, "L(s)": self.X}
        if self.pool is None:
            for t, b in self.T_nbr.items():
                out[f"T({t})"] = b
            for t, b in self.X_nbr.items():
                out[f"X({t})"] = b
        return out

    def counts(self):
        """(|W(s)|, |L(s)|) after a step."""
        self.m.select()
        tbg.unbind_all()
        tbg.bind(0, self.T)
        tbg.bind(1, self.X)
        return tbg.count(0), tbg.count(1)


def bitmap_digest(a) -> str:
    """SHA-256 of a bitmap's bytes (a numpy array or a tensor, any device)."""
    import hashlib

    import numpy as np

    if isinstance(a, torch.Tensor):
        a = a.detach().contiguous().cpu().numpy()
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def output_digests(outputs: dict) -> dict:
    """{name: SHA-256} of the bitmaps of SlicePly.outputs() (or of the CPU
    twin's outputs()), names sorted."""
    return {k: bitmap_digest(outputs[k]) for k in sorted(outputs)}


def record_step(jobs):
    """Records one step of every job (phase by phase: all W scatters, all
    epilogues, all L scatters, all verifies) as a batch; returns
    (recorded calls, work items).  tbg.batch_run(0 | 1 | 2) then runs it."""
    tbg.batch_begin()
    try:
        for ph in SlicePly.PHASES:
            for j in jobs:
                getattr(j, ph)()
    finally:
        n = tbg.batch_end()
    return n
