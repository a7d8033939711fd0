"""Oracle test infrastructure -- NOT product code.

The CPU twin of tb8gen_b200.plyjob.SlicePly: the same slice-ply step (W step
and L step of one king slice, same bindings) run by a CPU oracle (the
reference's own workers through oracle/_ref, or the C restatement) on host
copies of the job's inputs.  Used by the parity tests and by bench.py's
CPU-baseline leg and reference arm.

A *sample* restricts the two scatter sources to their first `frac` of the
slice's positions (whole 64-bit words); the epilogue and the verify then run
over the whole slice as usual, and their cost scales with the candidates the
sampled sources produce.
"""
from __future__ import annotations

import time

import numpy as np

WHITE, BLACK = 0, 1


def _sample(a: np.ndarray, nbits: int, frac: float) -> np.ndarray:
    if frac >= 1.0:
        return a.copy()
    out = np.zeros_like(a)
    nbytes = (int(nbits * frac) // 64) * 8
    out[:nbytes] = a[:nbytes]
    return out


def inputs_from_engine_job(job) -> dict:
    """Host copies of an engine job's inputs (tb8gen_b200.plyjob.SlicePly)."""
    h = lambda t: t.cpu().numpy().copy()
    d = {"material": job.material, "s": job.s, "N": job.N, "B": job.B,
         "L_prev": h(job.L_prev), "W_prev": h(job.W_prev), "wins_in": h(job.wins_in),
         "sub_win": h(job.sub_win), "wk": list(job.wk), "bk": list(job.bk),
         "shared": job.pool is not None}
    if job.pool is not None:
        d["wins_nbr"] = {t: None for t in job.bk}
        d["pool_wins"], d["pool_sub"] = h(job.pool.wins_nbr), h(job.pool.sub_nbr)
        d["sub_nbr"] = {t: None for t in job.bk}
    else:
        d["wins_nbr"] = {t: h(job.wins_nbr[t]) for t in job.bk}
        d["sub_nbr"] = {t: h(job.sub_nbr[t]) for t in job.bk}
    return d


def inputs_from_oracle(O, material: str, s: int, p: float, seed: int,
                       shared: bool = False) -> dict:
    """The same inputs as tb8gen_b200.plyjob.SlicePly(material, s, p, seed)
    computed on the CPU by the oracle O itself: the illegal masks and
    sub/win bitmaps by its calc_illegal / calc_sub, the Bernoulli sources by
    the same seeded splitmix64 stream.  With `shared`, the neighbours are
    those of a MaterialPool: one "wins" (white's illegal mask of slice 0) and
    one sub/win (of slice 0) for every neighbour, marks into shared sinks."""
    from oracle.oracle import bitmap_tag, gen_bitmap, king_targets

    N, B = O.size, O.bytes

    def illegal(t):
        w, b = np.zeros(B, np.uint8), np.zeros(B, np.uint8)
        O.calc_illegal(t, w, b)
        return w, b

    def sub_win(t):
        cls = [np.zeros(O.sub_bytes, np.uint8) for _ in range(5)]
        O.calc_sub(WHITE, t, cls)
        return cls[4]

    ill_w, ill_b = illegal(s)
    d = {"material": material, "s": s, "N": N, "B": B,
         "L_prev": gen_bitmap(N, B, seed, bitmap_tag(0, BLACK, s), p) & ~ill_b,
         "W_prev": gen_bitmap(N, B, seed, bitmap_tag(3, WHITE, s), p) & ~ill_w,
         "wins_in": ill_w, "sub_win": sub_win(s),
         "wk": king_targets(WHITE, s), "bk": king_targets(BLACK, s), "shared": False}
    if shared:
        d["shared"] = True
        d["pool_wins"], d["pool_sub"] = illegal(0)[0], sub_win(0)
        d["wins_nbr"] = {t: None for t in d["bk"]}
        d["sub_nbr"] = {t: None for t in d["bk"]}
        return d
    d["wins_nbr"] = {t: illegal(t)[0] for t in d["bk"]}
    d["sub_nbr"] = {t: sub_win(t) for t in d["bk"]}
    return d


class CpuSlicePly:
    def __init__(self, O, job, frac: float = 1.0):
        """O: oracle.Ref or oracle.Port for the job's material; job: an
        engine SlicePly (its inputs are copied to the host) or a dict from
        inputs_from_oracle / inputs_from_engine_job."""
        d = job if isinstance(job, dict) else inputs_from_engine_job(job)
        self.O, self.s, self.frac = O, d["s"], frac
        self.N, self.B = d["N"], d["B"]
        self.L_prev = _sample(d["L_prev"], self.N, frac)
        self.W_prev = _sample(d["W_prev"], self.N, frac)
        self.wins_in = d["wins_in"]
        self.sub_win = d["sub_win"]
        self.wk, self.bk = list(d["wk"]), list(d["bk"])
        self.shared = d["shared"]
        if self.shared:
            ts, xs = np.zeros(self.B, np.uint8), np.zeros(self.B, np.uint8)
            self.T_nbr = {t: ts for t in self.wk}
            self.X_nbr = {t: xs for t in self.bk}
            self.wins_nbr = {t: d["pool_wins"] for t in self.bk}
            self.sub_nbr = {t: d["pool_sub"] for t in self.bk}
        else:
            self.T_nbr = {t: np.zeros(self.B, np.uint8) for t in self.wk}
            self.X_nbr = {t: np.zeros(self.B, np.uint8) for t in self.bk}
            self.wins_nbr = dict(d["wins_nbr"])
            self.sub_nbr = dict(d["sub_nbr"])
        self.T = np.zeros(self.B, np.uint8)
        self.X = np.zeros(self.B, np.uint8)
        self.wins = np.zeros(self.B, np.uint8)
        self.zsub = np.zeros(O.sub_bytes, np.uint8)
        self.times = {}

    def step(self):
        O, s = self.O, self.s
        t0 = time.perf_counter()
        O.unbind_all()
        O.bind(-1, self.L_prev)
        self.T[:] = 0
        O.bind(s, self.T, self.zsub)
        for t, b in self.T_nbr.items():
            O.bind(t, b, self.zsub)
        O.predecessors(WHITE, s)
        t1 = time.perf_counter()
        self.wins[:] = self.wins_in
        self.cnt_w = O.epilogue_W(self.T, self.wins)
        t2 = time.perf_counter()
        O.unbind_all()
        O.bind(-1, self.W_prev)
        self.X[:] = 0
        O.bind(s, self.X, self.zsub)
        for t, b in self.X_nbr.items():
            O.bind(t, b, self.zsub)
        O.predecessors(BLACK, s)
        t3 = time.perf_counter()
        O.unbind_all()
        O.bind(-1, self.X)
        O.bind(s, self.wins, self.sub_win)
        for t in self.bk:
            O.bind(t, self.wins_nbr[t], self.sub_nbr[t])
        O.check_successors(BLACK, s)
        t4 = time.perf_counter()
        self.times = {"w_scatter": t1 - t0, "w_epilogue": t2 - t1,
                      "l_scatter": t3 - t2, "l_verify": t4 - t3}
        return t4 - t0

    def outputs(self) -> dict:
        """Every bitmap a step writes, named as tb8gen_b200.plyjob.SlicePly
        .outputs() names them: W(s), wins(s), L(s) and the king-move marks
        into the neighbour slices (T(t) of white's, X(t) of black's)."""
        out = {"W(s)": self.T, "wins(s)": self.wins, "L(s)": self.X}
        if not self.shared:
            for t, b in self.T_nbr.items():
                out[f"T({t})"] = b
            for t, b in self.X_nbr.items():
                out[f"X({t})"] = b
        return out

    def counts(self):
        """(|W(s)|, |L(s)|) after a step."""
        return self.O.count(self.T), self.O.count(self.X)
