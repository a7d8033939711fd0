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


class CpuSlicePly:
    def __init__(self, O, job, frac: float = 1.0):
        """O: oracle.Ref or oracle.Port for job.material; job: a SlicePly
        whose device inputs are copied to the host."""
        self.O, self.s, self.frac = O, job.s, frac
        self.N, self.B = job.N, job.B
        h = lambda t: t.cpu().numpy().copy()
        self.L_prev = _sample(h(job.L_prev), self.N, frac)
        self.W_prev = _sample(h(job.W_prev), self.N, frac)
        self.wins_in = h(job.wins_in)
        self.sub_win = h(job.sub_win)
        self.wk, self.bk = list(job.wk), list(job.bk)
        self.shared = job.pool is not None
        # neighbour buffers, shared or not exactly as on the device
        if self.shared:
            ts, xs = np.zeros(self.B, np.uint8), np.zeros(self.B, np.uint8)
            wn, sn = h(job.pool.wins_nbr), h(job.pool.sub_nbr)
            self.T_nbr = {t: ts for t in self.wk}
            self.X_nbr = {t: xs for t in self.bk}
            self.wins_nbr = {t: wn for t in self.bk}
            self.sub_nbr = {t: sn for t in self.bk}
        else:
            self.T_nbr = {t: np.zeros(self.B, np.uint8) for t in self.wk}
            self.X_nbr = {t: np.zeros(self.B, np.uint8) for t in self.bk}
            self.wins_nbr = {t: h(job.wins_nbr[t]) for t in self.bk}
            self.sub_nbr = {t: h(job.sub_nbr[t]) for t in self.bk}
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
