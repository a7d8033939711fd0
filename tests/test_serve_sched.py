"""The serving scheduler (tb8gen_b200.serve.Scheduler) on the CPU with a fake
executor and a simulated clock: requests are admitted in arrival order into
free slots while their memory fits, never more than `slots` at once or
beyond the budget, every request finishes, and the latency bookkeeping adds
up.  The request generator is seeded and rate-independent."""
from __future__ import annotations

import pytest

from tb8gen_b200.serve import Request, Scheduler, make_requests, summarize


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def idle(self, dt):
        self.t += max(dt, 1e-4)


class FakeExecutor:
    """Each request takes `dur` seconds of simulated time and `mem` bytes."""

    def __init__(self, clock, budget, dur, mem):
        self.clock, self.budget, self.dur, self.mem = clock, budget, dur, mem
        self.used = 0
        self.max_used = 0
        self.inflight = 0
        self.max_inflight = 0
        self.order = []

    def positions(self, req):
        return 10

    def can_admit(self, req):
        return self.used + self.mem[req.rid] <= self.budget

    def issue(self, req, slot):
        self.used += self.mem[req.rid]
        self.max_used = max(self.max_used, self.used)
        self.inflight += 1
        self.max_inflight = max(self.max_inflight, self.inflight)
        self.order.append(req.rid)
        return (req, self.clock() + self.dur[req.rid])

    def done(self, h):
        return self.clock() >= h[1]

    def finish(self, h):
        self.used -= self.mem[h[0].rid]
        self.inflight -= 1
        return h[0].rid


def _reqs(n, gap):
    return [Request(i, i * gap, "ply", "KRvK") for i in range(n)]


@pytest.mark.parametrize("slots", [1, 3, 8])
def test_slots_budget_and_order(slots):
    clk = FakeClock()
    n = 30
    reqs = _reqs(n, 0.001)
    dur = {i: 0.01 * (1 + i % 4) for i in range(n)}
    mem = {i: 100 * (1 + i % 3) for i in range(n)}
    ex = FakeExecutor(clk, 450, dur, mem)
    recs, makespan = Scheduler(ex, slots).run(reqs, clock=clk, idle=clk.idle)
    assert sorted(r.rid for r in recs) == list(range(n))
    assert ex.order == list(range(n))            # FIFO admission
    assert ex.max_inflight <= slots
    assert ex.max_used <= 450
    for r in recs:
        assert r.arrival <= r.admitted <= r.finished
        assert r.finished - r.admitted >= dur[r.rid] - 1e-9
        assert r.result == r.rid
    s = summarize(recs, makespan)
    assert s["jobs"] == n and s["p50_ms"] <= s["p99_ms"]


def test_overlap_beats_serial():
    """With idle slots, requests arriving during others' work are admitted
    at once: the makespan shrinks against one slot."""
    n = 20
    reqs = _reqs(n, 0.0005)
    dur = {i: 0.01 for i in range(n)}
    mem = {i: 1 for i in range(n)}
    c1, c4 = FakeClock(), FakeClock()
    _, m1 = Scheduler(FakeExecutor(c1, 10 ** 9, dur, mem), 1).run(reqs, clock=c1, idle=c1.idle)
    _, m4 = Scheduler(FakeExecutor(c4, 10 ** 9, dur, mem), 4).run(reqs, clock=c4, idle=c4.idle)
    assert m4 < m1 / 2.5


def test_unadmittable_request_raises():
    clk = FakeClock()
    reqs = _reqs(1, 0.0)
    ex = FakeExecutor(clk, 10, {0: 0.01}, {0: 11})
    with pytest.raises(RuntimeError):
        Scheduler(ex, 2).run(reqs, clock=clk, idle=clk.idle)


def test_request_stream_seeded_and_rate_independent():
    a = make_requests(200, 10.0, ["KRRRvKRRR", "KQRvKRRR"], ["KQRvKRR"])
    b = make_requests(200, 1000.0, ["KRRRvKRRR", "KQRvKRRR"], ["KQRvKRR"])
    assert [(r.kind, r.material, r.slice, r.p, r.seed, r.n, r.offset) for r in a] == \
           [(r.kind, r.material, r.slice, r.p, r.seed, r.n, r.offset) for r in b]
    assert abs(a[-1].arrival / b[-1].arrival - 100.0) < 1e-6
    kinds = [r.kind for r in a]
    assert 0.55 < kinds.count("ply") / len(kinds) < 0.85
    sizes = [r.n for r in a if r.kind == "probe"]
    assert min(sizes) >= 1000 and max(sizes) <= 1_000_000
    assert all(r.offset + r.n <= 1 << 20 for r in a if r.kind == "probe")
