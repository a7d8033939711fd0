"""Serving loop: ply jobs and probe batches arriving over time, run with
continuous batching on one GPU.

A request is either a *ply job* -- one slice-ply (W step + L step, as
``plyjob.SlicePly``) of king slice ``s`` of a material, its sources seeded
by (seed, p) -- or a *probe batch* -- ``n`` positions probed (WDL) against a
resident 7-piece table.  The server

* keeps every material's per-slice table bitmaps (the illegal masks, which
  are the initial "wins" and mask the sources, and the capture class
  sub/win) resident in HBM, computing them on first use and, when the
  admission budget runs short, spilling the least recently used ones to
  pinned host memory (the disk tier of the reference, ``kslice_read`` /
  ``kslice_write``, becomes host memory) and reading them back on the
  next use;
* admits a waiting request as soon as a slot (a CUDA stream) is free and
  its memory fits the budget, so that requests arriving while others run
  are admitted as slots and memory free up and their kernels overlap on the
  device;
* reports per-request latency (arrival to result on the host) and
  throughput.

The scheduler is independent of the device (``Scheduler`` drives any
executor with ``can_admit``/``issue``/``done``/``finish``); ``GpuExecutor``
runs the work through the C ABI.  One host thread drives everything, as the
library requires; its calls are stream-ordered on the stream it is given
per request.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

WHITE, BLACK = 0, 1


# ------------------------------------------------------------------ requests
@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the stream
    kind: str                   # "ply" | "probe"
    material: str
    slice: int = 0              # ply: king slice
    p: float = 0.01             # ply: source density
    seed: int = 0               # ply: input seed
    n: int = 0                  # probe: positions
    offset: int = 0             # probe: first position in the material's pool


@dataclass
class Record:
    rid: int
    kind: str
    material: str
    positions: int
    arrival: float
    admitted: float
    finished: float
    result: object = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_requests(njobs: int, rate: float, ply_materials, probe_materials, seed: int = 4,
                  ply_frac: float = 0.7, probe_min: int = 1000, probe_max: int = 1_000_000,
                  pool_n: int = 1 << 20, ps=(0.001, 0.01, 0.05)):
    """A Poisson stream of `njobs` requests at `rate` per second: ply jobs
    (fraction `ply_frac`) on uniform king slices of `ply_materials`, probe
    batches of log-uniform size in [probe_min, probe_max] on
    `probe_materials`.  The jobs depend on `seed` only; `rate` scales the
    arrival times, so every rate serves the same jobs."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0, njobs)
    out, t = [], 0.0
    for i in range(njobs):
        t += gaps[i] / rate
        if rng.random() < ply_frac:
            out.append(Request(i, t, "ply", str(rng.choice(ply_materials)),
                               slice=int(rng.integers(0, 462)), p=float(rng.choice(ps)),
                               seed=int(rng.integers(1, 1 << 30))))
        else:
            n = int(round(math.exp(rng.uniform(math.log(probe_min), math.log(probe_max)))))
            n = min(n, pool_n)
            out.append(Request(i, t, "probe", str(rng.choice(probe_materials)), n=n,
                               offset=int(rng.integers(0, pool_n - n + 1))))
    return out


def percentile(xs, q):
    if not xs:
        return None
    return float(np.percentile(np.asarray(xs), q))


def summarize(records, makespan):
    lat = [r.latency for r in records]
    pos = sum(r.positions for r in records)
    return {"jobs": len(records), "p50_ms": round(1e3 * percentile(lat, 50), 3),
            "p99_ms": round(1e3 * percentile(lat, 99), 3),
            "mean_ms": round(1e3 * float(np.mean(lat)), 3),
            "makespan_s": round(makespan, 4), "positions": pos,
            "positions_per_s": round(pos / makespan, 1) if makespan > 0 else None}


# ------------------------------------------------------------------ scheduler
class Scheduler:
    """Continuous batching over `slots` concurrent requests: requests are
    admitted in arrival order (the head waits when its memory does not fit
    yet), each into a free slot; finished requests free their slot and
    memory at once."""

    def __init__(self, executor, slots: int):
        self.ex = executor
        self.slots = slots

    def run(self, requests, clock=time.perf_counter, idle=time.sleep):
        reqs = sorted(requests, key=lambda r: r.arrival)
        waiting = collections.deque()
        inflight = {}                     # slot -> (request, handle, admitted)
        free = list(range(self.slots))
        records = []
        i = 0
        t0 = clock()
        while i < len(reqs) or waiting or inflight:
            now = clock() - t0
            while i < len(reqs) and reqs[i].arrival <= now:
                waiting.append(reqs[i])
                i += 1
            progressed = False
            for slot in list(inflight):
                req, h, adm = inflight[slot]
                if self.ex.done(h):
                    result = self.ex.finish(h)
                    fin = clock() - t0
                    records.append(Record(req.rid, req.kind, req.material,
                                          self.ex.positions(req), req.arrival, adm, fin, result))
                    del inflight[slot]
                    free.append(slot)
                    progressed = True
            while waiting and free:
                req = waiting[0]
                if not self.ex.can_admit(req):
                    if not inflight:
                        raise RuntimeError(f"request {req.rid} can never be admitted")
                    break
                waiting.popleft()
                slot = free.pop()
                adm = clock() - t0
                inflight[slot] = (req, self.ex.issue(req, slot), adm)
                progressed = True
            if not progressed:
                if inflight:
                    idle(0)
                elif i < len(reqs):
                    idle(max(0.0, reqs[i].arrival - (clock() - t0)))
        makespan = (max(r.finished for r in records) if records else 0.0)
        return records, makespan


# ------------------------------------------------------------------ GPU side
@dataclass
class _State:
    """Resident table bitmaps of one (material, slice)."""
    dev: list | None = None           # [ill_w, ill_b, sub_win] on the device
    host: list | None = None          # pinned copies while spilled
    bytes: int = 0
    pins: int = 0
    ready: object = None              # CUDA event: dev holds valid data after it
    last_use: float = 0.0


@dataclass
class _Job:
    req: Request
    event: object
    bufs: list = field(default_factory=list)
    nbytes: int = 0
    state_key: tuple | None = None
    out: list | None = None


class SpillError(RuntimeError):
    """The pinned host tier cannot take a spilled slice state (its budget
    is spent, or the host refused to lock more memory)."""


class GpuExecutor:
    """Runs requests through the C ABI, one CUDA stream per slot.

    `host_budget_bytes` caps the page-locked host memory that spilled slice
    states may hold (None: whatever the host grants); a spill beyond it
    raises SpillError instead of admitting the request, as the reference
    exits when its disk tier fails (util.c:229-243)."""

    def __init__(self, ply_materials, tables: dict, pools: dict, slots: int,
                 budget_bytes: int, keep_results: bool = False, probe_max: int = 1_000_000,
                 query_bytes: int = 16, host_budget_bytes: int | None = None):
        import torch

        import tb8gen_b200 as tbg
        from tb8gen_b200.plyjob import MaterialPool

        self.torch, self.tbg = torch, tbg
        self.budget = budget_bytes
        self.keep = keep_results
        self.streams = [torch.cuda.Stream() for _ in range(slots)]
        self.spill_stream = torch.cuda.Stream()
        self.tables = tables                        # material -> DeviceTable (resident)
        self.table_busy = {m: False for m in tables}
        self.qpool = pools                          # material -> pinned host queries
        if query_bytes not in (8, 16):
            raise ValueError("queries are 16-byte tbg_query or 8-byte compact ones")
        self.qb = query_bytes
        self.used = sum(t.bytes for t in tables.values())
        self.mpools = {}
        for m in ply_materials:
            mp = MaterialPool(m, 7)
            self.mpools[m] = mp
            self.used += 2 * mp.m.bytes + mp.m.bytes + mp.m.sub_bytes
        # per-table probe scratch: a batch of probe_max positions holds at most
        # min(probe_max, blocks) blocks of 16 KiB plus 8 B per position
        self.probe_scratch = {}
        for m, t in tables.items():
            nb = sum(t.layout(b)[1] for b in self._sides(t))
            self.probe_scratch[m] = min(probe_max, nb) * 16384 + 8 * probe_max + 20 * nb
            self.used += self.probe_scratch[m]
        self.states = collections.OrderedDict()     # (material, slice) -> _State
        self.spills = 0
        self.host_budget = host_budget_bytes
        self.host_used = 0
        self.reloads = 0
        self.builds = 0
        self.peak = self.used

    @staticmethod
    def _sides(t):
        try:
            t.layout(1)
            return (0, 1)
        except Exception:
            return (0,)

    # -- memory --------------------------------------------------------------
    def positions(self, req):
        return self.mpools[req.material].m.size if req.kind == "ply" else req.n

    def _job_bytes(self, req):
        if req.kind == "probe":
            return req.n * (self.qb + 1)
        m = self.mpools[req.material].m
        need = 5 * m.bytes
        st = self.states.get((req.material, req.slice))
        if st is None or st.dev is None:
            need += 2 * m.bytes + m.sub_bytes
        return need

    def _evict_for(self, need):
        """Spills unpinned states, least recently used first, until `need`
        more bytes fit; False if they cannot."""
        for key in list(self.states):
            if self.used + need <= self.budget:
                break
            st = self.states[key]
            if st.pins or st.dev is None:
                continue
            self._spill(st)
        return self.used + need <= self.budget

    def _host_tier(self, sizes):
        """Page-locked host buffers for a spilled state, within the host
        budget; SpillError when they do not fit or cannot be locked."""
        need = sum(sizes)
        if self.host_budget is not None and self.host_used + need > self.host_budget:
            raise SpillError(f"pinned host tier full: {self.host_used} + {need} bytes > "
                             f"budget {self.host_budget}")
        try:
            bufs = [self.torch.empty(n, dtype=self.torch.uint8, pin_memory=True) for n in sizes]
        except RuntimeError as e:
            raise SpillError(f"cannot lock {need} bytes of host memory: {e}") from e
        self.host_used += need
        return bufs

    def _spill(self, st):
        torch = self.torch
        if st.host is None:
            st.host = self._host_tier([b.numel() for b in st.dev])
        with torch.cuda.stream(self.spill_stream):
            if st.ready is not None:
                self.spill_stream.wait_event(st.ready)
            for h, d in zip(st.host, st.dev):
                h.copy_(d, non_blocking=True)
        self.spill_stream.synchronize()
        st.dev = None
        st.ready = None
        self.used -= st.bytes
        self.spills += 1

    def can_admit(self, req):
        if req.kind == "probe" and self.table_busy[req.material]:
            return False
        return self._evict_for(self._job_bytes(req))

    # -- work ----------------------------------------------------------------
    def _state(self, req, stream):
        """The table bitmaps of the job's slice on the device, valid on
        `stream` (computed on first use, read back after a spill)."""
        torch, tbg = self.torch, self.tbg
        key = (req.material, req.slice)
        mp = self.mpools[req.material]
        st = self.states.get(key)
        if st is None:
            st = self.states[key] = _State(bytes=2 * mp.m.bytes + mp.m.sub_bytes)
        self.states.move_to_end(key)
        st.last_use = time.perf_counter()
        st.pins += 1
        if st.dev is None:
            z = lambda n: torch.empty(n, dtype=torch.uint8, device="cuda")
            st.dev = [z(mp.m.bytes), z(mp.m.bytes), z(mp.m.sub_bytes)]
            self.used += st.bytes
            if st.host is not None:
                for d, h in zip(st.dev, st.host):
                    d.copy_(h, non_blocking=True)
                self.reloads += 1
            else:
                mp.m.select()
                tbg.calc_illegal(req.slice, st.dev[0], st.dev[1])
                cls = [z(mp.m.sub_bytes) for _ in range(4)] + [st.dev[2]]
                tbg.calc_sub(WHITE, req.slice, cls)
                del cls
                self.builds += 1
            st.ready = torch.cuda.Event()
            st.ready.record(stream)
        else:
            stream.wait_event(st.ready)
        return key, st

    def issue(self, req, slot):
        torch, tbg = self.torch, self.tbg
        stream = self.streams[slot]
        tbg.set_stream(stream)
        job = _Job(req, torch.cuda.Event())
        try:
            with torch.cuda.stream(stream):
                if req.kind == "ply":
                    self._issue_ply(job, stream)
                else:
                    self._issue_probe(job, stream)
                job.event.record(stream)
        finally:
            # later library calls of the caller go to its own current stream
            tbg.set_stream(torch.cuda.current_stream())
        self.peak = max(self.peak, self.used)
        return job

    def _issue_ply(self, job, stream):
        from tb8gen_b200.plyjob import bern_threshold, king_slices, tag

        torch, tbg = self.torch, self.tbg
        req = job.req
        mp = self.mpools[req.material]
        m, s = mp.m, req.slice
        job.state_key, st = self._state(req, stream)
        ill_w, ill_b, sub_win = st.dev
        B, N = m.bytes, m.size
        z = lambda: torch.empty(B, dtype=torch.uint8, device="cuda")
        L_prev, W_prev, T, X, wins = z(), z(), z(), z(), z()
        job.bufs = [L_prev, W_prev, T, X, wins]
        job.nbytes = 5 * B
        self.used += job.nbytes
        m.select()
        tbg.gen_bernoulli(L_prev, N, req.seed, tag(0, BLACK, s), bern_threshold(req.p))
        L_prev &= ~ill_b
        tbg.gen_bernoulli(W_prev, N, req.seed, tag(3, WHITE, s), bern_threshold(req.p))
        W_prev &= ~ill_w
        wk, bk = king_slices(WHITE, s), king_slices(BLACK, s)
        # W step (tb8gen.c:1028-1084): T = predecessors of L_prev, epilogue
        tbg.unbind_all()
        tbg.bind(-1, L_prev)
        tbg.bind(s, T)
        for t in wk:
            tbg.bind(t, mp.t_sink)
        tbg.clear(s)
        tbg.predecessors(WHITE, s)
        tbg.unbind_all()
        tbg.bind(s, T)
        tbg.epilogue_W_to(s, ill_w, wins, count=False)
        # L step (tb8gen.c:943-1026): candidates from W_prev, verify
        tbg.unbind_all()
        tbg.bind(-1, W_prev)
        tbg.bind(s, X)
        for t in bk:
            tbg.bind(t, mp.x_sink)
        tbg.clear(s)
        tbg.predecessors(BLACK, s)
        tbg.unbind_all()
        tbg.bind(-1, X)
        tbg.bind(s, wins)
        tbg.bind_sub(s, sub_win)
        for t in bk:
            tbg.bind(t, mp.wins_nbr)
            tbg.bind_sub(t, mp.sub_nbr)
        tbg.check_successors(BLACK, s)
        tbg.unbind_all()
        # the response: W(s) and L(s) to pinned host memory
        out = [torch.empty(B, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        out[0].copy_(T, non_blocking=True)
        out[1].copy_(X, non_blocking=True)
        job.out = out

    def _issue_probe(self, job, stream):
        torch = self.torch
        req = job.req
        t = self.tables[req.material]
        self.table_busy[req.material] = True
        qb = self.qb
        host = self.qpool[req.material][req.offset * qb:(req.offset + req.n) * qb]
        q = torch.empty(req.n * qb, dtype=torch.uint8, device="cuda")
        out = torch.empty(req.n, dtype=torch.int8, device="cuda")
        job.bufs = [q, out]
        job.nbytes = req.n * (qb + 1)
        self.used += job.nbytes
        q.copy_(host, non_blocking=True)
        if qb == 8:
            t.probe8(q, out, 0)
        else:
            t.probe(q, out, 0)
        res = torch.empty(req.n, dtype=torch.int8, pin_memory=True)
        res.copy_(out, non_blocking=True)
        job.out = [res]

    def done(self, job):
        return job.event.query()

    def finish(self, job):
        req = job.req
        if req.kind == "probe":
            self.table_busy[req.material] = False
        else:
            self.states[job.state_key].pins -= 1
        self.used -= job.nbytes
        job.bufs = []
        if not self.keep:
            return None
        if req.kind == "probe":
            return job.out[0].numpy().copy()
        return tuple(o.numpy().copy() for o in job.out)


def run_alone(executor, requests):
    """Each request on its own (one slot, nothing else in flight), arrivals
    ignored: the reference results for the same-result check."""
    sch = Scheduler(executor, 1)
    out = {}
    for r in requests:
        r0 = Request(**{**r.__dict__, "arrival": 0.0})
        recs, _ = sch.run([r0])
        out[r.rid] = recs[0].result
    return out
