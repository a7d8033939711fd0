"""The serving loop on the GPU (tb8gen_b200.serve): a seeded Poisson stream
of ply jobs and probe batches served with continuous batching (several
requests in flight on separate streams) under an admission budget small
enough to force spills of the resident slice bitmaps to pinned host
memory.  Every request's result (the W and L bitmaps of a ply job, the WDL
values of a probe batch) must be the same as when it runs alone."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PLY = ["KRRvKR", "KQRvKR"]
PROBE = ["KQRvKR", "KRRvK"]
POOL = 1 << 16
PROBE_MAX = 4000


@pytest.fixture(scope="module")
def server():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tbg
    from tb8gen_b200.serve import GpuExecutor

    tbg.init()
    tbg.set_stub(1)
    tables, pools = {}, {}
    for m in PROBE:
        tables[m] = tbg.DeviceTable(m, 3, 3)
        q = torch.empty(POOL * 16, dtype=torch.uint8, device="cuda")
        assert tbg.gen_positions(m, 3, q) == 0
        pools[m] = q.cpu().pin_memory()
    ex = GpuExecutor(PLY, tables, pools, slots=4, budget_bytes=1 << 40, keep_results=True,
                     probe_max=PROBE_MAX)
    yield torch, tbg, ex
    for t in tables.values():
        t.close()


def _requests():
    from tb8gen_b200.serve import make_requests

    return make_requests(48, 3000.0, PLY, PROBE, seed=4, probe_min=1000, probe_max=PROBE_MAX,
                         pool_n=POOL)


def test_results_same_alone_and_in_mix(server):
    torch, tbg, ex = server
    from tb8gen_b200.serve import Scheduler, run_alone, summarize

    reqs = _requests()
    alone = run_alone(ex, reqs)
    # room for the tables and pools, the in-flight jobs and about 3 resident
    # slice states: the mix must spill and read back
    one = max(2 * p.m.bytes + p.m.sub_bytes for p in ex.mpools.values())
    job = max(5 * p.m.bytes for p in ex.mpools.values())
    resident = sum(st.bytes for st in ex.states.values() if st.dev is not None)
    ex.budget = ex.used - resident + 3 * one + 4 * job + 2 * PROBE_MAX * 17
    spills0, reloads0 = ex.spills, ex.reloads
    recs, makespan = Scheduler(ex, 4).run(reqs)
    assert len(recs) == len(reqs)
    assert ex.spills > spills0 and ex.reloads > reloads0
    assert ex.peak >= ex.used
    overlapped = 0
    by_fin = sorted(recs, key=lambda r: r.admitted)
    for a, b in zip(by_fin, by_fin[1:]):
        overlapped += b.admitted < a.finished
    assert overlapped > 0, "no request was admitted while another ran"
    for r in recs:
        want = alone[r.rid]
        if r.kind == "probe":
            np.testing.assert_array_equal(r.result, want)
            assert (r.result != -128).all()
        else:
            assert np.array_equal(r.result[0], want[0]) and np.array_equal(r.result[1], want[1])
    s = summarize(recs, makespan)
    assert s["jobs"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0


def test_probe_results_match_direct_probe(server):
    """A served probe batch equals the per-position probe of the same table."""
    torch, tbg, ex = server
    from tb8gen_b200.serve import Request, Scheduler

    req = Request(0, 0.0, "probe", "KQRvKR", n=5000, offset=123)
    recs, _ = Scheduler(ex, 2).run([req])
    q = ex.qpool["KQRvKR"][123 * 16:(123 + 5000) * 16].cuda()
    out = torch.empty(5000, dtype=torch.int8, device="cuda")
    ex.tables["KQRvKR"].probe(q, out, 1)
    np.testing.assert_array_equal(recs[0].result, out.cpu().numpy())


def test_compact_probe_requests(server):
    """An executor fed 8-byte compact queries answers a probe batch like the
    16-byte per-position probe of the same positions."""
    torch, tbg, ex = server
    from tb8gen_b200.serve import GpuExecutor, Request, Scheduler

    pools8 = {m: tbg.compact_queries(p.cuda()).cpu().pin_memory() for m, p in ex.qpool.items()}
    ex8 = GpuExecutor([], ex.tables, pools8, slots=2, budget_bytes=1 << 40, keep_results=True,
                      probe_max=PROBE_MAX, query_bytes=8)
    req = Request(0, 0.0, "probe", "KQRvKR", n=3000, offset=77)
    recs, _ = Scheduler(ex8, 2).run([req])
    q = ex.qpool["KQRvKR"][77 * 16:(77 + 3000) * 16].cuda()
    out = torch.empty(3000, dtype=torch.int8, device="cuda")
    ex.tables["KQRvKR"].probe(q, out, 1)
    np.testing.assert_array_equal(recs[0].result, out.cpu().numpy())
