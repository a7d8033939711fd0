"""The batched ply (tbg_batch_*): a recorded step of several slice-ply jobs
of two materials gives the same bitmaps through one launch per call
(mode 0) and through the persistent kernel (mode 1, block-wide work items,
and mode 2, one part of an item per warp; several grid sizes),
and each job's W, L and wins equal the reference's CPU workers on the same
inputs."""
import numpy as np
import pytest

from oracle import oracle as orc
from oracle.plyjob_cpu import CpuSlicePly

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tbg
    from tb8gen_b200.plyjob import MaterialPool, SlicePly, record_step

    tbg.init()
    tbg.set_stub(1)
    spec = [("KRRvKR", 96, 0.02), ("KQRvKRR", 300, 0.01), ("KRRvKR", 452, 0.05),
            ("KQRvKRR", 5, 0.03), ("KRRvKR", 441, 0.01)]
    pools, jobs = {}, []
    for mat, s, p in spec:
        if mat not in pools:
            pools[mat] = MaterialPool(mat, 7)
        jobs.append(SlicePly(mat, s, p, 7, pools[mat]))
    nops, nitems = record_step(jobs)
    return torch, tbg, jobs, pools, nops


def outputs(jobs, pools):
    out = [(j.T.cpu().numpy(), j.X.cpu().numpy(), j.wins.cpu().numpy()) for j in jobs]
    sinks = {m: (p.t_sink.cpu().numpy(), p.x_sink.cpu().numpy()) for m, p in pools.items()}
    return out, sinks


def run(torch, tbg, jobs, pools, mode, cps=2):
    for p in pools.values():
        p.t_sink.zero_()
        p.x_sink.zero_()
    for j in jobs:
        j.T.fill_(0xA5)
        j.X.fill_(0x5A)
        j.wins.zero_()
    tbg.batch_tune(cps)
    tbg.batch_run(mode)
    tbg.sync()
    return outputs(jobs, pools), tbg.batch_counts(len(jobs))


def test_persistent_equals_plain(setup):
    torch, tbg, jobs, pools, nops = setup
    (a, sa), ca = run(torch, tbg, jobs, pools, 0)
    for mode, cps in ((1, 1), (1, 2), (1, 4), (2, 1), (2, 2), (2, 4)):
        (b, sb), cb = run(torch, tbg, jobs, pools, mode, cps)
        assert ca == cb
        for x, y in zip(a, b):
            for u, v in zip(x, y):
                assert np.array_equal(u, v)
        for m in sa:
            assert np.array_equal(sa[m][0], sb[m][0]) and np.array_equal(sa[m][1], sb[m][1])


@pytest.mark.parametrize("mode", [1, 2])
def test_batch_matches_reference(setup, mode):
    torch, tbg, jobs, pools, nops = setup
    (b, _), counts = run(torch, tbg, jobs, pools, mode)
    for j, (T, X, W), c in zip(jobs, b, counts):
        O = orc.Ref(j.material, 8) if orc.ref_available() else orc.Port(j.material)
        O.set_stub(1)
        cpu = CpuSlicePly(O, j)
        cpu.step()
        assert c == cpu.cnt_w
        assert np.array_equal(T, cpu.T), f"W of {j.material} slice {j.s}"
        assert np.array_equal(W, cpu.wins), f"wins of {j.material} slice {j.s}"
        assert np.array_equal(X, cpu.X), f"L of {j.material} slice {j.s}"


def test_count_strided(setup):
    """tbg_count_strided: ones below the slice size in each of n bitmaps at a
    fixed stride (bits past the size and the gaps between bitmaps are not
    counted), equal to numpy's count."""
    torch, tbg, jobs, pools, nops = setup
    m = tbg.Material("KRRvKR").select()
    rng = np.random.default_rng(5)
    for n, gap in ((1, 0), (7, 0), (462, 48)):
        stride = m.bytes + gap
        host = rng.integers(0, 256, size=n * stride, dtype=np.uint8)
        dev = torch.from_numpy(host).cuda()
        want = 0
        for i in range(n):
            bits = np.unpackbits(host[i * stride:i * stride + m.bytes], bitorder="little")
            want += int(bits[:m.size].sum())
        assert tbg.count_strided(dev, stride, n) == want


def test_copy_tickets(setup):
    """Host-tier copies on the library's copy streams, ordered by tickets: a
    copy in, a kernel joined after it (a count), a copy out after the
    kernel's mark; a ticket 8192 tickets old is refused."""
    torch, tbg, jobs, pools, nops = setup
    m = tbg.Material("KRRvKR").select()
    rng = np.random.default_rng(11)
    host = torch.from_numpy(rng.integers(0, 256, size=m.bytes, dtype=np.uint8)).pin_memory()
    back = torch.zeros(m.bytes, dtype=torch.uint8).pin_memory()
    dev = torch.zeros(m.bytes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    first = tbg.mark()
    t_in = tbg.copy_in(dev, host, first, ticket=True)
    tbg.join(t_in)
    tbg.bind(0, dev)
    got = tbg.count(0)
    bits = np.unpackbits(host.numpy(), bitorder="little")[:m.size]
    assert got == int(bits.sum())
    mk = tbg.mark()
    t_out = tbg.copy_out(back, dev, mk, ticket=True)
    tbg.wait_ticket(t_out)
    assert torch.equal(back, host)
    for _ in range(8193):
        tbg.mark()
    with pytest.raises(tbg.TbgError):
        tbg.wait_ticket(first)
    tbg.unbind_all()


def test_batch_slots(setup):
    """Two batches recorded in two slots over different buffers keep their
    own queues: running slot 1 then slot 0 gives each job's results of its
    own buffers, equal to slot 0's results when the inputs are equal; a
    recorded count equals tbg_count of the same bitmap."""
    torch, tbg, jobs, pools, nops = setup
    (a, _), ca = run(torch, tbg, jobs, pools, 1)
    names = ("L_prev", "W_prev", "T", "X")
    orig = [tuple(getattr(j, n) for n in names) for j in jobs]
    alt = [(lp.clone(), wp.clone(), torch.zeros_like(t), torch.zeros_like(x))
           for lp, wp, t, x in orig]
    from tb8gen_b200.plyjob import record_step
    try:
        for j, bufs in zip(jobs, alt):
            for n, t in zip(names, bufs):
                setattr(j, n, t)
        tbg.batch_select(1)
        record_step(jobs)
        tbg.batch_run(1)
        tbg.sync()
        cb = tbg.batch_counts(len(jobs))
        tbg.batch_select(0)
        tbg.batch_run(1)
        tbg.sync()
        assert tbg.batch_counts(len(jobs)) == ca == cb
        for (t0, x0, _), (_, _, t1, x1) in zip(a, alt):
            assert np.array_equal(t0, t1.cpu().numpy()) and np.array_equal(x0, x1.cpu().numpy())
        # a recorded count of one job's L bitmap
        j = jobs[0]
        j.m.select()
        tbg.batch_select(2)
        tbg.batch_begin()
        tbg.bind(-1, alt[0][3])
        tbg.batch_count(-1)
        tbg.batch_end()
        tbg.batch_run(1)
        tbg.bind(0, alt[0][3])
        assert tbg.batch_counts(1)[0] == tbg.count(0)
    finally:
        tbg.batch_select(0)
        for j, bufs in zip(jobs, orig):
            for n, t in zip(names, bufs):
                setattr(j, n, t)
        tbg.unbind_all()


def test_item_shapes_do_not_change_results(setup):
    """Tiles per work item of the scatters and of the filtered candidates
    (tbg_batch_shape) re-cut the recorded batch; every shape, persistent and
    plain, gives the same bitmaps."""
    torch, tbg, jobs, pools, nops = setup
    try:
        tbg.batch_shape(1, 1)
        (a, sa), ca = run(torch, tbg, jobs, pools, 1, 4)
        for gw, gl in ((2, 4), (4, 8), (1, 16)):
            n = tbg.batch_shape(gw, gl)
            assert n > 0
            for mode in (1, 2, 0):
                (b, sb), cb = run(torch, tbg, jobs, pools, mode, 3)
                assert ca == cb
                for x, y in zip(a, b):
                    for u, v in zip(x, y):
                        assert np.array_equal(u, v)
    finally:
        tbg.batch_shape(0, 0)
