"""Failure paths, made on the host or by a bounded device wait that runs out
(no GPU is faulted, trapped or hung):

* the persistent kernel's dependency wait with an iteration limit of 1: the
  launch ends, tbg_sync reports TBG_ERR_DEVICE (the kernel's status word),
  and the next run with the normal limit is correct;
* tbg_sync with a 1 ms limit behind queued work returns TBG_ERR_TIMEOUT, and
  a later tbg_sync succeeds;
* an allocation refused on the host (TBG_FAIL_ALLOC_AT): tbg_alloc returns
  TBG_ERR_NOMEM and the C host driver exits nonzero with the library's
  message, as the reference exits on a failed allocation (util.c:111-115);
* bad job descriptors (side to move, slice, batch mode, slot, unbound
  scratch) are refused with a status, before any launch;
* the serving executor's pinned host tier refuses a spill beyond its budget
  (SpillError) on the CPU.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TBG_ERR_ARG, TBG_ERR_STATE, TBG_ERR_UNBOUND = -1, -2, -3
TBG_ERR_NOMEM, TBG_ERR_DEVICE, TBG_ERR_TIMEOUT = -5, -6, -7
DEFAULT_SPIN = 50_000_000


# ------------------------------------------------------------------ CPU
class _FakeState:
    def __init__(self, sizes):
        import torch

        self.dev = [torch.zeros(n, dtype=torch.uint8) for n in sizes]
        self.host = None
        self.ready = None
        self.bytes = sum(sizes)
        self.pins = 0


def test_spill_beyond_host_budget_raises():
    """GpuExecutor._spill refuses a state the pinned host tier cannot take,
    before any copy is queued."""
    import torch

    from tb8gen_b200.serve import GpuExecutor, SpillError

    ex = object.__new__(GpuExecutor)
    ex.torch = torch
    ex.host_budget = 1000
    ex.host_used = 600
    with pytest.raises(SpillError, match="pinned host tier full"):
        ex._spill(_FakeState([300, 200]))
    assert ex.host_used == 600


def test_host_tier_within_budget_counts_bytes():
    import torch

    from tb8gen_b200.serve import GpuExecutor, SpillError

    ex = object.__new__(GpuExecutor)
    ex.torch = torch
    ex.host_budget = 1000
    ex.host_used = 0
    if torch.cuda.is_available():
        bufs = ex._host_tier([100, 200])
        assert [b.numel() for b in bufs] == [100, 200] and ex.host_used == 300
    with pytest.raises(SpillError):
        ex._host_tier([2000])


def test_batch_slot_refused_without_gpu():
    import tb8gen_b200 as tbg

    L = tbg.lib()
    assert L.tbg_batch_select(-1) == TBG_ERR_ARG
    assert L.tbg_batch_select(4) == TBG_ERR_ARG
    assert L.tbg_batch_tune(0, 0) == TBG_ERR_ARG
    assert L.tbg_batch_tune(33, 0) == TBG_ERR_ARG


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tbg

    tbg.init()
    tbg.set_stub(1, 3)
    return torch, tbg


def _job(tbg):
    """One slice-ply of KRRRvKRR (8 MB bitmaps, 1,989 scatter tiles) recorded
    as a batch: W scatter, epilogue (waits for the scatter), L scatter,
    verify (waits for the L scatter and the epilogue)."""
    from tb8gen_b200.plyjob import SlicePly, record_step

    job = SlicePly("KRRRvKRR", 96, 0.02, 5)
    record_step([job])
    return job


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
def test_dependency_wait_runs_out(gpu, mode):
    torch, tbg = gpu
    job = _job(tbg)
    try:
        tbg.batch_tune(4, DEFAULT_SPIN)
        tbg.batch_run(mode)
        tbg.sync()
        want = {k: v.cpu().numpy().copy() for k, v in job.outputs().items()}
        failed = 0
        for _ in range(3):
            tbg.batch_tune(4, 1)
            job.T.fill_(0xA5)
            job.X.fill_(0x5A)
            tbg.batch_run(mode)
            with pytest.raises(tbg.TbgError) as ei:
                tbg.sync(20000)
            assert ei.value.code == TBG_ERR_DEVICE
            assert "status 3" in str(ei.value)
            failed += 1
        assert failed == 3
        # the status word is cleared, the next run with the normal limit is right
        tbg.batch_tune(4, DEFAULT_SPIN)
        tbg.batch_run(mode)
        tbg.sync()
        got = {k: v.cpu().numpy() for k, v in job.outputs().items()}
        assert all(np.array_equal(got[k], want[k]) for k in want)
    finally:
        tbg.batch_tune(4, DEFAULT_SPIN)
        del job
        torch.cuda.empty_cache()


@pytest.mark.gpu
def test_sync_timeout_then_success(gpu):
    torch, tbg = gpu
    job = _job(tbg)
    try:
        tbg.batch_tune(4, DEFAULT_SPIN)
        for _ in range(40):
            tbg.batch_run(0)          # one launch per call: ~160 launches queued
        with pytest.raises(tbg.TbgError) as ei:
            tbg.sync(1)
        assert ei.value.code == TBG_ERR_TIMEOUT
        tbg.sync(0)
    finally:
        del job
        torch.cuda.empty_cache()


@pytest.mark.gpu
def test_bad_descriptors_refused(gpu):
    import ctypes as C

    torch, tbg = gpu
    L = tbg.lib()
    m = tbg.Material("KRRvKR").select()
    tbg.unbind_all()
    n0 = tbg.launches()
    assert L.tbg_predecessors(2, 0) == TBG_ERR_ARG
    assert L.tbg_predecessors(0, 462) == TBG_ERR_ARG
    assert L.tbg_predecessors(0, -1) == TBG_ERR_ARG
    assert L.tbg_check_successors(1, 500) == TBG_ERR_ARG
    # targets bound but no scratch (source) slot
    dev = torch.zeros(m.bytes, dtype=torch.uint8, device="cuda")
    tbg.bind(96, dev)
    rc = L.tbg_predecessors(0, 96)
    assert rc in (TBG_ERR_UNBOUND,), rc
    assert L.tbg_batch_run(7) in (TBG_ERR_ARG, TBG_ERR_STATE)
    assert L.tbg_batch_begin() == 0
    assert L.tbg_batch_end(None, None) == TBG_ERR_ARG     # empty batch
    assert L.tbg_batch_run(1) == TBG_ERR_STATE            # nothing recorded
    nb = C.c_uint64()
    assert L.tbg_alloc(0, C.byref(C.c_void_p())) == TBG_ERR_ARG
    assert tbg.launches() == n0
    tbg.unbind_all()
    del nb


@pytest.mark.gpu
def test_alloc_failure_reported_by_tbgen(gpu):
    """The C host driver exits with the library's message when an
    allocation it cannot do without is refused; without the injection it
    runs to the end; where it has a fallback it takes it."""
    tbgen = os.path.join(ROOT, "tb8gen_b200", "tbgen")
    if not os.path.exists(tbgen):
        pytest.skip("tbgen not built")
    env = dict(os.environ, TBG_FAIL_ALLOC_AT="1")
    r = subprocess.run([tbgen, "KRvK"], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode != 0
    assert "refused (TBG_FAIL_ALLOC_AT)" in r.stderr
    env.pop("TBG_FAIL_ALLOC_AT")
    r0 = subprocess.run([tbgen, "KRvK"], capture_output=True, text=True, timeout=300, env=env)
    assert r0.returncode == 0, r0.stderr[-2000:]
    # streamed mode: a refused device "wins" plane (the first allocation)
    # falls back to the host tier, and the generation prints the same counts
    env["TBG_FAIL_ALLOC_AT"] = "1"
    r1 = subprocess.run([tbgen, "-S", "KRvK"], capture_output=True, text=True, timeout=300,
                        env=env)
    assert r1.returncode == 0, r1.stderr[-2000:]
    counts = lambda out: [l for l in out.splitlines() if " = " in l]
    assert counts(r1.stdout) == counts(r0.stdout) and counts(r0.stdout)
