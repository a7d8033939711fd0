"""Parity on the benchmarked configurations themselves, against the
reference's own code (oracle/_ref, compiled in place from the reference
sources):

* the KRRRvKRRR slice-ply the ply bench times (king slice 96, sources
  Bernoulli(0.01), seed 1; N = 1,229,490,380): W step, epilogue, L step and
  verify through the recorded batch, persistent and plain, equal to the
  reference's workers run on the same inputs and to the digests recorded
  from them (tests/golden/slice_ply.json);
* slices of the uneven mix's other two materials, KQRvKRRR and KQRRvKRR, at
  the mix's densities 0.001, 0.01 and 0.05, diagonal slices among them, with
  per-slice and with shared neighbour buffers, in one batch;
* the probe workload's tables, KRRRvKRR and KQRvKRR: 65,536 positions of
  each probed on the device and by the reference's probe_table
  (probe.c:1522-1597) reading the same table bytes.
"""
from __future__ import annotations

import os
import shutil
import tempfile

import numpy as np
import pytest

from oracle import oracle as orc
from oracle.plyjob_cpu import CpuSlicePly

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")]

CORES = os.cpu_count() or 1


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tbg

    tbg.init()
    tbg.set_stub(1, 3)
    return torch, tbg


def _diff(eng: dict, ref: dict) -> list:
    assert sorted(eng) == sorted(ref)
    return [k for k in sorted(eng) if not np.array_equal(eng[k].cpu().numpy(), ref[k])]


def test_bench_slice_ply_equals_reference(env):
    """The ply bench's KRRRvKRRR slice-ply, persistent and plain, equals the
    reference's workers on the same inputs and the recorded digests."""
    torch, tbg = env
    from bench import golden_slice
    from tb8gen_b200.plyjob import SlicePly, output_digests, record_step

    job = SlicePly("KRRRvKRRR", 96, 0.01, 1)
    record_step([job])
    try:
        tbg.batch_tune(4)
        tbg.batch_run(1)
        tbg.sync()
        eng1 = {k: v.clone() for k, v in job.outputs().items()}
        counts1 = list(job.counts())
        for mode in (0, 2):
            tbg.batch_run(mode)
            tbg.sync()
            assert list(job.counts()) == counts1
            assert _diff(job.outputs(), {k: v.cpu().numpy() for k, v in eng1.items()}) == []
        O = orc.Ref("KRRRvKRRR", CORES)
        O.set_stub(1, 3)
        cpu = CpuSlicePly(O, job, 1.0)
        cpu.step()
        assert counts1 == list(cpu.counts())
        assert _diff(eng1, cpu.outputs()) == []
        g = golden_slice("KRRRvKRRR", 96, 0.01, 1)
        assert g is not None, "tests/golden/slice_ply.json has no KRRRvKRRR/96 entry"
        assert counts1 == g["counts"]
        assert output_digests(eng1) == g["sha256"]
    finally:
        del job
        torch.cuda.empty_cache()


# (material, slice, p): slice 452 and 441 are diagonal slices (both kings on
# a1-h8), 0 a corner slice
MIX_CASES = [("KQRvKRRR", 17, 0.001), ("KQRvKRRR", 452, 0.01), ("KQRvKRRR", 230, 0.05),
             ("KQRRvKRR", 96, 0.05), ("KQRRvKRR", 441, 0.001), ("KQRRvKRR", 0, 0.01),
             ("KQRRvKRR", 460, 0.05)]


@pytest.mark.parametrize("shared,mode", [(False, 1), (True, 1), (True, 2)])
def test_mix_materials_equal_reference(env, shared, mode):
    """Slices of KQRvKRRR and KQRRvKRR at the mix densities, recorded in one
    batch and run by the persistent kernel, equal the reference's workers."""
    torch, tbg = env
    from tb8gen_b200.plyjob import MaterialPool, SlicePly, record_step

    pools, jobs = {}, []
    for mat, s, p in MIX_CASES:
        pool = None
        if shared:
            pools.setdefault(mat, MaterialPool(mat, 2))
            pool = pools[mat]
        jobs.append(SlicePly(mat, s, p, 2, pool))
    record_step(jobs)
    tbg.batch_tune(4)
    tbg.batch_run(mode)
    tbg.sync()
    counts = tbg.batch_counts(len(jobs))
    for j, c in zip(jobs, counts):
        O = orc.Ref(j.material, CORES)
        O.set_stub(1, 3)
        cpu = CpuSlicePly(O, j, 1.0)
        cpu.step()
        assert c == cpu.cnt_w, f"{j.material} slice {j.s}"
        bad = _diff(j.outputs(), cpu.outputs())
        assert bad == [], f"{j.material} slice {j.s} p={j.p}: {bad}"


@pytest.mark.parametrize("material", ["KRRRvKRR", "KQRvKRR"])
def test_probe_tables_equal_reference(env, material):
    """65,536 seeded legal positions of a probe-workload table: the device's
    grouped probe (compact and 16-byte queries) equals the reference's
    probe_table reading the same table bytes."""
    torch, tbg = env
    from oracle import probe_ref as PR

    if not PR.probe_available():
        pytest.skip("libtbprobe.so not built")
    import bench

    n = 1 << 16
    ps = bench.ProbeSet(n, materials=(material,))
    d = tempfile.mkdtemp(prefix="tbprobe_")
    try:
        ps.probe()
        tbg.sync()
        got8 = ps.items[0][3].cpu().numpy().copy()
        ps.probe16()
        tbg.sync()
        got16 = ps.items[0][3].cpu().numpy().copy()
        samples = bench.write_sparse_tables(ps, n, d)
        _, _, first = bench.time_reference_probe(d, samples, 0.0, CORES)
        want = first[material]
        assert len(want) == n
        assert np.array_equal(got8, want)
        assert np.array_equal(got16, want)
        assert int((want == -128).sum()) == 0
        m, t, q, _ = ps.items[0]
        assert bench.probe_roundtrip(m, t, q) == 0
    finally:
        shutil.rmtree(d, ignore_errors=True)
        ps.close()
        del ps
        torch.cuda.empty_cache()
