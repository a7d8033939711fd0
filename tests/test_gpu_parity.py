"""Bit-exact parity of the CUDA ply step with the CPU oracles.

Every worker runs through the C ABI (libtbgpu.so) and through the oracle on
the same seeded inputs; the outputs must be identical byte for byte.  Where
the reference-worker harness (oracle/_ref/libtbref.so) is present it is the
oracle; otherwise the C restatement (oracle/liboracle.so), itself pinned to
the reference by tests/test_oracle_pin.py.

Slices cover the ordinary case (96: wK c1, bK e6), the a1/b1 corner (0), the
far end of the off-diagonal range (440) and the diagonal slices (441..461),
where the reference marks both mirror images (tb8gen.c:257-260).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.parity import GpuSide, OracleSide, diff_report, verify_inputs

pytestmark = pytest.mark.gpu

SLICES = [0, 96, 300, 440, 441, 452, 461]


def oracle_for(material):
    if orc.ref_available():
        return OracleSide(orc.Ref(material, 8))
    return OracleSide(orc.Port(material))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR", "KNBvKB"])
def test_predecessors(torch_cuda, material):
    G, O = GpuSide(material), oracle_for(material)
    for s in SLICES:
        for stm in (0, 1):
            for p in (0.01, 0.2):
                src = orc.gen_bitmap(G.size, G.bytes, 11, orc.bitmap_tag(0, stm ^ 1, s), p)
                a, b = G.predecessors(stm, s, src), O.predecessors(stm, s, src)
                assert a.keys() == b.keys()
                rep = diff_report(a, b)
                assert not rep, f"{material} stm={stm} s={s} p={p}: {rep}"


@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR", "KBBvKN"])
def test_check_successors(torch_cuda, material):
    G, O = GpuSide(material), oracle_for(material)
    G.set_stub(7)
    O.set_stub(7)
    for s in SLICES:
        for stm in (0, 1):
            for wins_p in (0.6, 0.98):
                cand, wins, subs = verify_inputs(O, stm, s, 0.3, wins_p)
                a = G.check_successors(stm, s, cand, wins, subs)
                b = O.check_successors(stm, s, cand, wins, subs)
                assert np.array_equal(a, b), (
                    f"{material} stm={stm} s={s} wins_p={wins_p}: "
                    f"{int((a != b).sum())} bytes differ")


@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR"])
def test_predecessors_sub(torch_cuda, material):
    G, O = GpuSide(material), oracle_for(material)
    for s in SLICES:
        for stm in (0, 1):
            for legality in (False, True):
                sub = orc.gen_bitmap(G.sub_bytes * 8, G.sub_bytes, 5,
                                     orc.bitmap_tag(2, stm ^ 1, s), 0.1)
                a = G.predecessors_sub(stm, s, legality, sub)
                b = O.predecessors_sub(stm, s, legality, sub)
                rep = diff_report(a, b)
                assert not rep, f"{material} stm={stm} s={s} legality={legality}: {rep}"


@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR", "KRvKNN", "KRvKNNN"])
@pytest.mark.parametrize("modulus", [3, 5])
def test_calc_sub(torch_cuda, material, modulus):
    G, O = GpuSide(material), oracle_for(material)
    G.set_stub(1234, modulus)
    O.set_stub(1234, modulus)
    for s in SLICES:
        for stm in (0, 1):
            a, b = G.calc_sub(stm, s), O.calc_sub(stm, s)
            for i in range(5):
                assert np.array_equal(a[i], b[i]), f"{material} s={s} stm={stm} class {i}"


# KRRRvK: one set, so a slice is a single row of the walk over consecutive
# indices; KRvKNNN: a three-piece last set (carries across its squares).
@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR", "KNBvKB", "KRRRvK", "KRvKNNN"])
def test_illegal_and_mate(torch_cuda, material):
    G, O = GpuSide(material), oracle_for(material)
    for s in SLICES:
        ga, oa = G.calc_illegal(s), O.calc_illegal(s)
        assert np.array_equal(ga[0], oa[0]) and np.array_equal(ga[1], oa[1]), f"illegal s={s}"
        gm, om = G.calc_mate(s, *oa), O.calc_mate(s, *oa)
        assert np.array_equal(gm[0], om[0]) and np.array_equal(gm[1], om[1]), f"mate s={s}"


def test_epilogue(torch_cuda):
    G, O = GpuSide("KQRvKRR"), oracle_for("KQRvKRR")
    for seed in range(3):
        T = orc.gen_bitmap(G.size, G.bytes, seed, 1, 0.3)
        W = orc.gen_bitmap(G.size, G.bytes, seed, 2, 0.4)
        # garbage in the padding bits must be carried like the reference does
        T[-8:] = 0xFF
        ca, ta, wa = G.epilogue_W(T, W)
        cb, tb, wb = O.epilogue_W(T, W)
        assert ca == cb and np.array_equal(ta, tb) and np.array_equal(wa, wb)


def test_attacks_exhaustive(torch_cuda):
    """Rook and bishop attacks for every square and every subset of the
    relevant occupancy mask, knight/king for every square, against the
    reference's magic tables (magic.h:23-38) or the restatement."""
    import tb8gen_b200 as tbg

    torch = torch_cuda
    tbg.init()
    use_ref = orc.ref_available()
    if use_ref:
        orc.Ref("KRvK", 8)  # initialises the reference's magic tables
    L = orc.ref_lib() if use_ref else orc.port_lib()
    for ptype, name in ((4, "rook"), (3, "bishop")):
        sqs, occs = [], []
        for sq in range(64):
            mask = (orc.port_lib().orc_rook_attacks(sq, 0) if ptype == 4
                    else orc.port_lib().orc_bishop_attacks(sq, 0))
            # relevant occupancy: the rays without their end squares, plus
            # random far squares (ignored by sliding attacks)
            bits = [b for b in range(64) if mask >> b & 1]
            n = len(bits)
            for sub in range(1 << min(n, 12)):
                o = 0
                for j, b in enumerate(bits[:12]):
                    if sub >> j & 1:
                        o |= 1 << b
                sqs.append(sq)
                occs.append(o)
        sq_t = torch.tensor(sqs, dtype=torch.uint8, device="cuda")
        occ_np = np.array(occs, dtype=np.uint64)
        occ_t = torch.from_numpy(occ_np.view(np.int64)).cuda()
        out = torch.zeros(len(sqs), dtype=torch.int64, device="cuda")
        tbg.attacks(ptype, sq_t, occ_t, out)
        tbg.sync()
        got = out.cpu().numpy().view(np.uint64)
        f = (L.ref_rook_attacks if ptype == 4 else L.ref_bishop_attacks) if use_ref else \
            (L.orc_rook_attacks if ptype == 4 else L.orc_bishop_attacks)
        want = np.array([f(int(s), int(o)) for s, o in zip(sqs, occs)], dtype=np.uint64)
        assert np.array_equal(got, want), f"{name} attacks differ"


@pytest.mark.parametrize("stm", [0, 1])
def test_full_size_krrrvkrrr_low_density(torch_cuda, stm):
    """KRRRvKRRR at full slice size (1.23e9 positions) with a
    sparse source, so that the single-threaded oracle finishes quickly."""
    material, s = "KRRRvKRRR", 96
    G, O = GpuSide(material), OracleSide(orc.Port(material))
    src = orc.gen_bitmap(G.size, G.bytes, 1, orc.bitmap_tag(0, stm ^ 1, s), 2e-5)
    a, b = G.predecessors(stm, s, src), O.predecessors(stm, s, src)
    rep = diff_report(a, b)
    assert not rep, rep
