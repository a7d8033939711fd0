"""The synthetic WDL table writer (tbg_table_build, host build) against the
reference's own reader: the table file the engine writes is mapped by the
reference's init_tablebases/init_table (probe.c:258, 1210-1344) and probed with
its probe_table (probe.c:1522-1597); every probed value must be the table's
defining formula at the index the reference's encode_piece computes.  The
frequency-table bytes are compared with the reference's write_freq_table
(rans.c:239-276) for the same histogram.  CPU only."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import probe_ref as PR

pytestmark = pytest.mark.skipif(not PR.probe_available(), reason="oracle/_ref/libtbprobe.so not built")

BLOCK = 65536


def _tb():
    import tb8gen_b200 as tb
    return tb


def _side_quads(seed: int, modulus: int, size: int, bside: int) -> np.ndarray:
    """Quad value codes of one side, the last block front-padded with zeros."""
    v = PR.table_wdl(seed, modulus, np.arange(size, dtype=np.uint64),
                     np.full(size, bside, dtype=np.uint64)).astype(np.int64)
    v = (v + 2) if modulus == 5 else (v + 2) // 2
    nb = (size + BLOCK - 1) // BLOCK
    last = size - (nb - 1) * BLOCK
    pad = (4 - last % 4) % 4
    v = np.concatenate([v[: (nb - 1) * BLOCK], np.zeros(pad, np.int64), v[(nb - 1) * BLOCK:]])
    q = v.reshape(-1, 4)
    M = modulus
    return ((q[:, 0] * M + q[:, 1]) * M + q[:, 2]) * M + q[:, 3]


def _parse(table: bytes, material: str):
    """Offsets of the header fields (init_table's walk, pawnless WDL)."""
    n = len(PR.material_pieces(material))
    split = table[4] & 1
    o = 5 + n + 1
    o += o & 1
    return split, o


CASES = [
    ("KRvK", 11, 3, 31332),        # 3 unique pieces: triangle encoding, split
    ("KRRvK", 5, 3, 873642),       # kk encoding, last block padded by 2
    ("KRvKR", 7, 5, 31332 * 61),   # symmetric (one side), modulus 5
    ("KQvKR", 3, 3, 31332 * 61),
]


@pytest.mark.parametrize("material,seed,modulus,size", CASES)
def test_reference_reads_engine_table(tmp_path, material, seed, modulus, size):
    tb = _tb()
    table = tb.table_build_host(material, seed, modulus)
    (tmp_path / (PR.table_file_name(material) + ".rtbw")).write_bytes(table)
    ref = PR.RefProbe(str(tmp_path))
    assert ref.found == 1
    q = PR.random_queries(material, 3000, seed=seed + 100)
    idx, side = ref.encode(material, q)
    assert int(idx.max()) < size
    got = ref.probe(material, q)
    want = PR.table_wdl(seed, modulus, idx, side)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("material,seed,modulus,size", CASES)
def test_freq_table_matches_reference_writer(material, seed, modulus, size):
    tb = _tb()
    table = tb.table_build_host(material, seed, modulus)
    split, o = _parse(table, material)
    M = modulus
    nsyms = M + M * M + M ** 4
    for bside in range(2 if split else 1):
        hist = np.bincount(_side_quads(seed, modulus, size, bside), minlength=M ** 4)
        freq = np.zeros(nsyms, np.int64)
        freq[M + M * M:] = hist
        ref = PR.ref_code(freq)
        assert table[o] == 0x40 and table[o + 1] == 16 and table[o + 2] == 16
        nblocks = int.from_bytes(table[o + 4: o + 8], "little")
        assert nblocks == (size + BLOCK - 1) // BLOCK
        ft = ref["ftab"]
        assert table[o + 10: o + 10 + len(ft)] == ft
        # the reference's reader recovers the sorted frequencies
        back = PR.ref_read_code(table[o + 10:])
        assert back["num"] == nsyms
        np.testing.assert_array_equal(back["freq"], ref["freq"])
        o += 10 + len(ft) + 3 * nsyms + (nsyms & 1)


@pytest.mark.parametrize("material,seed,modulus,size", CASES[:3])
def test_reference_decode_round_trip(tmp_path, material, seed, modulus, size):
    """decode_piece (through the harness's set_dec_info) inverts encode_piece:
    pins the checker used by the GPU decode tests."""
    tb = _tb()
    (tmp_path / (PR.table_file_name(material) + ".rtbw")).write_bytes(
        tb.table_build_host(material, seed, modulus))
    ref = PR.RefProbe(str(tmp_path))
    q = PR.random_queries(material, 500, seed=seed)
    q[:, 8] = 0                          # white to move: side 0, no flip
    idx, side = ref.encode(material, q)
    assert not side.any()
    sq = ref.decode(material, 0, idx)
    # table order -> material order by piece type
    pt = PR.material_pieces(material)
    table_pt = _table_order(material)
    back = np.zeros_like(q)
    for r in range(len(q)):
        used = [False] * len(pt)
        for t, s in zip(table_pt, sq[r, : len(pt)]):
            j = next(j for j in range(len(pt)) if pt[j] == t and not used[j])
            used[j] = True
            back[r, j] = s
    idx2, _ = ref.encode(material, back)
    np.testing.assert_array_equal(idx2, idx)


def _table_order(material: str) -> list[int]:
    """The engine's table piece order: kings, then (unless only the kings are
    unique) the first unique other piece, then the rest in material order."""
    pt = PR.material_pieces(material)
    cnt = {p: pt.count(p) for p in pt}
    rest = pt[2:]
    out = pt[:2]
    if sum(1 for p in cnt if cnt[p] == 1) > 2:
        u = next(p for p in rest if cnt[p] == 1)
        out.append(u)
        rest = list(rest)
        rest.remove(u)
    return out + rest


def test_bad_material_rejected():
    tb = _tb()
    with pytest.raises(tb.TbgError):
        tb.table_build_host("KPvK", 1, 3)
    with pytest.raises(tb.TbgError):
        tb.table_build_host("KRvK", 1, 4)
