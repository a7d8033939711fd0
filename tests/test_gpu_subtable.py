"""Capture classification with the 7-piece values read from tables
(tbg_calc_sub_table): the classes computed by probing the tables of the
capture materials on the GPU (grouped rANS decode, mode 0) equal those from
the tables' defining formula (mode 1), and both equal the reference's own
calc_sub_worker (tb8gen.c:280-314) whose probe_wdl returns, for each capture
position, the value such a table stores at the reference's encode_piece
index of the position."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")]

CASES = [("KRRvKR", 1, 3), ("KQvKR", 7, 5), ("KRvKN", 3, 3), ("KRRvK", 2, 3)]
SLICES = [0, 96, 300, 441, 461]


def _sets(tb, material):
    """(set index, colour) of the material's like-piece sets in engine order."""
    pt = tb.material_pieces(material)[2:]
    out, k, i = [], 0, 0
    while i < len(pt):
        j = i
        while j < len(pt) and pt[j] == pt[i]:
            j += 1
        out.append((k, pt[i] >> 3))
        k += 1
        i = j
    return out


@pytest.mark.parametrize("material,seed,modulus", CASES)
def test_sub_through_tables(material, seed, modulus):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tb

    tb.init()
    m = tb.Material(material).select()
    sets = _sets(tb, material)
    tables = {}
    try:
        handles = {0: [-1] * 6, 1: [-1] * 6}
        for k, color in sets:
            name = tb.capture_material(k)
            if len(name.replace("v", "")) <= 2:
                continue  # the kings alone: a draw, no table
            if name not in tables:
                tables[name] = tb.DeviceTable(name, seed, modulus)
            handles[color][k] = tables[name].handle
        ref = orc.Ref(material, 8)
        ref.set_stub_table(seed, modulus)
        SB = m.sub_bytes
        for s in SLICES:
            for stm in (0, 1):
                m.select()
                got = []
                for mode in (0, 1):
                    cls = [torch.full((SB,), 0xA5, dtype=torch.uint8, device="cuda")
                           for _ in range(5)]
                    tb.calc_sub_table(stm, s, cls, handles[stm], mode, seed, modulus)
                    got.append([c.cpu().numpy() for c in cls])
                want = [np.full(SB, 0xA5, dtype=np.uint8) for _ in range(5)]
                ref.calc_sub(stm, s, want)
                for i in range(5):
                    assert np.array_equal(got[1][i], want[i]), \
                        f"{material} s={s} stm={stm} class {i}: formula vs reference"
                    assert np.array_equal(got[0][i], got[1][i]), \
                        f"{material} s={s} stm={stm} class {i}: tables vs formula"
    finally:
        for t in tables.values():
            t.close()
