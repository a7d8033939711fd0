"""Pins the C restatement's tables and index functions against the
reference itself (oracle/_ref/libtbref.so), exhaustively where the domain is
small: king-pair tables, slice schedule, attack sets, index round trips."""
import numpy as np
import pytest

from oracle import oracle as orc

needs_ref = pytest.mark.skipif(not orc.ref_available(), reason="reference harness not built")


@pytest.fixture(scope="module")
def ref():
    return orc.Ref("KRRvKR", 4)


@needs_ref
def test_king_tables(ref):
    P, R = orc.port_lib(), orc.ref_lib()
    for t in range(10):
        for sq in range(64):
            assert P.orc_kkidx(t, sq) == R.ref_kkidx(t, sq)
    for a in range(64):
        for b in range(64):
            assert P.orc_kkmap(a, b) == R.ref_kkmap(a, b)
            assert P.orc_fliptest(a, b) == R.ref_fliptest(a, b)
    for s in range(462):
        assert P.orc_kksquare(s, 0) == R.ref_kksquare(s, 0)
        assert P.orc_kksquare(s, 1) == R.ref_kksquare(s, 1)


@needs_ref
def test_manager_schedule(ref):
    P, R = orc.port_lib(), orc.ref_lib()
    a_in, a_out = np.zeros(11, np.int16), np.zeros(11, np.int16)
    b_in, b_out = np.zeros(11, np.int16), np.zeros(11, np.int16)
    for stm in (0, 1):
        for i in range(462):
            ka = P.orc_manager(stm, i, a_in.ctypes.data, a_out.ctypes.data)
            kb = R.ref_manager(stm, i, b_in.ctypes.data, b_out.ctypes.data)
            assert ka == kb
            n_in = list(b_in).index(-1) if -1 in list(b_in) else 11
            n_out = list(b_out).index(-1) if -1 in list(b_out) else 11
            assert list(a_in[:n_in + 1 if n_in < 11 else 11]) == list(b_in[:n_in + 1 if n_in < 11 else 11])
            assert list(a_out[:n_out + 1 if n_out < 11 else 11]) == list(b_out[:n_out + 1 if n_out < 11 else 11])


@needs_ref
def test_attacks_exhaustive(ref):
    P, R = orc.port_lib(), orc.ref_lib()
    rng = np.random.default_rng(0)
    for sq in range(64):
        for f_p, f_r in ((P.orc_rook_attacks, R.ref_rook_attacks),
                         (P.orc_bishop_attacks, R.ref_bishop_attacks)):
            mask = f_p(sq, 0)
            bits = [b for b in range(64) if mask >> b & 1]
            for sub in range(1 << len(bits)) if len(bits) <= 12 else rng.integers(0, 1 << len(bits), 4096):
                occ = 0
                for j, b in enumerate(bits):
                    if int(sub) >> j & 1:
                        occ |= 1 << b
                occ |= int(rng.integers(0, 1 << 62)) & ~mask & ~(1 << sq)
                assert f_p(sq, occ) == f_r(sq, occ)


@needs_ref
@pytest.mark.parametrize("material", ["KRRvKR", "KQRvKRR", "KRRRvK", "KNNvKBB"])
def test_index_round_trip(material):
    R, P = orc.Ref(material, 4), orc.Port(material)
    assert (R.size, R.bytes, R.sub_bytes) == (P.size, P.bytes, P.sub_bytes)
    rng = np.random.default_rng(1)
    for s in (0, 96, 441, 461):
        for k in [-1] + list(range(P.numsets)):
            n = P.size if k < 0 else P.capt_size(k)
            for idx in rng.integers(0, n, 300):
                a, occ_a = P.idx_to_sq(int(idx), s, k)
                b, occ_b = R.idx_to_sq(int(idx), s, k)
                assert occ_a == occ_b
                assert P.sq_to_idx(a, k) == int(idx) == R.sq_to_idx(b, k)
