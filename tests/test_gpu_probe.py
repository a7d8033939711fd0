"""GPU table probes (tbg_table_build on the device, tbg_probe_wdl_batch,
tbg_encode_batch, tbg_decode_batch, tbg_gen_positions) against the
reference's own reader and probe (probe_table, encode_piece, decode_piece of
probe.c, compiled in place): the device-built table is byte-identical to the
host-built one, and every probed value equals the reference's probe of the
same table file.  Grouped (block-at-a-time) and direct (per-position)
probes must agree bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import probe_ref as PR

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not PR.probe_available(), reason="libtbprobe.so not built")]


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tb8gen_b200 as tb
    tb.init()
    return torch, tb


def _to_host(torch, tb, addr: int, nbytes: int) -> bytes:
    """Device bytes at a raw address (a table tbg_table_build allocated)."""
    return _tensor_from_ptr(torch, addr, nbytes).cpu().numpy().tobytes()


def _tensor_from_ptr(torch, addr: int, nbytes: int):
    class _Arr:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (addr, False),
                                    "version": 3}
    return torch.as_tensor(_Arr(), device="cuda")


SMALL = [("KRvK", 11, 3), ("KRRvK", 5, 3), ("KRvKR", 7, 5), ("KQvKR", 3, 3)]


@pytest.mark.parametrize("material,seed,modulus", SMALL)
def test_device_build_equals_host_build(env, material, seed, modulus):
    torch, tb = env
    host = tb.table_build_host(material, seed, modulus)
    with tb.DeviceTable(material, seed, modulus) as t:
        assert t.bytes == len(host)
        dev = _to_host(torch, tb, t.addr, t.bytes)
    assert dev == host


def _queries(torch, material, n, seed):
    q = PR.random_queries(material, n, seed)
    return q, torch.from_numpy(q.reshape(-1)).cuda()


@pytest.mark.parametrize("material,seed,modulus", SMALL)
def test_probe_matches_reference(env, tmp_path, material, seed, modulus):
    torch, tb = env
    host = tb.table_build_host(material, seed, modulus)
    (tmp_path / (PR.table_file_name(material) + ".rtbw")).write_bytes(host)
    ref = PR.RefProbe(str(tmp_path))
    q, dq = _queries(torch, material, 4000, seed + 1)
    want = ref.probe(material, q)
    with tb.DeviceTable(material, seed, modulus) as t:
        for mode in (0, 1):
            out = torch.full((len(q),), 99, dtype=torch.int8, device="cuda")
            t.probe(dq, out, mode)
            np.testing.assert_array_equal(out.cpu().numpy(), want, err_msg=f"mode {mode}")
        idx = torch.zeros(len(q), dtype=torch.int64, device="cuda")
        side = torch.zeros(len(q), dtype=torch.uint8, device="cuda")
        t.encode(dq, idx, side)
        ridx, rside = ref.encode(material, q)
        np.testing.assert_array_equal(idx.cpu().numpy().view(np.uint64), ridx)
        np.testing.assert_array_equal(side.cpu().numpy(), rside)
        for b in (0, 1) if rside.any() else (0,):
            sel = ridx[rside == b]
            dsel = torch.from_numpy(sel.view(np.int64)).cuda()
            sq = torch.zeros((len(sel), 8), dtype=torch.uint8, device="cuda")
            t.decode(b, dsel, sq)
            np.testing.assert_array_equal(sq.cpu().numpy(), ref.decode(material, b, sel))


def test_larger_table_probe_and_blocks(env, tmp_path):
    """A 5-piece table of 1,750 blocks per side, probed by 2^20 queries
    (every block touched many times): device table read by the reference,
    grouped == direct == reference on a sample."""
    torch, tb = env
    material, seed, modulus = "KQRvKR", 9, 3
    with tb.DeviceTable(material, seed, modulus) as t:
        img = _to_host(torch, tb, t.addr, t.bytes)
        (tmp_path / (PR.table_file_name(material) + ".rtbw")).write_bytes(img)
        ref = PR.RefProbe(str(tmp_path))
        n = 1 << 20
        dq = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
        assert tb.gen_positions(material, 3, dq) == 0
        a = torch.zeros(n, dtype=torch.int8, device="cuda")
        b = torch.zeros(n, dtype=torch.int8, device="cuda")
        t.probe(dq, a, 0)
        t.probe(dq, b, 1)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
        q = dq.cpu().numpy().reshape(n, 16)
        pick = np.random.default_rng(0).choice(n, 20000, replace=False)
        np.testing.assert_array_equal(a.cpu().numpy()[pick], ref.probe(material, q[pick]))
        # the values follow the table's formula at the reference's index
        idx, side = ref.encode(material, q[pick])
        np.testing.assert_array_equal(a.cpu().numpy()[pick], PR.table_wdl(seed, modulus, idx, side))


def test_gen_positions(env):
    torch, tb = env
    n = 100000
    a = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    b = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    assert tb.gen_positions("KRRRvKRR", 3, a) == 0
    assert tb.gen_positions("KRRRvKRR", 3, b) == 0
    assert torch.equal(a, b)
    q = a.cpu().numpy().reshape(n, 16)
    sq = q[:, :7].astype(np.int64)
    assert (sq < 64).all() and (q[:, 7] == 0).all() and (q[:, 8] <= 1).all()
    assert all(len(set(r)) == 7 for r in sq[:2000])
    kd = np.maximum(abs(sq[:, 0] % 8 - sq[:, 1] % 8), abs(sq[:, 0] // 8 - sq[:, 1] // 8))
    assert (kd > 1).all()
    assert 0.4 < q[:, 8].mean() < 0.6


def test_invalid_queries(env):
    torch, tb = env
    with tb.DeviceTable("KRRvK", 5, 3) as t:
        q = PR.random_queries("KRRvK", 4, 1)
        q[0, 1] = q[0, 0]                     # two pieces on one square
        wk = int(q[1, 0])
        q[1, 1] = wk + 1 if wk % 8 < 7 else wk - 1   # kings adjacent (kk table)
        q[2, 3] = 64                          # off the board
        q[3, 8] = 2                           # bad side to move
        dq = torch.from_numpy(q.reshape(-1)).cuda()
        for mode in (0, 1):
            out = torch.zeros(4, dtype=torch.int8, device="cuda")
            t.probe(dq, out, mode)
            assert (out.cpu().numpy() == -128).all()


@pytest.mark.parametrize("material,seed,modulus", SMALL[:2] + [("KQRvKR", 9, 3)])
def test_block_stream_starts(env, material, seed, modulus):
    """The stream start of every block, found once at open (the decoders'
    zero-padding scan: the first nonzero 32-bit word, at most 8 bytes before
    the block's end), against the same scan over the host-built image."""
    torch, tb = env
    host = np.frombuffer(tb.table_build_host(material, seed, modulus), dtype=np.uint8)
    with tb.DeviceTable(material, seed, modulus) as t:
        for side in (0, 1):
            try:
                off, nb, _ = t.layout(side)
            except tb.TbgError:
                break
            words = host[off: off + nb * 65536].view(np.uint32).reshape(nb, 16384)
            nz = words != 0
            first = np.where(nz.any(axis=1), nz.argmax(axis=1), 16382)
            first = np.minimum(first, 16382)
            assert t.stream_bytes(side) == int((65536 - 4 * first.astype(np.int64)).sum())


def test_misaligned_queries_refused(env):
    """Query arrays must start on a 16-byte boundary (each query is read as
    one vector): a misaligned array is refused before any launch."""
    torch, tb = env
    with tb.DeviceTable("KRRvK", 5, 3) as t:
        q = PR.random_queries("KRRvK", 8, 1)
        buf = torch.zeros(q.size + 16, dtype=torch.uint8, device="cuda")
        view = buf[1: 1 + q.size]
        out = torch.zeros(8, dtype=torch.int8, device="cuda")
        with pytest.raises(tb.TbgError):
            t.probe(view, out, 0)
        idx = torch.zeros(8, dtype=torch.int64, device="cuda")
        side = torch.zeros(8, dtype=torch.uint8, device="cuda")
        with pytest.raises(tb.TbgError):
            t.encode(view, idx, side)


def test_compact_queries(env, tmp_path):
    """8-byte queries (squares 0-6, side to move in byte 7) give the same
    values as the 16-byte ones, grouped and direct, invalid ones included."""
    torch, tb = env
    material, seed, modulus = "KQRvKR", 9, 3
    with tb.DeviceTable(material, seed, modulus) as t:
        n = 1 << 18
        dq = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
        assert tb.gen_positions(material, 5, dq) == 0
        dq.view(n, 16)[:64, 1] = dq.view(n, 16)[:64, 0]   # a few invalid ones
        q8 = tb.compact_queries(dq)
        assert q8.numel() == n * 8
        for mode in (0, 1):
            a = torch.zeros(n, dtype=torch.int8, device="cuda")
            b = torch.ones(n, dtype=torch.int8, device="cuda")
            t.probe(dq, a, mode)
            t.probe8(q8, b, mode)
            torch.cuda.synchronize()
            assert torch.equal(a, b), f"mode {mode}"
        assert (a[:64] == -128).all()
