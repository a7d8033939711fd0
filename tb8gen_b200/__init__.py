"""tb8gen_b200: B200 engine for the per-king-slice ply step of tb8gen.

The product is the C-ABI library ``libtbgpu.so`` (``include/tbgpu.h``), built
in-tree from ``csrc/`` for sm_100a.  This module loads it with ctypes and
mirrors its entry points for Python callers (tests, bench, the serving
loop).  There is no CPU fallback: if the library is missing, importing
``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# TBGPU_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = os.environ.get("TBGPU_LIB") or os.path.join(HERE, "libtbgpu.so")

STATUS = {
    0: "TBG_OK", -1: "TBG_ERR_ARG", -2: "TBG_ERR_STATE", -3: "TBG_ERR_UNBOUND",
    -4: "TBG_ERR_CUDA", -5: "TBG_ERR_NOMEM", -6: "TBG_ERR_DEVICE", -7: "TBG_ERR_TIMEOUT",
    -8: "TBG_ERR_RANGE",
}


class TbgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded libtbgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m tb8gen_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp, u64, i, sz = C.c_void_p, C.c_uint64, C.c_int, C.c_size_t
        sig = {
            "tbg_init": [],
            "tbg_material_from_name": [C.c_char_p],
            "tbg_material_select": [i],
            "tbg_geometry": [C.POINTER(u64), C.POINTER(u64), C.POINTER(u64),
                             C.POINTER(u64), C.POINTER(u64)],
            "tbg_set_stream": [vp],
            "tbg_set_stub": [u64, i],
            "tbg_slot_bind": [i, vp, sz],
            "tbg_sub_bind": [i, vp, sz],
            "tbg_unbind_all": [],
            "tbg_predecessors": [i, i],
            "tbg_candidates": [i, i, vp, sz],
            "tbg_predecessors_sub": [i, i, i],
            "tbg_check_successors": [i, i],
            "tbg_calc_sub": [i, i, vp * 5],
            "tbg_calc_illegal": [i, vp, vp],
            "tbg_calc_mate": [i, vp, vp, vp, vp],
            "tbg_epilogue_W": [i, i, C.POINTER(u64)],
            "tbg_count": [i, C.POINTER(u64)],
            "tbg_count_strided": [vp, u64, i, C.POINTER(u64)],
            "tbg_clear": [i],
            "tbg_sub_and_not": [i, i, i],
            "tbg_sync": [i],
            "tbg_gen_bernoulli": [vp, u64, u64, u64, u64, u64],
            "tbg_attacks": [i, vp, vp, vp, u64],
            "tbg_check_successors_to": [i, i, vp],
            "tbg_epilogue_W_to": [i, vp, vp, C.POINTER(u64)],
            "tbg_launches": [C.POINTER(u64)],
            "tbg_batch_begin": [],
            "tbg_batch_end": [C.POINTER(i), C.POINTER(u64)],
            "tbg_batch_run": [i],
            "tbg_batch_counts": [C.POINTER(u64), i],
            "tbg_batch_tune": [i, C.c_longlong],
            "tbg_batch_shape": [i, i, C.POINTER(u64)],
            "tbg_batch_select": [i],
            "tbg_batch_count": [i],
            "tbg_mark": [C.POINTER(u64)],
            "tbg_copy_in": [vp, vp, sz, u64, C.POINTER(u64)],
            "tbg_copy_out": [vp, vp, sz, u64, C.POINTER(u64)],
            "tbg_join": [u64],
            "tbg_wait_ticket": [u64, i],
            "tbg_table_build": [C.c_char_p, u64, i, i, C.POINTER(vp), C.POINTER(u64)],
            "tbg_table_free_host": [vp],
            "tbg_probe_open": [vp, u64, C.c_char_p, C.POINTER(i)],
            "tbg_probe_close": [i],
            "tbg_probe_tune": [u64],
            "tbg_calc_sub_table": [i, i, vp * 5, C.POINTER(i), i, u64, i],
            "tbg_capture_material": [i, C.c_char_p, i],
            "tbg_probe_phase_ms": [i, C.POINTER(C.c_float), C.POINTER(u64)],
            "tbg_probe_stream_bytes": [i, i, C.POINTER(u64)],
            "tbg_probe_layout": [i, i, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64)],
            "tbg_probe_wdl_batch": [i, vp, u64, vp, i],
            "tbg_probe_wdl_batch8": [i, vp, u64, vp, i],
            "tbg_encode_batch": [i, vp, u64, vp, vp],
            "tbg_decode_batch": [i, i, vp, u64, vp],
            "tbg_gen_positions": [C.c_char_p, u64, u64, vp, C.POINTER(C.c_uint32)],
            "tbg_alloc": [sz, C.POINTER(vp)],
            "tbg_free": [vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.tbg_last_error.restype = C.c_char_p
        L.tbg_last_error.argtypes = []
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc < 0:
        raise TbgError(rc, lib().tbg_last_error().decode(errors="replace"))
    return rc


def ptr(t) -> C.c_void_p | None:
    """Device address of a torch tensor (or an int address / None)."""
    if t is None:
        return None
    if isinstance(t, int):
        return C.c_void_p(t)
    return C.c_void_p(t.data_ptr())


def init(stream=None):
    check(lib().tbg_init())
    if stream is not None:
        set_stream(stream)


def set_stream(stream):
    handle = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", 0)
    check(lib().tbg_set_stream(C.c_void_p(handle)))


def set_stub(seed: int, modulus: int = 3):
    check(lib().tbg_set_stub(seed, modulus))


class Material:
    """A registered material (tbg_material_from_name) and its geometry."""

    def __init__(self, name: str):
        self.name = name
        self.handle = check(lib().tbg_material_from_name(name.encode()))
        size, nbytes, sub = C.c_uint64(), C.c_uint64(), C.c_uint64()
        offs, capt = (C.c_uint64 * 6)(), (C.c_uint64 * 6)()
        check(lib().tbg_geometry(C.byref(size), C.byref(nbytes), C.byref(sub), offs, capt))
        self.size = size.value
        self.bytes = nbytes.value
        self.sub_bytes = sub.value
        self.sub_offset = list(offs)
        self.capt_size = list(capt)

    def select(self):
        check(lib().tbg_material_select(self.handle))
        return self


def bind(s: int, t) -> None:
    check(lib().tbg_slot_bind(s, ptr(t), 0 if t is None else t.numel() * t.element_size()))


def bind_sub(s: int, t) -> None:
    check(lib().tbg_sub_bind(s, ptr(t), 0 if t is None else t.numel() * t.element_size()))


def unbind_all():
    check(lib().tbg_unbind_all())


def predecessors(stm: int, s: int):
    check(lib().tbg_predecessors(stm, s))


def predecessors_sub(stm: int, s: int, legality: bool):
    check(lib().tbg_predecessors_sub(stm, s, int(bool(legality))))


def candidates(stm: int, s: int, opp_wins):
    """predecessors(stm, s) without the predecessors that a one-square slider
    step takes out of opp_wins (the opponent's "wins" of slice s), for an L
    step that verifies against the same opp_wins next."""
    check(lib().tbg_candidates(stm, s, ptr(opp_wins), opp_wins.numel() * opp_wins.element_size()))


def check_successors(stm: int, s: int):
    check(lib().tbg_check_successors(stm, s))


def calc_sub(stm: int, s: int, cls):
    arr = (C.c_void_p * 5)(*[t.data_ptr() for t in cls])
    check(lib().tbg_calc_sub(stm, s, arr))


def calc_sub_table(stm: int, s: int, cls, handles=None, mode: int = 0, seed: int = 0,
                   modulus: int = 3):
    """tbg_calc_sub_table: capture classes with the 7-piece values from the
    tables of the capture materials (mode 0) or their formula (mode 1)."""
    arr = (C.c_void_p * 5)(*[t.data_ptr() for t in cls])
    h = None if handles is None else (C.c_int * 6)(*(list(handles) + [-1] * (6 - len(handles))))
    check(lib().tbg_calc_sub_table(stm, s, arr, h, mode, seed, modulus))


def capture_material(set_index: int) -> str:
    buf = C.create_string_buffer(32)
    check(lib().tbg_capture_material(set_index, buf, 32))
    return buf.value.decode()


def calc_illegal(s: int, ill_w, ill_b):
    check(lib().tbg_calc_illegal(s, ptr(ill_w), ptr(ill_b)))


def calc_mate(s: int, ill_w, ill_b, mate_w, mate_b):
    check(lib().tbg_calc_mate(s, ptr(ill_w), ptr(ill_b), ptr(mate_w), ptr(mate_b)))


def epilogue_W(s: int, s_wins: int = -1, count: bool = True):
    c = C.c_uint64()
    check(lib().tbg_epilogue_W(s, s_wins, C.byref(c) if count else None))
    return c.value if count else None


def check_successors_to(stm: int, s: int, out):
    check(lib().tbg_check_successors_to(stm, s, ptr(out)))


def epilogue_W_to(s: int, wins_in, wins_out, count: bool = True):
    c = C.c_uint64()
    check(lib().tbg_epilogue_W_to(s, ptr(wins_in), ptr(wins_out), C.byref(c) if count else None))
    return c.value if count else None


def launches() -> int:
    n = C.c_uint64()
    check(lib().tbg_launches(C.byref(n)))
    return n.value


def count(s: int) -> int:
    c = C.c_uint64()
    check(lib().tbg_count(s, C.byref(c)))
    return c.value


def count_strided(base, stride_bytes: int, n: int) -> int:
    """Ones below the slice size in n bitmaps at base + i * stride_bytes."""
    c = C.c_uint64()
    check(lib().tbg_count_strided(ptr(base), stride_bytes, n, C.byref(c)))
    return c.value


def clear(s: int):
    check(lib().tbg_clear(s))


def sub_and_not(s1: int, s2: int, stm: int):
    check(lib().tbg_sub_and_not(s1, s2, stm))


def sync(timeout_ms: int = 0):
    check(lib().tbg_sync(timeout_ms))


def gen_bernoulli(t, nbits: int, seed: int, tag: int, thr: int):
    check(lib().tbg_gen_bernoulli(ptr(t), nbits, t.numel() * t.element_size(), seed, tag, thr))


def attacks(piece_type: int, sq, occ, out):
    check(lib().tbg_attacks(piece_type, ptr(sq), ptr(occ), ptr(out), out.numel()))


def batch_begin():
    check(lib().tbg_batch_begin())


def batch_end():
    n, items = C.c_int(), C.c_uint64()
    check(lib().tbg_batch_end(C.byref(n), C.byref(items)))
    return n.value, items.value


def batch_run(mode: int):
    """mode 0: one launch per recorded call; mode 1: one persistent launch
    (block-wide work items); mode 2: one persistent launch, each work item
    cut into one part per warp."""
    check(lib().tbg_batch_run(mode))


def batch_counts(n: int):
    out = (C.c_uint64 * max(n, 1))()
    check(lib().tbg_batch_counts(out, n))
    return list(out)[:n]


def batch_tune(ctas_per_sm: int, spin_limit: int = 0):
    check(lib().tbg_batch_tune(ctas_per_sm, spin_limit))


def batch_shape(scatter_tiles: int = 0, candidate_tiles: int = 0) -> int:
    """Tiles per work item of predecessors (0: 1) and of candidates (0: 4);
    re-cuts the selected recorded batch and returns its work items (0 if
    none is recorded)."""
    n = C.c_uint64()
    check(lib().tbg_batch_shape(scatter_tiles, candidate_tiles, C.byref(n)))
    return n.value


def batch_count(s: int):
    """Records, in the batch being recorded, the count of slot s's bitmap."""
    check(lib().tbg_batch_count(s))


def batch_select(slot: int):
    """Batch slot (0..3) that recording and runs act on."""
    check(lib().tbg_batch_select(slot))


# ------------------------------------------------------- copy streams, tickets
def mark() -> int:
    """Ticket of the library stream's current point."""
    t = C.c_uint64()
    check(lib().tbg_mark(C.byref(t)))
    return t.value


def _nbytes(t) -> int:
    return t.numel() * t.element_size()


def copy_in(dev, host, after: int = 0, ticket: bool = False):
    """Host-to-device copy (pinned host tensor -> device tensor of the same
    size) on the inbound copy stream after ticket `after`; returns the
    ticket after it when asked."""
    t = C.c_uint64()
    check(lib().tbg_copy_in(ptr(dev), ptr(host), _nbytes(host), after,
                            C.byref(t) if ticket else None))
    return t.value if ticket else None


def copy_out(host, dev, after: int = 0, ticket: bool = False):
    """Device-to-host copy on the outbound copy stream after ticket `after`."""
    t = C.c_uint64()
    check(lib().tbg_copy_out(ptr(host), ptr(dev), _nbytes(dev), after,
                             C.byref(t) if ticket else None))
    return t.value if ticket else None


def join(ticket: int):
    """Later work on the library stream waits for the ticket."""
    check(lib().tbg_join(ticket))


def wait_ticket(ticket: int, timeout_ms: int = 0):
    check(lib().tbg_wait_ticket(ticket, timeout_ms))


# ---------------------------------------------------------------- table probes
QUERY_BYTES = 16  # tbg_query: sq[8], stm, pad[7]


def table_build_host(material: str, seed: int, modulus: int = 3) -> bytes:
    """The synthetic WDL table of `material`, built on the CPU (small
    materials): the bytes of the .rtbw file the reference reads."""
    p, n = C.c_void_p(), C.c_uint64()
    check(lib().tbg_table_build(material.encode(), seed, modulus, 0, C.byref(p), C.byref(n)))
    try:
        return C.string_at(p.value, n.value)
    finally:
        lib().tbg_table_free_host(p)


class DeviceTable:
    """A synthetic WDL table built on the device (tbg_table_build) and opened
    for probing (tbg_probe_open)."""

    def __init__(self, material: str, seed: int, modulus: int = 3, image=None):
        self.material = material
        p, n = C.c_void_p(), C.c_uint64()
        if image is None:
            check(lib().tbg_table_build(material.encode(), seed, modulus, 1, C.byref(p),
                                        C.byref(n)))
            self._owned = p.value
            self.addr, self.bytes = p.value, n.value
        else:  # a torch uint8 device tensor holding a table image
            self._owned = None
            self._image = image
            self.addr, self.bytes = image.data_ptr(), image.numel()
        h = C.c_int()
        check(lib().tbg_probe_open(C.c_void_p(self.addr), self.bytes, material.encode(),
                                   C.byref(h)))
        self.handle = h.value

    def close(self):
        if self.handle is not None:
            check(lib().tbg_probe_close(self.handle))
            self.handle = None
        if self._owned:
            check(lib().tbg_free(C.c_void_p(self._owned)))
            self._owned = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def layout(self, side: int):
        """(data offset, blocks, positions) of one side of the table."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().tbg_probe_layout(self.handle, side, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def stream_bytes(self, side: int) -> int:
        """Bytes of one side's compressed streams (zero padding excluded)."""
        b = C.c_uint64()
        check(lib().tbg_probe_stream_bytes(self.handle, side, C.byref(b)))
        return b.value

    def phase_ms(self):
        """((locate, decode, answer) device ms, touched blocks) of the last
        grouped batch."""
        ms = (C.c_float * 3)()
        nb = C.c_uint64()
        check(lib().tbg_probe_phase_ms(self.handle, ms, C.byref(nb)))
        return tuple(ms), nb.value

    def image(self):
        """The table image as a uint8 torch tensor on the device (a view)."""
        import torch

        addr, nbytes = self.addr, self.bytes

        class _Arr:
            __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                        "data": (addr, False), "version": 3}
        return torch.as_tensor(_Arr(), device="cuda")

    def probe(self, queries, out, mode: int = 0):
        n = queries.numel() // QUERY_BYTES
        check(lib().tbg_probe_wdl_batch(self.handle, ptr(queries), n, ptr(out), mode))

    def probe8(self, queries8, out, mode: int = 0):
        """Probe on compact 8-byte queries (see compact_queries)."""
        n = queries8.numel() // 8
        check(lib().tbg_probe_wdl_batch8(self.handle, ptr(queries8), n, ptr(out), mode))

    def encode(self, queries, idx, side=None):
        n = queries.numel() // QUERY_BYTES
        check(lib().tbg_encode_batch(self.handle, ptr(queries), n, ptr(idx), ptr(side)))

    def decode(self, side: int, idx, squares):
        check(lib().tbg_decode_batch(self.handle, side, ptr(idx), idx.numel(), ptr(squares)))


def compact_queries(queries):
    """16-byte queries (uint8 tensor) -> 8-byte compact ones: squares 0-6,
    side to move in byte 7 (materials of at most 7 pieces)."""
    q = queries.view(-1, QUERY_BYTES)
    import torch
    return torch.cat([q[:, :7], q[:, 8:9]], dim=1).contiguous().view(-1)


def probe_tune(scratch_bytes: int):
    check(lib().tbg_probe_tune(scratch_bytes))


_PIECE_RANK = {6: 1, 14: 2, 2: 3, 10: 4, 3: 5, 11: 6, 4: 7, 12: 8, 5: 9, 13: 10}


def material_pieces(material: str) -> list[int]:
    """Piece codes (type | 8 for black) in main()'s order (tb8gen.c:1331-1339):
    the order of a query's squares."""
    pt, black = [], 0
    for ch in material:
        if ch == "v":
            black = 8
            continue
        pt.append(("PNBRQK".index(ch) + 1) | black)
    return sorted(pt, key=lambda p: _PIECE_RANK[p])


def table_pieces(material: str) -> list[int]:
    """The piece order of the synthetic tables (tbg_table_build): the kings,
    then, unless only the kings are unique, the first other unique piece,
    then the rest in material order.  tbg_decode_batch lists squares so."""
    pt = material_pieces(material)
    cnt = {p: pt.count(p) for p in pt}
    out, rest = pt[:2], list(pt[2:])
    if sum(1 for p in cnt if cnt[p] == 1) > 2:
        u = next(p for p in rest if cnt[p] == 1)
        out.append(u)
        rest.remove(u)
    return out + rest


def table_to_query_columns(material: str) -> list[int]:
    """cols[j] = the table-order column holding the square of query column j."""
    tp, mp = table_pieces(material), material_pieces(material)
    used = [False] * len(tp)
    cols = []
    for p in mp:
        k = next(k for k in range(len(tp)) if tp[k] == p and not used[k])
        used[k] = True
        cols.append(k)
    return cols


def gen_positions(material: str, seed: int, queries) -> int:
    """Fills a uint8 device tensor of n*16 bytes with n seeded legal
    positions; returns how many draws found no legal position."""
    failed = C.c_uint32()
    n = queries.numel() // QUERY_BYTES
    check(lib().tbg_gen_positions(material.encode(), seed, n, ptr(queries), C.byref(failed)))
    return failed.value
