"""Oracle test infrastructure -- NOT product code.

ctypes front ends over the two CPU checkers of the ply step:

* ``Port``: this project's plain-C restatement (``oracle/liboracle.so``,
  built from ``oracle/tbg_oracle.c``);
* ``Ref``: the reference generator's own workers compiled in place from its
  sources (``oracle/_ref/libtbref.so``, built by ``oracle/Makefile`` where the
  reference tree exists; the built library travels with the repository).

Both expose the same methods, named after the reference functions they drive
(tb8gen.c ``predecessors``, ``predecessors_sub``, ``check_successors``,
``calc_sub_worker``, ``calc_illegal_worker``, ``calc_mate_worker``; kslice.c
``kslice_and_not``/``kslice_count``/``kslice_or``), over numpy host buffers.
Only tests, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg use them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtbref.so")

MIX_GAMMA = 0x9E3779B97F4A7C15


def bern_threshold(p: float) -> int:
    """Threshold for the seeded Bernoulli generator: P(bit) = thr / 2**64."""
    if p >= 1.0:
        return (1 << 64) - 1
    return int(p * float(1 << 64))


def bitmap_tag(bitmap_id: int, stm: int, s: int) -> int:
    """Stream tag of one synthetic bitmap: (id << 32) | (stm << 16) | slice."""
    return (bitmap_id << 32) | (stm << 16) | (s & 0xFFFF)


class _Idx(C.Structure):
    _fields_ = [("numsets", C.c_int), ("size", C.c_uint64),
                ("factor", C.c_uint64 * 6), ("subfactor", C.c_uint32 * 6),
                ("first", C.c_int * 6), ("mult", C.c_int * 6), ("last", C.c_int * 6)]


class _OrcCtx(C.Structure):
    _fields_ = [("num", C.c_int), ("pt", C.c_uint8 * 8), ("pcs", (C.c_int8 * 8) * 2),
                ("pc_to_set", C.c_int * 8), ("ii", _Idx), ("capt", _Idx * 6),
                ("bytes", C.c_uint64), ("sub_offset", C.c_uint64 * 6),
                ("sub_size", C.c_uint64 * 2), ("sub_bytes", C.c_uint64),
                ("slot", C.c_void_p * 463), ("sub", C.c_void_p * 463),
                ("oob_reads", C.c_uint64), ("stub_seed", C.c_uint64), ("stub_mod", C.c_int)]


def _ptr(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


_port_lib = None


def port_lib():
    global _port_lib
    if _port_lib is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError(f"oracle port not built: {PORT_SO} (make -C oracle port)")
        L = C.CDLL(PORT_SO)
        vp, u64, i = C.c_void_p, C.c_uint64, C.c_int
        L.orc_setup.argtypes = [C.POINTER(_OrcCtx), C.c_char_p]
        L.orc_bind.argtypes = [C.POINTER(_OrcCtx), i, vp, vp]
        L.orc_unbind_all.argtypes = [C.POINTER(_OrcCtx)]
        for f in ("orc_predecessors", "orc_check_successors"):
            getattr(L, f).argtypes = [C.POINTER(_OrcCtx), i, i]
        L.orc_predecessors_sub.argtypes = [C.POINTER(_OrcCtx), i, i, i]
        L.orc_calc_sub.argtypes = [C.POINTER(_OrcCtx), i, i, vp * 5]
        L.orc_calc_illegal.argtypes = [C.POINTER(_OrcCtx), i, vp, vp]
        L.orc_calc_mate.argtypes = [C.POINTER(_OrcCtx), i, vp, vp, vp, vp]
        L.orc_epilogue_W.argtypes = [C.POINTER(_OrcCtx), vp, vp]
        L.orc_epilogue_W.restype = u64
        L.orc_count.argtypes = [C.POINTER(_OrcCtx), vp]
        L.orc_count.restype = u64
        L.orc_gen_bernoulli.argtypes = [vp, u64, u64, u64, u64, u64]
        L.orc_rook_attacks.argtypes = [i, u64]
        L.orc_rook_attacks.restype = u64
        L.orc_bishop_attacks.argtypes = [i, u64]
        L.orc_bishop_attacks.restype = u64
        L.orc_sq_to_idx.argtypes = [C.POINTER(_OrcCtx), vp, i]
        L.orc_sq_to_idx.restype = u64
        L.orc_idx_to_sq.argtypes = [C.POINTER(_OrcCtx), u64, i, i, vp]
        L.orc_idx_to_sq.restype = u64
        L.orc_manager.argtypes = [i, i, vp, vp]
        L.orc_mix64.argtypes = [u64]
        L.orc_mix64.restype = u64
        L.orc_stub_value.argtypes = [u64, i, vp, vp, i, i]
        if L.orc_init() != 0:
            raise RuntimeError("oracle table initialisation failed")
        _port_lib = L
    return _port_lib


def gen_bitmap(nbits: int, nbytes: int, seed: int, tag: int, p: float) -> np.ndarray:
    """Seeded Bernoulli(p) bitmap of nbits bits in an nbytes buffer."""
    a = np.zeros(nbytes, dtype=np.uint8)
    port_lib().orc_gen_bernoulli(_ptr(a), nbits, nbytes, seed, tag, bern_threshold(p))
    return a


class Port:
    """The C restatement (oracle/tbg_oracle.c), single-threaded."""

    kind = "port"

    def __init__(self, material: str):
        self.L = port_lib()
        self.ctx = _OrcCtx()
        if self.L.orc_setup(C.byref(self.ctx), material.encode()) != 0:
            raise ValueError(f"bad material {material!r}")
        self.material = material
        self._keep = {}

    # geometry
    @property
    def size(self):
        return int(self.ctx.ii.size)

    @property
    def bytes(self):
        return int(self.ctx.bytes)

    @property
    def numsets(self):
        return int(self.ctx.ii.numsets)

    def sub_size(self, stm):
        return int(self.ctx.sub_size[stm])

    def sub_offset(self, k):
        return int(self.ctx.sub_offset[k])

    def capt_size(self, k):
        return int(self.ctx.capt[k].size)

    @property
    def sub_bytes(self):
        return int(self.ctx.sub_bytes)

    @property
    def oob_reads(self):
        return int(self.ctx.oob_reads)

    def set_stub(self, seed, modulus=3):
        self.ctx.stub_seed = seed
        self.ctx.stub_mod = modulus

    def bind(self, s, bitmap, sub=None):
        self._keep[s] = (bitmap, sub)
        self.L.orc_bind(C.byref(self.ctx), s, _ptr(bitmap), _ptr(sub))

    def unbind_all(self):
        self._keep.clear()
        self.L.orc_unbind_all(C.byref(self.ctx))

    def predecessors(self, stm, s):
        self.L.orc_predecessors(C.byref(self.ctx), stm, s)

    def predecessors_sub(self, stm, s, legality):
        self.L.orc_predecessors_sub(C.byref(self.ctx), stm, s, int(bool(legality)))

    def check_successors(self, stm, s):
        self.L.orc_check_successors(C.byref(self.ctx), stm, s)

    def calc_sub(self, stm, s, cls):
        arr = (C.c_void_p * 5)(*[a.ctypes.data for a in cls])
        self.L.orc_calc_sub(C.byref(self.ctx), stm, s, arr)

    def calc_illegal(self, s, ill_w, ill_b):
        self.L.orc_calc_illegal(C.byref(self.ctx), s, _ptr(ill_w), _ptr(ill_b))

    def calc_mate(self, s, ill_w, ill_b, mate_w, mate_b):
        self.L.orc_calc_mate(C.byref(self.ctx), s, _ptr(ill_w), _ptr(ill_b),
                             _ptr(mate_w), _ptr(mate_b))

    def epilogue_W(self, T, wins):
        return int(self.L.orc_epilogue_W(C.byref(self.ctx), _ptr(T), _ptr(wins)))

    def count(self, p):
        return int(self.L.orc_count(C.byref(self.ctx), _ptr(p)))

    def sq_to_idx(self, sq8, k=-1):
        a = np.ascontiguousarray(sq8, dtype=np.uint8)
        return int(self.L.orc_sq_to_idx(C.byref(self.ctx), _ptr(a), k))

    def idx_to_sq(self, idx, s, k=-1):
        a = np.zeros(8, np.uint8)
        occ = self.L.orc_idx_to_sq(C.byref(self.ctx), idx, s, k, _ptr(a))
        return a, int(occ)


_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib(nthreads: int = 1):
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference harness not built: {REF_SO} (make -C oracle ref)")
        L = C.CDLL(REF_SO)
        vp, u64, i = C.c_void_p, C.c_uint64, C.c_int
        L.ref_setup.argtypes = [C.c_char_p, i]
        L.ref_set_stub.argtypes = [u64, i]
        L.ref_set_stub_table.argtypes = [u64, i]
        L.ref_bind.argtypes = [i, vp, vp]
        L.ref_predecessors.argtypes = [i, i]
        L.ref_check_successors.argtypes = [i, i]
        L.ref_predecessors_sub.argtypes = [i, i, i]
        L.ref_calc_sub.argtypes = [i, i, vp * 5]
        L.ref_calc_illegal.argtypes = [i, vp, vp]
        L.ref_calc_mate.argtypes = [i, vp, vp, vp, vp]
        L.ref_epilogue_W.argtypes = [vp, vp]
        L.ref_epilogue_W.restype = u64
        L.ref_count.argtypes = [vp]
        L.ref_count.restype = u64
        L.ref_sub_and_not.argtypes = [i, vp, vp]
        for f in ("ref_kslice_size", "ref_kslice_bytes", "ref_binomial",
                  "ref_rook_attacks", "ref_bishop_attacks", "ref_knight_attacks",
                  "ref_king_attacks", "ref_sub_size", "ref_sub_offset",
                  "ref_capt_size", "ref_sq_to_idx", "ref_idx_to_sq"):
            getattr(L, f).restype = u64
        L.ref_binomial.argtypes = [i, i]
        L.ref_rook_attacks.argtypes = [i, u64]
        L.ref_bishop_attacks.argtypes = [i, u64]
        L.ref_sq_to_idx.argtypes = [vp, i]
        L.ref_idx_to_sq.argtypes = [u64, i, i, vp]
        L.ref_manager.argtypes = [i, i, vp, vp]
        _ref_lib = L
        _ref_lib._nthreads = nthreads
    return _ref_lib


class Ref:
    """The reference's own workers (oracle/_ref/libtbref.so).

    The reference keeps its state in globals, so only one Ref is live at a
    time; its thread pool is sized by the first Ref created in the process.
    """

    kind = "reference"

    def __init__(self, material: str, nthreads: int = 1):
        self.L = ref_lib(nthreads)
        if self.L.ref_setup(material.encode(), nthreads) != 0:
            raise ValueError(f"bad material {material!r}")
        self.material = material
        self._keep = {}

    @property
    def nthreads(self):
        return int(self.L.ref_num_threads())

    @property
    def size(self):
        return int(self.L.ref_kslice_size())

    @property
    def bytes(self):
        return int(self.L.ref_kslice_bytes())

    @property
    def numsets(self):
        return int(self.L.ref_numsets())

    def sub_size(self, stm):
        return int(self.L.ref_sub_size(stm))

    def sub_offset(self, k):
        return int(self.L.ref_sub_offset(k))

    def capt_size(self, k):
        return int(self.L.ref_capt_size(k))

    @property
    def sub_bytes(self):
        return max(self.sub_size(0), self.sub_size(1))

    def set_stub(self, seed, modulus=3):
        self.L.ref_set_stub(seed, modulus)

    def set_stub_table(self, seed, modulus=3):
        """probe_wdl answers with the value a synthetic table of the
        position's material stores (its formula at the reference's own
        encode_piece index) instead of the key stub."""
        self.L.ref_set_stub_table(seed, modulus)

    def bind(self, s, bitmap, sub=None):
        self._keep[s] = (bitmap, sub)
        if self.L.ref_bind(s, _ptr(bitmap), _ptr(sub)) != 0:
            raise RuntimeError(f"cannot bind slice {s} (19 slots at most)")

    def unbind_all(self):
        self._keep.clear()
        self.L.ref_unbind_all()

    def predecessors(self, stm, s):
        self.L.ref_predecessors(stm, s)

    def predecessors_sub(self, stm, s, legality):
        self.L.ref_predecessors_sub(stm, s, int(bool(legality)))

    def check_successors(self, stm, s):
        self.L.ref_check_successors(stm, s)

    def calc_sub(self, stm, s, cls):
        arr = (C.c_void_p * 5)(*[a.ctypes.data for a in cls])
        self.L.ref_calc_sub(stm, s, arr)

    def calc_illegal(self, s, ill_w, ill_b):
        self.L.ref_calc_illegal(s, _ptr(ill_w), _ptr(ill_b))

    def calc_mate(self, s, ill_w, ill_b, mate_w, mate_b):
        self.L.ref_calc_mate(s, _ptr(ill_w), _ptr(ill_b), _ptr(mate_w), _ptr(mate_b))

    def epilogue_W(self, T, wins):
        return int(self.L.ref_epilogue_W(_ptr(T), _ptr(wins)))

    def count(self, p):
        return int(self.L.ref_count(_ptr(p)))

    def sq_to_idx(self, sq8, k=-1):
        a = np.ascontiguousarray(sq8, dtype=np.uint8)
        return int(self.L.ref_sq_to_idx(_ptr(a), k))

    def idx_to_sq(self, idx, s, k=-1):
        a = np.zeros(8, np.uint8)
        occ = self.L.ref_idx_to_sq(idx, s, k, _ptr(a))
        return a, int(occ)


def king_attacks(sq: int) -> int:
    f, r = sq & 7, sq >> 3
    b = 0
    for df in (-1, 0, 1):
        for dr in (-1, 0, 1):
            if (df or dr) and 0 <= f + df < 8 and 0 <= r + dr < 8:
                b |= 1 << ((r + dr) * 8 + f + df)
    return b


def kksquare(s: int):
    L = port_lib()
    return L.orc_kksquare(s, 0), L.orc_kksquare(s, 1)


def kkmap(a: int, b: int) -> int:
    return port_lib().orc_kkmap(a, b)


def king_targets(stm: int, s: int) -> list[int]:
    """Slices reached from slice s by a king move of side stm (the slices
    mark_king_unmoves / check_king_moves touch, tb8gen.c:246-262, 537-569),
    in ascending order, without s itself."""
    ks = list(kksquare(s))
    me, opp = ks[stm], ks[stm ^ 1]
    b = king_attacks(me) & ~king_attacks(opp) & ~(1 << opp)
    out = set()
    L = port_lib()
    for to in range(64):
        if b >> to & 1:
            k2 = list(ks)
            k2[stm] = to
            m = (0x07 if (k2[0] & 7) >= 4 else 0) | (0x38 if (k2[0] >> 3) >= 4 else 0)
            a, c = k2[0] ^ m, k2[1] ^ m
            if L.orc_fliptest(k2[0], k2[1]):
                a, c = ((a & 7) << 3) | (a >> 3), ((c & 7) << 3) | (c >> 3)
            out.add(L.orc_kkmap(k2[0], k2[1]))
    out.discard(s)
    return sorted(out)
