"""Oracle test infrastructure -- NOT product code.

The checker of the table probe: the reference's own table reader, WDL probe
(``probe_table``, probe.c:1522-1597), ``encode_piece``/``decode_piece`` and
rANS code construction (rans.c), compiled in place from the reference
sources into ``oracle/_ref/libtbprobe.so`` by ``oracle/Makefile`` (target
``probe``), plus a numpy restatement of the synthetic table's value formula.
Only tests use it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE_SO = os.path.join(HERE, "_ref", "libtbprobe.so")

QUERY_BYTES = 16
# piece_order of main() (tb8gen.c:1331-1334): K, k, N, n, B, b, R, r, Q, q
PIECE_ORDER = {6: 1, 14: 2, 2: 3, 10: 4, 3: 5, 11: 6, 4: 7, 12: 8, 5: 9, 13: 10}
LETTERS = "PNBRQK"


def material_pieces(name: str) -> list[int]:
    """Piece codes (type | 8 for black) of a material in main()'s order."""
    pt, black = [], 0
    for ch in name:
        if ch == "v":
            black = 8
            continue
        pt.append((LETTERS.index(ch) + 1) | black)
    return sorted(pt, key=lambda p: PIECE_ORDER[p])


def table_file_name(name: str) -> str:
    """The file name the reference looks for (create_material_string order:
    K Q R B N P per side, probe.c:1484-1501)."""
    w, b = name.split("v")
    key = {c: i for i, c in enumerate("KQRBNP")}
    return "".join(sorted(w, key=key.get)) + "v" + "".join(sorted(b, key=key.get))


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def table_wdl(seed: int, modulus: int, idx: np.ndarray, bside: np.ndarray) -> np.ndarray:
    """wdl of the synthetic table at index idx of side bside:
    VALS[splitmix64(seed ^ idx ^ bside << 63) mod modulus]."""
    h = _mix64(np.uint64(seed) ^ idx.astype(np.uint64)
               ^ (bside.astype(np.uint64) << np.uint64(63)))
    r = (h % np.uint64(modulus)).astype(np.int64)
    vals = np.array([-2, 0, 2] if modulus == 3 else [-2, -1, 0, 1, 2], dtype=np.int8)
    return vals[r]


def probe_available() -> bool:
    return os.path.exists(PROBE_SO)


_lib = None


def probe_lib():
    global _lib
    if _lib is None:
        if not probe_available():
            raise FileNotFoundError(f"{PROBE_SO} missing (make -C oracle probe)")
        L = C.CDLL(PROBE_SO)
        vp, u64, i = C.c_void_p, C.c_uint64, C.c_int
        L.refp_init.argtypes = [C.c_char_p]
        L.refp_init.restype = i
        L.refp_probe.argtypes = [vp, i, vp, u64, vp]
        L.refp_probe.restype = None
        L.refp_encode.argtypes = [vp, i, vp, u64, vp, vp]
        L.refp_encode.restype = i
        L.refp_decode.argtypes = [vp, i, i, vp, u64, vp]
        L.refp_decode.restype = i
        L.refp_code.argtypes = [vp, i, vp, vp, vp, vp, vp, C.POINTER(u64)]
        L.refp_code.restype = i
        L.refp_read_code.argtypes = [vp, vp, vp, vp, C.POINTER(u64)]
        L.refp_read_code.restype = i
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class RefProbe:
    """The reference's probe over the tables of one directory."""

    def __init__(self, directory: str):
        import sys

        self.L = probe_lib()
        # init_tablebases prints a count line on stdout; keep stdout clean for
        # callers that print one result line there
        sys.stdout.flush()
        saved = os.dup(1)
        try:
            with open(os.devnull, "w") as null:
                os.dup2(null.fileno(), 1)
                self.found = self.L.refp_init(directory.encode())
                C.CDLL(None).fflush(None)
        finally:
            os.dup2(saved, 1)
            os.close(saved)

    @staticmethod
    def _pt(material: str) -> np.ndarray:
        return np.array(material_pieces(material), dtype=np.uint8)

    def probe(self, material: str, queries: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(queries, dtype=np.uint8).reshape(-1, QUERY_BYTES)
        out = np.zeros(len(q), dtype=np.int8)
        pt = self._pt(material)
        self.L.refp_probe(_p(pt), len(pt), _p(q), len(q), _p(out))
        return out

    def encode(self, material: str, queries: np.ndarray):
        q = np.ascontiguousarray(queries, dtype=np.uint8).reshape(-1, QUERY_BYTES)
        idx = np.zeros(len(q), dtype=np.uint64)
        side = np.zeros(len(q), dtype=np.uint8)
        pt = self._pt(material)
        if self.L.refp_encode(_p(pt), len(pt), _p(q), len(q), _p(idx), _p(side)) != 0:
            raise RuntimeError(f"no table for {material}")
        return idx, side

    def decode(self, material: str, bside: int, idx: np.ndarray) -> np.ndarray:
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        sq = np.zeros((len(idx), 8), dtype=np.uint8)
        pt = self._pt(material)
        if self.L.refp_decode(_p(pt), len(pt), bside, _p(idx), len(idx), _p(sq)) != 0:
            raise RuntimeError(f"table of {material} not mapped")
        return sq


def ref_code(freq: np.ndarray):
    """create_code_rans + write_freq_table of a histogram."""
    L = probe_lib()
    f = np.ascontiguousarray(freq, dtype=np.int64)
    fo = np.zeros(4096, np.uint16)
    cum = np.zeros(4096, np.uint16)
    remap = np.zeros(1 << 16, np.uint16)
    smap = np.zeros(4096, np.uint16)
    ftab = np.zeros(16384, np.uint8)
    n = C.c_uint64()
    if L.refp_code(_p(f), len(f), _p(fo), _p(cum), _p(remap), _p(smap), _p(ftab), C.byref(n)):
        raise RuntimeError("refp_code failed")
    return {"freq": fo, "cum": cum, "remap": remap, "map": smap, "ftab": ftab[: n.value].tobytes()}


def ref_read_code(ftab: bytes):
    """read_freq_table + make_alias_table(d, NULL)."""
    L = probe_lib()
    buf = np.frombuffer(ftab + bytes(64), dtype=np.uint8).copy()
    fo = np.zeros(4096, np.uint16)
    ad = np.zeros(4096, np.uint16)
    st = np.zeros(4096, np.uint16)
    used = C.c_uint64()
    num = L.refp_read_code(_p(buf), _p(fo), _p(ad), _p(st), C.byref(used))
    return {"num": num, "freq": fo, "alias_div": ad, "start": st, "consumed": used.value}


def random_queries(material: str, n: int, seed: int) -> np.ndarray:
    """n seeded placements of a material as probe queries (distinct squares,
    kings not adjacent, random side to move); not necessarily legal."""
    rng = np.random.default_rng(seed)
    pt = material_pieces(material)
    out = np.zeros((n, QUERY_BYTES), dtype=np.uint8)
    for r in range(n):
        while True:
            sq = rng.choice(64, size=len(pt), replace=False)
            wk, bk = sq[0], sq[1]
            if max(abs(int(wk % 8) - int(bk % 8)), abs(int(wk // 8) - int(bk // 8))) > 1:
                break
        out[r, : len(pt)] = sq
        out[r, 8] = rng.integers(0, 2)
    return out
