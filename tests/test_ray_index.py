"""The slider unmove's incremental index (mark_unmoves_inc in
tb8gen_b200/csrc/tbg_kernels.cuh) restated in Python and checked against a
full re-rank of the moved position (sq_to_idx_helper, tb8gen.c:129-149: per
set, the sum over its squares in increasing order of C(r, i + 1), r the
square's rank among the squares not taken by the kings and earlier sets).

Along a ray the kernel keeps, from the previous square to the next, the
count of occupied squares of the earlier sets below the target, the count of
the moving set's other pieces below it, and the sum of the later sets' Pascal
terms of the squares passed (seg_delta); the target's index is then
base + (C(to - cnt, pos + 1) + g[pos]) * factor[k] + dx.  CPU only."""
import random
from math import comb

import pytest

DIRS = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1), (1, -1), (-1, -1)]


def popc(x):
    return bin(x).count("1")


def bit(q):
    return 1 << q


def between(a, b):
    lo, hi = min(a, b), max(a, b)
    return ((1 << hi) - 1) & ~((1 << (lo + 1)) - 1)


def rank_set(mask, occ):
    r, i = 0, 0
    for q in range(64):
        if mask >> q & 1:
            r += comb(q - popc(occ & (bit(q) - 1)), i + 1)
            i += 1
    return r


def full_index(sets, kings, factor):
    occ, idx = kings, 0
    for j, s in enumerate(sets):
        idx += rank_set(s, occ) * factor[j]
        occ |= s
    return idx


def seg_delta(sets, kings, j0, seg, up, factor):
    occ, d = kings, 0
    for j, s in enumerate(sets):
        if j >= j0:
            for q in range(64):
                if (s & seg) >> q & 1:
                    below = bit(q) - 1
                    r, i = q - popc(occ & below), popc(s & below)
                    v = (comb(r, i) if up else comb(r - 1, i)) * factor[j]
                    d += v if up else -v
        occ |= s
    return d


def mover_g(others, occk):
    a, b = [0, 0, 0], [0, 0, 0]
    for i, q in enumerate([q for q in range(64) if others >> q & 1][:3]):
        r = q - popc(occk & (bit(q) - 1))
        a[i], b[i] = comb(r, i + 1), comb(r, i + 2)
    return [b[0] + b[1] + b[2], a[0] + b[1] + b[2], a[0] + a[1] + b[2], a[0] + a[1] + a[2]]


def check(mult, types, trials, rng):
    ns = len(mult)
    free = [62 - sum(mult[:j]) for j in range(ns)]
    factor = [1] * ns
    for j in range(ns - 2, -1, -1):
        factor[j] = factor[j + 1] * comb(free[j + 1], mult[j + 1])
    checked = 0
    for _ in range(trials):
        sqs = rng.sample(range(64), 2 + sum(mult))
        kings = bit(sqs[0]) | bit(sqs[1])
        sets, p = [], 2
        for m in mult:
            sets.append(sum(bit(q) for q in sqs[p:p + m]))
            p += m
        occ = kings
        for s in sets:
            occ |= s
        idx = full_index(sets, kings, factor)
        occk = kings
        for k in range(ns):
            if types[k] in (3, 4, 5):
                base = idx - rank_set(sets[k], occk) * factor[k]
                for x in (q for q in range(64) if sets[k] >> q & 1):
                    others = sets[k] & ~bit(x)
                    g = mover_g(others, occk)
                    cnt0, pos0 = popc(occk & (bit(x) - 1)), popc(others & (bit(x) - 1))
                    dirs = {3: range(4, 8), 4: range(0, 4), 5: range(8)}[types[k]]
                    for d in dirs:
                        df, dr = DIRS[d]
                        up = dr > 0 or (dr == 0 and df > 0)
                        f, r, cur, cnt, pos, dx = x & 7, x >> 3, x, cnt0, pos0, 0
                        while True:
                            f += df
                            r += dr
                            if not (0 <= f < 8 and 0 <= r < 8):
                                break
                            to = r * 8 + f
                            if occ >> to & 1:
                                break
                            seg = between(cur, to)
                            cnt += popc(occk & seg) * (1 if up else -1)
                            pos += popc(others & seg) * (1 if up else -1)
                            dx += seg_delta(sets, kings, k + 1, seg, up, factor)
                            cur = to
                            got = base + (comb(to - cnt, pos + 1) + g[pos]) * factor[k] + dx
                            moved = list(sets)
                            moved[k] = others | bit(to)
                            assert got == full_index(moved, kings, factor), (mult, k, x, to)
                            checked += 1
            occk |= sets[k]
    return checked


# (piece counts per set, piece type per set: 3 bishop, 4 rook, 5 queen)
CASES = [([3, 3], [4, 4]),            # KRRRvKRRR
         ([1, 3, 1], [4, 4, 5]),      # KQRvKRRR: wR, bR x3, wQ
         ([2, 2, 1], [4, 4, 5]),      # KQRRvKRR
         ([1, 1, 2, 1], [3, 3, 4, 5]),
         ([4, 1], [4, 5])]


@pytest.mark.parametrize("mult,types", CASES)
def test_ray_index_equals_full_rank(mult, types):
    assert check(mult, types, 60, random.Random(sum(mult) * 7 + len(mult))) > 0
