"""How the warp-wide kernels (tb8gen_b200/csrc/tbg_warp.cuh) cut a sparse
op's bitmap into parts, restated in Python and checked on the CPU: every
word of the bitmap belongs to exactly one part, and every part is run by
exactly one warp.

* Persistent kernel (k_batch_w): block item b of an op with gt tiles per
  item covers tiles [b*gt, (b+1)*gt) (1,024 words each); its part s of
  kWarps covers gt x 128 words from sub_word0.  Parts are taken in order
  from one counter.
* Per-call kernel (k_op_w): parts of 32 words, in runs of kRun consecutive
  parts dealt to the grid's warps in turn (warp g: runs g, g + warps, ...)."""
import pytest

K_WARPS, K_SUB_WORDS, K_TILE_WORDS, K_RUN = 8, 128, 1024, 4


def sub_word0(u, gt, wpl):
    if wpl == 1:
        return u * 32
    b, s = divmod(u, K_WARPS)
    return b * gt * K_TILE_WORDS + s * gt * K_SUB_WORDS


@pytest.mark.parametrize("nwords,gt", [(1, 1), (1000, 1), (1024, 1), (5000, 2), (70000, 4),
                                       (3 * 1024 + 17, 8)])
def test_persistent_parts_cover_each_word_once(nwords, gt):
    tiles = (nwords + K_TILE_WORDS - 1) // K_TILE_WORDS
    ntiles_items = (tiles + gt - 1) // gt          # op_tiles: block items of gt tiles
    seen = [0] * nwords
    for u in range(ntiles_items * K_WARPS):         # the op's parts
        c0 = sub_word0(u, gt, 4)
        for g in range(gt):
            start = c0 + g * K_SUB_WORDS
            if start >= nwords:
                break
            for lane in range(32):
                for i in range(4):
                    w = start + lane * 4 + i
                    if w < nwords:
                        seen[w] += 1
    assert seen == [1] * nwords


def op_w_parts(nsub, grid):
    """Sub-items each warp of k_op_w runs (its fetch: +1 inside a run, then
    past the other warps' runs)."""
    nw = grid * K_WARPS
    skip = (nw - 1) * K_RUN
    runs = []
    for g in range(nw):
        it, mine = g * K_RUN, []
        while it < nsub:
            mine.append(it)
            it = it + 1 if (it + 1) % K_RUN else it + 1 + skip
        runs.append(mine)
    return runs


@pytest.mark.parametrize("nwords,grid", [(1, 1), (31, 1), (33, 2), (4096, 3), (100000, 592),
                                         (12345, 7)])
def test_per_call_parts_cover_each_part_once(nwords, grid):
    nsub = (nwords + 31) // 32 if nwords else 1
    runs = op_w_parts(nsub, grid)
    flat = sorted(u for r in runs for u in r)
    assert flat == list(range(nsub))
    for r in runs:  # within a warp: increasing, contiguous within each run
        assert r == sorted(r)
        for a, b in zip(r, r[1:]):
            assert b == a + 1 or a % K_RUN == K_RUN - 1
    seen = [0] * nwords
    for u in flat:
        for lane in range(32):
            w = sub_word0(u, 1, 1) + lane
            if w < nwords:
                seen[w] += 1
    assert seen == [1] * nwords
