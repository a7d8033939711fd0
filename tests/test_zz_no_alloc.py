"""The allocation-free epilogue entry point (tbg_epilogue_W_static).

It serves callers that cannot allocate device memory -- processes whose HBM
belongs to a caching allocator or a fixed-budget pool, and foreign hosts
whose bindings forbid a library to allocate -- so it runs without tbg_init
and keeps its scratch in a static device array.  The GPU test compares it,
through the C ABI, with the allocating entry point tbg_epilogue_W_to on two
calls in a row (different inputs, so stale scratch would show); the CPU
test checks that bitmaps beyond the 1 GiB limit are refused before any
CUDA call.  Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import tb8gen_b200 as tbg
from oracle import oracle as orc


def _fn():
    L = tbg.lib()
    f = L.tbg_epilogue_W_static
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p,
                  C.POINTER(C.c_uint64)]
    f.restype = C.c_int
    return f


def test_rejects_oversize_bitmap():
    f = _fn()
    cnt = C.c_uint64(0)
    big = (1 << 30) + 16
    rc = f(C.c_void_p(256), C.c_void_p(512), C.c_void_p(768), big * 8, big, None, C.byref(cnt))
    assert rc == -8  # TBG_ERR_RANGE


@pytest.mark.gpu
def test_static_epilogue_matches_allocating_epilogue():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    f = _fn()
    # The allocating entry point needs the engine set up; the static one does not.
    tbg.init()
    m = tbg.Material("KRRRvKRRR").select()
    for seed in (1, 2):
        T = orc.gen_bitmap(m.size, m.bytes, seed, 10, 0.05)
        W = orc.gen_bitmap(m.size, m.bytes, seed, 11, 0.3)
        T[-16:] = 0xFF  # padding bits are carried, not counted
        # allocating path
        t_a, w_in = torch.from_numpy(T).cuda(), torch.from_numpy(W).cuda()
        w_a = torch.empty_like(w_in)
        tbg.unbind_all()
        tbg.bind(7, t_a)
        c_a = tbg.epilogue_W_to(7, w_in, w_a)
        # allocation-free path
        t_b = torch.from_numpy(T).cuda()
        w_b = torch.empty_like(w_in)
        cnt = C.c_uint64(0)
        torch.cuda.synchronize()
        rc = f(C.c_void_p(t_b.data_ptr()), C.c_void_p(w_in.data_ptr()), C.c_void_p(w_b.data_ptr()),
               m.size, m.bytes, None, C.byref(cnt))
        assert rc == 0
        assert cnt.value == c_a
        assert torch.equal(t_a, t_b) and torch.equal(w_a, w_b)
        # and the in-place form (wins_in == wins_out)
        t_c, w_c = torch.from_numpy(T).cuda(), torch.from_numpy(W).cuda()
        rc = f(C.c_void_p(t_c.data_ptr()), C.c_void_p(w_c.data_ptr()), C.c_void_p(w_c.data_ptr()),
               m.size, m.bytes, None, C.byref(cnt))
        assert rc == 0 and cnt.value == c_a
        assert torch.equal(t_c, t_a) and torch.equal(w_c, w_a)
        assert c_a == int(np.unpackbits((T & ~W)[: (m.size + 7) // 8], bitorder="little")[: m.size].sum())
