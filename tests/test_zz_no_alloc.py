"""gx_sort_column_pair_noalloc: the allocation-free pair sort gives exactly
what gx_sort_column_pair gives, on two calls in a row that reuse the same
fixed scratch without clearing it, allocates nothing, and rejects sorts
whose scratch would exceed the fixed 8 MiB before launching anything."""
import ctypes as C

import numpy as np
import pytest

import eiger_b200 as gx

pytestmark = pytest.mark.gpu

LIMIT = 8 << 20


def noalloc():
    f = gx.lib.gx_sort_column_pair_noalloc
    f.argtypes = [gx.ColumnView, gx.ColumnView, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int32
    return f


def mem_stats():
    cur, peak = C.c_int64(), C.c_int64()
    gx.check(gx.lib.gx_mem_stats(C.byref(cur), C.byref(peak)))
    return cur.value, peak.value


def make(n, kdt, vdt, seed):
    import torch
    rng = np.random.default_rng(seed)
    if np.dtype(kdt).kind == "f":
        k = rng.normal(size=n).astype(kdt)
        if n > 8:
            k[:4] = [0.0, -0.0, np.inf, -np.inf]
    elif np.dtype(kdt).kind == "u":
        k = rng.integers(0, np.iinfo(kdt).max, size=n, dtype=kdt)
    else:
        k = rng.integers(np.iinfo(kdt).min, np.iinfo(kdt).max, size=n, dtype=kdt)
    k[n // 2:] = k[: n - n // 2]  # duplicates exercise stability
    v = np.arange(n, dtype=np.int64).astype(vdt)
    return torch.from_numpy(k).cuda(), torch.from_numpy(v).cuda()


def run_noalloc(k, v, begin, end, order):
    import torch
    ko, vo = torch.empty_like(k), torch.empty_like(v)
    st = noalloc()(gx.view(k), gx.view(v), begin, end, order, ko.data_ptr(), vo.data_ptr(), gx._stream_ptr(None))
    assert st == 0, gx.last_error()
    torch.cuda.synchronize()
    return ko, vo


CASES = [
    (300_001, np.int32, np.int64, 0, -1, gx.ASCENDING),
    (200_000, np.int64, np.int32, 0, -1, gx.DESCENDING),
    (250_000, np.float64, np.int64, 0, -1, gx.ASCENDING),
    (400_000, np.float32, np.uint32, 4, 20, gx.ASCENDING),
    (100_000, np.uint64, np.float64, 8, 40, gx.DESCENDING),
    (1, np.int32, np.int32, 0, -1, gx.ASCENDING),
    (4096, np.int32, np.int32, 8, 8, gx.ASCENDING),  # no bits: a plain copy
]


@pytest.mark.parametrize("n,kdt,vdt,begin,end,order", CASES)
def test_two_calls_in_a_row_match_the_allocating_sort(n, kdt, vdt, begin, end, order):
    import torch
    for seed in (1, 2):  # the second call reuses scratch the first one left dirty
        k, v = make(n, kdt, vdt, seed + n)
        ek, ev = gx.sort_column_pair(k, v, begin, end, order)
        torch.cuda.synchronize()
        gk, gv = run_noalloc(k, v, begin, end, order)
        assert torch.equal(gk.view(torch.uint8), ek.view(torch.uint8))
        assert torch.equal(gv.view(torch.uint8), ev.view(torch.uint8))


def test_allocates_nothing():
    import torch
    k, v = make(500_000, np.int32, np.int32, 7)
    run_noalloc(k, v, 0, -1, gx.ASCENDING)  # first call on the device: one-time setup
    ko, vo = torch.empty_like(k), torch.empty_like(v)
    torch.cuda.synchronize()
    gx.check(gx.lib.gx_mem_reset_peak())
    before, torch_before = mem_stats(), torch.cuda.memory_allocated()
    launches = gx.kernel_launches()
    st = noalloc()(gx.view(k), gx.view(v), 0, -1, gx.ASCENDING, ko.data_ptr(), vo.data_ptr(), gx._stream_ptr(None))
    assert st == 0, gx.last_error()
    torch.cuda.synchronize()
    assert gx.kernel_launches() > launches
    assert mem_stats() == (before[0], before[0])
    assert torch.cuda.memory_allocated() == torch_before


def test_rejects_sorts_beyond_the_scratch_limit():
    import torch
    n = 600_000  # 8+8-byte pairs: 2 * 4.8 MB of ping-pong halves alone exceed 8 MiB
    k = torch.zeros(n, dtype=torch.int64, device="cuda")
    v = torch.zeros(n, dtype=torch.int64, device="cuda")
    ko, vo = torch.empty_like(k), torch.empty_like(v)
    launches = gx.kernel_launches()
    st = noalloc()(gx.view(k), gx.view(v), 0, -1, gx.ASCENDING, ko.data_ptr(), vo.data_ptr(), gx._stream_ptr(None))
    assert st == 1  # GX_EINVAL
    msg = gx.last_error()
    assert str(LIMIT) in msg and "8 MiB" in msg
    assert gx.kernel_launches() == launches
    # The same sort fits when it is small enough.
    ks, vs = k[:100_000].contiguous(), v[:100_000].contiguous()
    run_noalloc(ks, vs, 0, -1, gx.ASCENDING)


def test_rejects_narrow_columns_and_overlapping_outputs():
    import torch
    k = torch.arange(1000, dtype=torch.int16, device="cuda")
    v = torch.arange(1000, dtype=torch.int32, device="cuda")
    out = torch.empty(1000, dtype=torch.int32, device="cuda")
    st = noalloc()(gx.view(k), gx.view(v), 0, -1, gx.ASCENDING, out.data_ptr(), out.data_ptr(), None)
    assert st == 6 and "4- or 8-byte" in gx.last_error()
    k32 = torch.arange(1000, dtype=torch.int32, device="cuda")
    vo = torch.empty_like(v)
    st = noalloc()(gx.view(k32), gx.view(v), 0, -1, gx.ASCENDING, k32.data_ptr(), vo.data_ptr(), None)
    assert st == 1 and "overlap" in gx.last_error()


def test_later_calls_of_other_width_pairs_after_the_first():
    """The first call (4+4 bytes) prepares every width pair; calls of the
    other three pairs that follow give the allocating sort's result."""
    import torch
    for kdt, vdt in ((np.int32, np.int32), (np.int64, np.int64), (np.uint32, np.float64), (np.float64, np.uint32)):
        k, v = make(123_457, kdt, vdt, 99)
        ek, ev = gx.sort_column_pair(k, v, 0, -1, gx.ASCENDING)
        torch.cuda.synchronize()
        gk, gv = run_noalloc(k, v, 0, -1, gx.ASCENDING)
        assert torch.equal(gk.view(torch.uint8), ek.view(torch.uint8))
        assert torch.equal(gv.view(torch.uint8), ev.view(torch.uint8))
