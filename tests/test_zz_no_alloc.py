"""rz_remove_noalloc: the entry point for callers that cannot allocate device memory.

Such callers (a memory pool that is fully committed or owned by someone else, a real-time path
that must not take the allocator's lock or synchronise) cannot use a context, because a context
allocates its scratch. rz_remove_noalloc works from a fixed device-global array instead. These
tests call it through the C-ABI and check it against rz_remove, bit for bit, on two calls in a row
(the second call runs on the array the first one left behind), for every item width, on both
the one-CTA path and the grid path; check that device-side errors come back through
rz_noalloc_sync_status; and check that an over-limit call is refused before anything runs. The
file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import redzone_b200 as rz
from redzone_b200 import _native, workloads

pytestmark = pytest.mark.gpu
MAX_K = 1 << 20


def _noalloc(d, di, stream):
    out = ctypes.c_int64(-1)
    st = _native.lib.rz_remove_noalloc(ctypes.c_void_p(d.data_ptr()), d.shape[0], rz.item_bytes(d),
                                       ctypes.c_void_p(di.data_ptr()), di.numel(), ctypes.byref(out),
                                       ctypes.c_void_p(stream.cuda_stream))
    return st, out.value


def _sync_status(stream):
    return _native.lib.rz_noalloc_sync_status(ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_noalloc_matches_rz_remove_on_two_calls_in_a_row(words):
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    ctx = rz.Context(0)
    # Calls back to back: a large k first (grid of CTAs), then a smaller one with many orphans,
    # then a list short enough for one CTA, so each call reads the array the previous one left.
    cases = [(1 << 22, MAX_K, "uniform", 1), (300007, 100003, "red50", 2), (5000, 700, "red30", 3)]
    if words == 8:
        cases[0] = (1 << 21, MAX_K, "uniform", 1)  # 32-byte items: keep the buffers modest
    for n, k, dist, seed in cases:
        rng = np.random.default_rng(seed)
        host = rng.integers(0, 1 << 31, size=(n, words), dtype=np.int64).astype(np.int32)
        idx = workloads.make(dist, n, k, seed).astype(np.int32)
        a = torch.from_numpy(host).to(dev)
        b = a.clone()
        di = torch.from_numpy(idx).to(dev)
        st, new_len = _noalloc(a, di, stream)
        assert st == 0, rz.status_string(st)
        assert new_len == n - k
        ctx.remove(b, di)
        assert _sync_status(stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(a[: n - k], b[: n - k]), (n, k, dist, words)
    ctx.close()


@pytest.mark.parametrize("n,k", [(5000, 700), (1 << 20, 1 << 16)])
def test_noalloc_reports_an_index_out_of_range(n, k):
    """An index >= n is skipped (never used as an address) and reported on the next
    rz_noalloc_sync_status, which then clears the report. Such a list has no canonical result
    (the reference requires every index < n), so the check is on what must still hold: the
    prefix holds n - k distinct survivors and no item whose index was removed."""
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
    idx = workloads.make("red20", n, k, 5).astype(np.int64)
    idx[k // 3] = n + 17  # replaces one in-range entry
    a = torch.arange(n, dtype=torch.int32, device=dev)
    di = torch.from_numpy(idx.astype(np.uint32).view(np.int32)).to(dev)
    assert _sync_status(stream) == 0  # nothing pending from earlier tests
    st, _ = _noalloc(a, di, stream)
    assert st == 0
    assert _sync_status(stream) == _native.RZ_ERR_OUT_OF_RANGE
    assert _sync_status(stream) == 0  # read and cleared
    pre = a[: n - k].cpu().numpy()
    assert np.unique(pre).size == pre.size == n - k
    removed = idx[idx < n]
    assert not np.isin(removed, pre).any()
    # The next call on the same array starts clean and reports nothing.
    b = torch.arange(n, dtype=torch.int32, device=dev)
    good = torch.from_numpy(workloads.make("red20", n, k, 6).astype(np.int32)).to(dev)
    assert _noalloc(b, good, stream)[0] == 0
    assert _sync_status(stream) == 0


def test_noalloc_rejects_sizes_beyond_its_limit():
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
    n = MAX_K + 10
    a = torch.zeros(n, dtype=torch.int32, device=dev)
    di = torch.arange(MAX_K + 1, dtype=torch.int32, device=dev)
    st, _ = _noalloc(a, di, stream)
    assert st == _native.RZ_ERR_UNSUPPORTED
