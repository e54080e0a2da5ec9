"""rz_remove_noalloc: the entry point for callers that cannot allocate device memory.

Such callers (a memory pool that is fully committed or owned by someone else, a real-time path
that must not take the allocator's lock or synchronise) cannot use a context, because a context
allocates its scratch. rz_remove_noalloc works from a fixed device-global array instead. These
tests call it through the C-ABI and check it against rz_remove, bit for bit, on two calls in a row
(the second call runs on the array the first one left behind), and check that an over-limit call
is refused before anything runs. The file is named to be collected last.
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


@pytest.mark.parametrize("words", [1, 4])
def test_noalloc_matches_rz_remove_on_two_calls_in_a_row(words):
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    ctx = rz.Context(0)
    # Two different calls back to back: a large k first, then a smaller one with many orphans,
    # so the second call reads the array the first one left behind.
    for n, k, dist, seed in [(1 << 22, MAX_K, "uniform", 1), (300007, 100003, "red50", 2)]:
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
        torch.cuda.synchronize()
        assert torch.equal(a[: n - k], b[: n - k]), (n, k, dist, words)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
    n = MAX_K + 10
    a = torch.zeros(n, dtype=torch.int32, device=dev)
    di = torch.arange(MAX_K + 1, dtype=torch.int32, device=dev)
    st, _ = _noalloc(a, di, stream)
    assert st == _native.RZ_ERR_UNSUPPORTED
