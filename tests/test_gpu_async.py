"""rz_remove_host_idx_async / rz_wait: the pipelined host-index removal, against the oracle.

Calls are issued back to back on one list (each removes from what the previous one left, as a
host program feeding removal lists in a loop would), with more calls in flight than the context
has staging slots, with growing k, and with every item width; each result is checked against
the oracle applied in the same order."""
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from redzone_b200 import _native, workloads

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def _chain(n0, ks, seed):
    """Index lists of a chain of removals: list j removes ks[j] items from the length left."""
    out, n = [], n0
    for j, k in enumerate(ks):
        dist = ("uniform", "red30", "clustered", "tail")[j % 4]
        if dist == "clustered" and k < 256:
            dist = "uniform"
        out.append(workloads.make(dist, n, k, seed + j))
        n -= k
    return out


@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_async_chain_matches_oracle(ctx, words):
    n0 = 1 << 20
    ks = [1000, 1 << 14, 5, 1 << 16, 300, 1 << 12, 70000, 1 << 10, 2, 1 << 15]
    lists = _chain(n0, ks, seed=40 + words)
    rng = np.random.default_rng(words)
    host = rng.integers(0, 1 << 32, size=(n0, words), dtype=np.uint64).astype(np.uint32)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    pinned = [torch.from_numpy(x.astype(np.int32)).pin_memory() for x in lists]
    # Issue every call before collecting any (10 calls > the context's 4 slots).
    n, tickets = n0, []
    for x in pinned:
        tickets.append(ctx.remove_host_idx_async(d[:n], x))
        n -= x.numel()
    exp = host.copy()
    n = n0
    for t, x in zip(tickets, lists):
        assert ctx.wait(t) == n - x.size
        sub = exp[:n].copy()
        oracle.remove(sub, x)
        exp[:n - x.size] = sub[:n - x.size]
        n -= x.size
    got = d.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[:n], exp[:n])


def test_async_interleaved_waits_and_errors(ctx):
    n = 1 << 18
    a = torch.arange(n, dtype=torch.int32, device=DEV)
    b = a.clone()
    idx = [workloads.uniform(n, 4096, seed=s).astype(np.int32) for s in range(6)]
    pinned = [torch.from_numpy(x).pin_memory() for x in idx]
    # Each call removes from the full length n of its own array copy: results are independent.
    arrays = [a.clone() for _ in idx]
    tickets = [ctx.remove_host_idx_async(arr, x) for arr, x in zip(arrays, pinned)]
    # Collect out of order.
    for j in (3, 0, 5, 1, 4, 2):
        assert ctx.wait(tickets[j]) == n - 4096
    for arr, x in zip(arrays, idx):
        exp = np.arange(n, dtype=np.int32)
        oracle.remove(exp, x.astype(np.uint32))
        assert np.array_equal(arr[: n - 4096].cpu().numpy(), exp[: n - 4096])
    # A ticket is collected once.
    with pytest.raises(rz.RedzoneError) as e:
        ctx.wait(tickets[0])
    assert e.value.code == _native.RZ_ERR_INVALID_ARG
    # A duplicate under RZ_VALIDATE comes back from rz_wait, with the list untouched.
    bad = idx[0].copy()
    bad[10] = bad[11]
    pb = torch.from_numpy(bad).pin_memory()
    t = ctx.remove_host_idx_async(b, pb, flags=rz.RZ_VALIDATE)
    with pytest.raises(rz.RedzoneError) as e:
        ctx.wait(t)
    assert e.value.code == _native.RZ_ERR_DUPLICATE
    assert torch.equal(b, torch.arange(n, dtype=torch.int32, device=DEV))
    # The context is usable afterwards.
    t = ctx.remove_host_idx_async(b, pinned[1])
    assert ctx.wait(t) == n - 4096
    exp = np.arange(n, dtype=np.int32)
    oracle.remove(exp, idx[1].astype(np.uint32))
    assert np.array_equal(b[: n - 4096].cpu().numpy(), exp[: n - 4096])


def test_async_errors_stay_with_their_call(ctx):
    """Each call has its own status word: a call rejected on the device (a repeated index under
    RZ_VALIDATE) reports it, and the calls issued around it, still in flight, report success and
    give the canonical result."""
    n, k = 1 << 18, 4096
    good = [workloads.uniform(n, k, seed=70 + s).astype(np.int32) for s in range(3)]
    bad = good[0].copy()
    bad[5] = bad[6]
    arrays = [torch.arange(n, dtype=torch.int32, device=DEV) for _ in range(4)]
    lists = [good[0], bad, good[1], good[2]]
    pinned = [torch.from_numpy(x).pin_memory() for x in lists]
    tickets = [ctx.remove_host_idx_async(arrays[0], pinned[0]),
               ctx.remove_host_idx_async(arrays[1], pinned[1], flags=rz.RZ_VALIDATE),
               ctx.remove_host_idx_async(arrays[2], pinned[2]),
               ctx.remove_host_idx_async(arrays[3], pinned[3])]
    results = []
    for t in tickets:
        try:
            results.append(ctx.wait(t))
        except rz.RedzoneError as e:
            results.append(-e.code)
    assert results == [n - k, -_native.RZ_ERR_DUPLICATE, n - k, n - k]
    assert torch.equal(arrays[1], torch.arange(n, dtype=torch.int32, device=DEV))  # rejected: untouched
    for j in (0, 2, 3):
        exp = np.arange(n, dtype=np.int32)
        oracle.remove(exp, lists[j].astype(np.uint32))
        assert np.array_equal(arrays[j][: n - k].cpu().numpy(), exp[: n - k])


@pytest.mark.parametrize("k", [1 << 10, 1 << 14, 1 << 18])
def test_async_error_reports_and_slot_reuse(ctx, k):
    """An out-of-range index in one call comes back from that call's rz_wait, whichever kernel ran
    (scan-all at 2^10, cluster scan at 2^14, the grid schedule at 2^18), and the calls issued
    after it on the same staging slots report success with the canonical result: the slot's
    status word, cleared on the call stream after the error, starts clean again."""
    n = 1 << 21
    calls = 20
    lists = [workloads.uniform(n, k, seed=500 + j).astype(np.int64) for j in range(calls)]
    bad_at = 3
    lists[bad_at][k // 2] = n + 5
    pinned = [torch.from_numpy(x.astype(np.uint32).view(np.int32)).pin_memory() for x in lists]
    arrays = [torch.arange(n, dtype=torch.int32, device=DEV) for _ in range(calls)]
    tickets = [ctx.remove_host_idx_async(a, x) for a, x in zip(arrays, pinned)]
    for j, t in enumerate(tickets):
        if j == bad_at:
            with pytest.raises(rz.RedzoneError) as e:
                ctx.wait(t)
            assert e.value.code == _native.RZ_ERR_OUT_OF_RANGE
        else:
            assert ctx.wait(t) == n - k
    for j in (0, bad_at + 1, bad_at + 8, calls - 1):
        exp = np.arange(n, dtype=np.int32)
        oracle.remove(exp, lists[j].astype(np.uint32))
        assert np.array_equal(arrays[j][: n - k].cpu().numpy(), exp[: n - k]), j
    # The same slots once more, one call at a time: every status word is zero.
    for j in range(10):
        b = torch.arange(n, dtype=torch.int32, device=DEV)
        assert ctx.wait(ctx.remove_host_idx_async(b, pinned[(j + 4) % calls])) == n - k


@pytest.mark.parametrize("k", [1 << 10, 1 << 14])
def test_async_validation_abort_reports_duplicate(ctx, k):
    """A repeated index under RZ_VALIDATE stops the removal kernel before it moves anything
    (scan-all at 2^10, cluster scan at 2^14: each kernel's own abort path), rz_wait returns
    RZ_ERR_DUPLICATE, the array is untouched, and the next call on the context succeeds."""
    n = 1 << 20
    good = workloads.uniform(n, k, seed=90 + k).astype(np.int32)
    bad = good.copy()
    bad[k // 2] = bad[k // 2 + 1]
    a = torch.arange(n, dtype=torch.int32, device=DEV)
    t = ctx.remove_host_idx_async(a, torch.from_numpy(bad).pin_memory(), flags=rz.RZ_VALIDATE)
    with pytest.raises(rz.RedzoneError) as e:
        ctx.wait(t)
    assert e.value.code == _native.RZ_ERR_DUPLICATE
    assert torch.equal(a, torch.arange(n, dtype=torch.int32, device=DEV))
    t = ctx.remove_host_idx_async(a, torch.from_numpy(good).pin_memory(), flags=rz.RZ_VALIDATE)
    assert ctx.wait(t) == n - k
    exp = np.arange(n, dtype=np.int32)
    oracle.remove(exp, good.astype(np.uint32))
    assert np.array_equal(a[: n - k].cpu().numpy(), exp[: n - k])
