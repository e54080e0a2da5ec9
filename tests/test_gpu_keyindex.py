"""Delete-by-key through the key -> row index: the table after each removal is the canonical
result for the rows those keys occupied (checked against the oracle), and the index maps every
live key to its current row and every deleted key to nothing."""
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from redzone_b200 import _native

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def make_table(n, words, seed):
    rng = np.random.default_rng(seed)
    # Distinct 61-bit keys: an odd multiplier is a bijection modulo 2^61.
    keys = (np.arange(n, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)) & np.uint64((1 << 61) - 1)
    keys = keys[rng.permutation(n)]
    t = np.zeros((n, words), np.uint32)
    t[:, 0] = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    t[:, 1] = (keys >> np.uint64(32)).astype(np.uint32)
    if words > 2:
        t[:, 2] = np.arange(n, dtype=np.uint32)
    return t


def keys_of(rows2d):
    return rows2d[:, 0].astype(np.uint64) | (rows2d[:, 1].astype(np.uint64) << np.uint64(32))


def dev_keys(k64):
    return torch.from_numpy(k64.view(np.int64).copy()).to(DEV)


@pytest.mark.parametrize("words", [2, 4, 8])
def test_remove_by_key_keeps_table_and_index_exact(ctx, words):
    n0 = (1 << 16) + 5
    host = make_table(n0, words, seed=words)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    ix = rz.KeyIndex(ctx, 1 << 18)
    ix.build(d)
    rng = np.random.default_rng(100 + words)
    n = n0
    for k in (1, 7, 300, 5000, 20000, 1):
        live = keys_of(host[:n])
        pick = rng.choice(n, size=k, replace=False)
        if k > 10:
            pick[:3] = [n - 1, n - 2, 0]  # rows at the very end and the very start
            pick = np.unique(pick)
            rng.shuffle(pick)
            k = pick.size
        new_n = ix.remove_by_key(d, n, dev_keys(live[pick]), flags=rz.RZ_SYNC)
        assert new_n == n - k
        exp = host[:n].copy()
        oracle.remove(exp, pick.astype(np.uint32))
        host[: n - k] = exp[: n - k]
        n -= k
        got = d.cpu().numpy().view(np.uint32).reshape(n0, words)
        assert np.array_equal(got[:n], host[:n]), (words, k)
        rows = ix.find(dev_keys(keys_of(host[:n]))).cpu().numpy()
        assert np.array_equal(rows, np.arange(n)), (words, k)
        assert np.all(ix.find(dev_keys(live[pick])).cpu().numpy() == -1)
    ix.close()


def test_remove_by_key_rejects_missing_and_repeated_keys(ctx):
    n, words = 4096, 4
    host = make_table(n, words, seed=7)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    ix = rz.KeyIndex(ctx, 1 << 14)
    ix.build(d)
    live = keys_of(host)
    missing = np.array([live[3], np.uint64(12345678901)], dtype=np.uint64)  # the second is not in the table
    with pytest.raises(rz.RedzoneError) as e:
        ix.remove_by_key(d, n, dev_keys(missing), flags=rz.RZ_SYNC)
    assert e.value.code == _native.RZ_ERR_OUT_OF_RANGE
    with pytest.raises(rz.RedzoneError) as e:
        ix.remove_by_key(d, n, dev_keys(np.array([live[5], live[9], live[5]], dtype=np.uint64)), flags=rz.RZ_SYNC)
    assert e.value.code == _native.RZ_ERR_DUPLICATE
    assert np.array_equal(d.cpu().numpy().view(np.uint32).reshape(n, words), host)  # nothing moved
    assert np.array_equal(ix.find(dev_keys(live)).cpu().numpy(), np.arange(n))  # index unchanged
    dup = host.copy()
    dup[10, :2] = dup[20, :2]
    with pytest.raises(rz.RedzoneError) as e:
        ix.build(torch.from_numpy(dup.view(np.int32)).to(DEV))
    assert e.value.code == _native.RZ_ERR_DUPLICATE
    ix.close()


def test_insert_after_append_then_remove_by_key(ctx):
    cap, words = 10000, 4
    n = 6000
    host = make_table(cap, words, seed=11)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    ix = rz.KeyIndex(ctx, 1 << 15)
    ix.build(d, n)
    ix.insert(d, n, 3000)  # rows appended earlier at [n, n + 3000)
    n += 3000
    live = keys_of(host[:n])
    rng = np.random.default_rng(3)
    pick = rng.choice(n, size=2500, replace=False)
    assert ix.remove_by_key(d, n, dev_keys(live[pick]), flags=rz.RZ_SYNC) == n - 2500
    exp = host[:n].copy()
    oracle.remove(exp, pick.astype(np.uint32))
    n -= 2500
    got = d.cpu().numpy().view(np.uint32).reshape(cap, words)
    assert np.array_equal(got[:n], exp[:n])
    assert np.array_equal(ix.find(dev_keys(keys_of(exp[:n]))).cpu().numpy(), np.arange(n))
    ix.close()
