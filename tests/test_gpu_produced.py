"""GPU parity of removal lists made on the GPU with fused red-zone marking (rz_producer_*,
rz_remove_produced): every result is checked against the oracle applied to the list the producer
actually wrote (read back), and against rz_remove on that same list."""
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def payload(n, words, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 1 << 32, size=(n, words), dtype=np.uint64).astype(np.uint32)
    a[:, 0] = np.arange(n, dtype=np.uint32)
    return a


def keys_for(n, k, seed, tail_heavy=False):
    """uint32 keys of which exactly k are below the threshold 2^31 (the rows to delete)."""
    rng = np.random.default_rng(seed)
    keys = rng.integers(1 << 31, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    if tail_heavy:  # most deletions in the last rows: many red entries
        pool = np.arange(n - 2 * k, n) if 2 * k <= n else np.arange(n)
        rows = rng.choice(pool, size=k, replace=False)
    else:
        rows = rng.choice(n, size=k, replace=False)
    keys[rows] = rng.integers(0, 1 << 31, size=k, dtype=np.uint64).astype(np.uint32)
    return keys


def run_round(ctx, prod, host, keys, flags=rz.RZ_SYNC):
    n = host.shape[0]
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    dk = torch.from_numpy(keys.view(np.int32)).to(DEV)
    prod.reset(n)
    prod.produce_where_less(dk, 1 << 31)
    lst, k, cands = prod.download()
    new_len = prod.remove(d, flags=flags)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.uint32).reshape(host.shape)
    exp = host.copy()
    oracle.remove(exp, lst)
    assert new_len == n - k
    assert sorted(lst.tolist()) == sorted(np.flatnonzero(keys < (1 << 31)).tolist())
    assert np.array_equal(got[: n - k], exp[: n - k]), (n, k, cands)
    assert np.array_equal(got[n - k:], host[n - k:]), "the tail must not be written"
    # The same list through the index-list entry point gives the same bits.
    d2 = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    ctx.remove(d2, torch.from_numpy(lst.view(np.int32)).to(DEV), flags=rz.RZ_SYNC)
    assert torch.equal(d2, d)
    return k, cands


@pytest.mark.parametrize("words", [1, 4])
@pytest.mark.parametrize("n,k", [(1 << 20, 1 << 14), (1 << 20, 1 << 16), (300001, 20000), (5000, 4000), (64, 33)])
def test_produced_matches_oracle(ctx, words, n, k):
    prod = rz.Producer(ctx, capacity=max(k, 64), cand_capacity=4096)
    host = payload(n, words, seed=n + k)
    run_round(ctx, prod, host, keys_for(n, k, seed=k))
    prod.close()


@pytest.mark.parametrize("tail_heavy", [False, True])
def test_candidate_overflow_reads_the_whole_list(ctx, tail_heavy):
    """With a candidate buffer too small, every CTA reads the whole list instead: same bits."""
    n, k = 1 << 18, 1 << 14
    prod = rz.Producer(ctx, capacity=k, cand_capacity=4)
    k_, cands = run_round(ctx, prod, payload(n, 2, seed=3), keys_for(n, k, seed=4, tail_heavy=tail_heavy))
    assert cands > 4
    prod.close()


@pytest.mark.parametrize("red", ["few", "some", "many"])
def test_red_entry_regimes(ctx, red):
    """<= 32 red entries (one warp ranks them), 33..1024 (ranked by the P map's word prefix) and
    more than 1024 (the map-only path)."""
    n, k = 1 << 18, 1 << 13
    rng = np.random.default_rng(11)
    keys = rng.integers(1 << 31, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    nred = {"few": 20, "some": 500, "many": 3000}[red]
    rows = np.concatenate([rng.choice(n - k, size=k - nred, replace=False), n - k + rng.choice(k, size=nred, replace=False)])
    keys[rows] = 7
    prod = rz.Producer(ctx, capacity=k, cand_capacity=8192)
    run_round(ctx, prod, payload(n, 1, seed=12), keys)
    prod.close()


def test_rounds_on_a_shrinking_list(ctx):
    """Several rounds on the same table, each on the list the previous one left."""
    n, words = 1 << 19, 2
    host = payload(n, words, seed=21)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    prod = rz.Producer(ctx, capacity=1 << 15, cand_capacity=2048)
    cur = host.copy()
    rng = np.random.default_rng(22)
    for r in range(6):
        m = cur.shape[0]
        k = int(rng.integers(1, 1 << 15))
        keys = keys_for(m, k, seed=100 + r)
        prod.reset(m)
        prod.produce_where_less(torch.from_numpy(keys.view(np.int32)).to(DEV), 1 << 31)
        lst, kk, _ = prod.download()
        assert kk == k
        assert prod.remove(d, flags=rz.RZ_SYNC) == m - k
        oracle.remove(cur, lst)
        cur = cur[: m - k].copy()
        got = d.cpu().numpy().view(np.uint32).reshape(n, words)[: m - k]
        assert np.array_equal(got, cur), r
    prod.close()


def test_empty_round_and_validation(ctx):
    n = 1 << 16
    host = payload(n, 1, seed=5)
    prod = rz.Producer(ctx, capacity=1 << 12)
    keys = np.full(n, 0xFFFFFFFF, np.uint32)  # nothing below the threshold
    k, _ = run_round(ctx, prod, host, keys)
    assert k == 0
    run_round(ctx, prod, host, keys_for(n, 1000, seed=6), flags=rz.RZ_SYNC | rz.RZ_VALIDATE)
    prod.close()


def test_capacity_exceeded_moves_nothing(ctx):
    n, k = 1 << 16, 5000
    host = payload(n, 1, seed=7)
    prod = rz.Producer(ctx, capacity=4096)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    prod.reset(n)
    prod.produce_where_less(torch.from_numpy(keys_for(n, k, seed=8).view(np.int32)).to(DEV), 1 << 31)
    with pytest.raises(rz.RedzoneError) as e:
        prod.remove(d, flags=rz.RZ_SYNC)
    assert e.value.code == 4
    assert np.array_equal(d.cpu().numpy().view(np.uint32), host)
    # The context is usable afterwards.
    run_round(ctx, prod, host, keys_for(n, 3000, seed=9))
    prod.close()


def test_producer_with_unaligned_keys(ctx):
    """Keys that do not start on a 16-byte boundary take the one-key loop: same rows emitted."""
    n, k = 100003, 3000
    keys = keys_for(n, k, seed=31)
    buf = torch.from_numpy(np.concatenate([[0], keys]).astype(np.uint32).view(np.int32)).to(DEV)
    prod = rz.Producer(ctx, capacity=4096)
    prod.reset(n)
    prod.produce_where_less(buf[1:], 1 << 31)
    lst, kk, _ = prod.download()
    assert kk == k and sorted(lst.tolist()) == sorted(np.flatnonzero(keys < (1 << 31)).tolist())
    prod.close()
