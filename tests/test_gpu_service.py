"""Streaming delete service: continuous batching gives every shard the same result as applying
its batches alone, lengths are tracked on the device, admission is bounded by memory."""
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from redzone_b200 import _native

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
SHARDS, CAP, WORDS = 8, 1 << 15, 8  # 8 shards x 32768 records of 32 bytes
FLOOR = CAP // 2


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def initial_table():
    t = np.zeros((SHARDS * CAP, WORDS), np.uint32)
    t[:, 0] = np.arange(SHARDS * CAP, dtype=np.uint32)
    t[:, 2] = 0xABCD
    return t


def batches(seed, count, max_log2=11):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        k = int(round(2 ** rng.uniform(0, max_log2)))
        out.append((int(rng.integers(0, SHARDS)), rng.choice(FLOOR, size=k, replace=False).astype(np.uint32)))
    return out


def run_service(ctx, seq, slots, max_batches, one_at_a_time):
    table = torch.from_numpy(initial_table().view(np.int32)).to(DEV)
    svc = rz.Service(ctx, table, SHARDS, CAP, slots=slots, max_batches_per_launch=max_batches,
                     index_budget_bytes=8 << 20, floor_rows=FLOOR)
    for shard, idx in seq:
        svc.submit(shard, idx)
        if one_at_a_time:
            svc.drain()
    svc.drain()
    host_len, dev_len = svc.lengths()
    stats = svc.stats()
    svc.close()
    torch.cuda.synchronize()
    return table.cpu().numpy().view(np.uint32).reshape(SHARDS, CAP, WORDS), host_len, dev_len, stats


def fill_rows(s, start_count, g):
    """The records the service appends on a refill (same formula as its fill kernel)."""
    key = (np.uint64(s) << np.uint64(40)) + np.uint64(start_count) + np.arange(g, dtype=np.uint64)
    r = np.zeros((g, WORDS), np.uint32)
    r[:, 0] = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    r[:, 1] = (key >> np.uint64(32)).astype(np.uint32)
    h = key * np.uint64(0x9E3779B97F4A7C15)
    for q in range(2, WORDS):
        r[:, q] = ((h >> np.uint64(8 * (q & 3))) & np.uint64(0xFFFFFFFF)).astype(np.uint32) ^ np.uint32(q)
    return r


def oracle_tables(seq):
    t = initial_table().reshape(SHARDS, CAP, WORDS)
    lens = [CAP] * SHARDS
    appended = [0] * SHARDS
    for s, idx in seq:
        if lens[s] - idx.size < FLOOR:
            g = CAP - lens[s]
            if g > 0:
                t[s, lens[s]:CAP] = fill_rows(s, appended[s], g)
                appended[s] += g
                lens[s] = CAP
        view = t[s, : lens[s]].copy()
        oracle.remove(view, idx)
        t[s, : lens[s]] = view
        lens[s] -= idx.size
    return t, lens


def test_each_result_is_the_same_alone_and_in_the_mix(ctx):
    seq = batches(1, 300)
    mix, mlen, mdev, mstats = run_service(ctx, seq, slots=4, max_batches=8, one_at_a_time=False)
    alone, alen, adev, astats = run_service(ctx, seq, slots=1, max_batches=1, one_at_a_time=True)
    assert mlen == alen == mdev == adev
    for s in range(SHARDS):
        assert np.array_equal(mix[s, : mlen[s]], alone[s, : alen[s]]), s
    assert mstats["completed"] == astats["completed"] == len(seq)
    assert astats["mean_batches_per_launch"] == 1.0
    # The mix really coalesced and overlapped work (more than one batch per launch on average).
    assert mstats["mean_batches_per_launch"] > 1.0
    exp, elen = oracle_tables(seq)
    assert elen == mlen
    for s in range(SHARDS):
        assert np.array_equal(mix[s, : mlen[s]], exp[s, : elen[s]]), s


def test_checkpoint_and_resume_give_the_same_tables(ctx):
    """Checkpoint half-way (lengths, refill counters, the caller's copy of its table), resume in a
    new service, apply the second half: the tables equal those of one uninterrupted run."""
    seq = batches(21, 1200)  # ~268 rows per batch: each shard refills after ~61 of its batches
    first, second = seq[:700], seq[700:]
    full, flen, _, _ = run_service(ctx, seq, slots=4, max_batches=8, one_at_a_time=False)

    table = torch.from_numpy(initial_table().view(np.int32)).to(DEV)
    svc = rz.Service(ctx, table, SHARDS, CAP, slots=4, max_batches_per_launch=8, index_budget_bytes=8 << 20,
                     floor_rows=FLOOR)
    for shard, idx in first:
        svc.submit(shard, idx)
    lengths, appended = svc.checkpoint()
    saved = table.cpu().clone()  # the caller's own copy of its table
    svc.close()
    assert any(a > 0 for a in appended)  # refills happened before the checkpoint

    table2 = saved.to(DEV)
    svc2 = rz.Service(ctx, table2, SHARDS, CAP, slots=2, max_batches_per_launch=4, index_budget_bytes=8 << 20,
                      floor_rows=FLOOR)
    svc2.restore(lengths, appended)
    for shard, idx in second:
        svc2.submit(shard, idx)
    svc2.drain()
    h, d = svc2.lengths()
    svc2.close()
    torch.cuda.synchronize()
    assert h == d == flen
    got = table2.cpu().numpy().view(np.uint32).reshape(SHARDS, CAP, WORDS)
    for s in range(SHARDS):
        assert np.array_equal(got[s, : h[s]], full[s, : flen[s]]), s


def test_statistics_and_admission_limit(ctx):
    table = torch.zeros((SHARDS * CAP, WORDS), dtype=torch.int32, device=DEV)
    svc = rz.Service(ctx, table, SHARDS, CAP, slots=2, max_batches_per_launch=4, index_budget_bytes=2 * 4 * 1000,
                     floor_rows=FLOOR)
    with pytest.raises(rz.RedzoneError) as e:  # 1001 indices never fit a 1000-index slot
        svc.submit(0, np.arange(1001, dtype=np.uint32))
    assert e.value.code == _native.RZ_ERR_BUSY
    for s, idx in batches(5, 50, max_log2=9):
        svc.submit(s, idx)
    svc.drain()
    st = svc.stats()
    assert st["completed"] == 50 and st["rejected"] == 1
    assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
    h, d = svc.lengths()
    assert h == d
    svc.close()


def test_poisson_load_generator(ctx):
    table = torch.zeros((SHARDS * CAP, WORDS), dtype=torch.int32, device=DEV)
    svc = rz.Service(ctx, table, SHARDS, CAP, slots=4, max_batches_per_launch=16, index_budget_bytes=8 << 20,
                     floor_rows=FLOOR)
    pool = [torch.from_numpy(idx.astype(np.int32)).pin_memory() for _, idx in batches(9, 64)]
    st = svc.run_poisson(pool, rate=5000.0, seconds=0.2, seed=3)
    assert st["completed"] == st["submitted"] > 500
    h, d = svc.lengths()
    assert h == d and all(FLOOR <= x <= CAP for x in h)
    svc.close()
