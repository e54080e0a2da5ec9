"""GPU parity of the single-list Redzone kernels against the oracle, through the C-ABI."""
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from redzone_b200 import workloads
from tests import _golden, _torch_rule

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def payload(n, words, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 1 << 32, size=(n, words), dtype=np.uint64).astype(np.uint32)
    a[:, 0] = np.arange(n, dtype=np.uint32)
    return a


def run_gpu(ctx, host, idx, cfg=None, flags=rz.RZ_SYNC):
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    di = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    di_before = di.clone()
    if cfg is None:
        ctx.remove(d, di, flags=flags)
    else:
        ctx.remove_cfg(d, di, cfg, flags=flags)
    torch.cuda.synchronize()
    assert torch.equal(di, di_before), "the removal list must not be written"
    got = d.cpu().numpy().view(np.uint32)
    k = int(idx.size)
    assert np.array_equal(got[host.shape[0] - k:], host[host.shape[0] - k:]), "the tail must not be written"
    return got


def expect_of(host, idx):
    e = host.copy()
    oracle.remove(e, idx)
    return e


def test_golden_vectors(ctx):
    for case in _golden.cases():
        n, k = case["n"], case["k"]
        got = run_gpu(ctx, np.arange(n, dtype=np.uint32).reshape(n, 1), case["idx"])
        assert _golden.check_prefix(case, got[: n - k, 0].view(np.int32)), case


@pytest.mark.parametrize("words", [1, 2, 4, 8])
@pytest.mark.parametrize("dist", ["uniform", "clustered", "tail", "red50", "red100", "red0"])
def test_widths_and_distributions(ctx, words, dist):
    for n, k in [(1 << 12, 1 << 8), (1 << 16, 1 << 12), (1 << 20, 1 << 16), (300000, 256 * 100)]:
        if dist == "tail" and k > n // 10:
            continue
        if dist == "red0" and k > n // 2:
            continue
        host = payload(n, words, seed=n + k)
        idx = workloads.make(dist, n, k, seed=k)
        got = run_gpu(ctx, host, idx)
        exp = expect_of(host, idx)
        assert np.array_equal(got[: n - k], exp[: n - k]), (words, dist, n, k)
        assert np.array_equal(got[n - k:], host[n - k:]), "tail must be left untouched"


SCHEDULES = {"cluster": 2, "grid": 3, "cscan": 4, "split": 5, "scanall": 6}


@pytest.mark.parametrize("sched", ["cluster", "grid", "cscan", "split", "scanall"])
def test_every_launch_config_gives_the_same_bits(ctx, sched):
    """The result depends only on (data, idx), never on schedule, block, items or grid."""
    cases = [(1 << 20, 1 << 16, "uniform"), (1 << 18, 1 << 17, "red50"), (1 << 16, 3001, "red100")]
    for n, k, dist in cases:
        for words in (1, 4):
            host = payload(n, words, seed=5)
            idx = workloads.make(dist, n, k, seed=6)
            exp = expect_of(host, idx)
            for block in (128, 256, 512, 1024):
                for items in (1, 2, 4, 8):
                    for cps in (1, 2, 4):
                        cfg = rz.LaunchCfg(block, items, cps, 0, SCHEDULES[sched])
                        got = run_gpu(ctx, host, idx, cfg=cfg)
                        assert np.array_equal(got[: n - k], exp[: n - k]), (sched, n, k, dist, words, block, items, cps)


@pytest.mark.parametrize("sched", ["cluster", "grid", "cscan", "split", "scanall"])
@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_schedules_on_large_k(ctx, sched, words):
    n = 1 << 21
    for k in (1 << 18, 1 << 20, (1 << 20) + 12345):
        host = payload(n, words, seed=k)
        idx = workloads.uniform(n, k, seed=k)
        got = run_gpu(ctx, host, idx, cfg=rz.LaunchCfg(256, 4, 4, 0, SCHEDULES[sched]))
        assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k]), (sched, words, k)


def test_single_cta_schedule(ctx):
    for n, k in [(5000, 4000), (1 << 16, 1 << 14), (1 << 20, 1 << 17)]:
        host = payload(n, 2, seed=1)
        idx = workloads.uniform(n, k, seed=2)
        got = run_gpu(ctx, host, idx, flags=rz.RZ_SYNC | rz.RZ_FORCE_BLOCK)
        assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


@pytest.mark.parametrize("n,k", [(1, 0), (1, 1), (2, 1), (7, 7), (100, 0), (100, 99), (100, 1), (33, 32), (4097, 4096)])
def test_edge_sizes(ctx, n, k):
    host = payload(n, 1, seed=n)
    idx = workloads.uniform(n, k, seed=k)
    got = run_gpu(ctx, host, idx)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


def test_exhaustive_tiny_lists_every_schedule(ctx):
    """Every ordered removal list of every length for n <= 5, through the single-CTA, cluster and
    grid schedules (the grid with 32-item tiles, so n = 5 already spans CTAs only at k > 32 -- see
    the n = 64 case below), against the oracle."""
    import itertools
    schedules = [("block", None, rz.RZ_FORCE_BLOCK), ("auto", None, 0),
                 ("grid32", rz.LaunchCfg(32, 1, 4, 0, 3), rz.RZ_FORCE_GRID)]
    count = 0
    for n in range(1, 6):
        host = np.arange(100 * n, 100 * n + n, dtype=np.uint32).reshape(n, 1)
        for k in range(n + 1):
            for perm in itertools.permutations(range(n), k):
                idx = np.array(perm, dtype=np.uint32)
                exp = expect_of(host, idx)
                for name, cfg, flags in schedules:
                    got = run_gpu(ctx, host, idx, cfg=cfg, flags=flags | rz.RZ_SYNC)
                    assert np.array_equal(got[: n - k], exp[: n - k]), (name, n, perm)
                count += 1
    assert count == sum(len(list(itertools.permutations(range(n), k))) for n in range(1, 6) for k in range(n + 1))


@pytest.mark.parametrize("words", [1, 4])
def test_n64_every_k_multi_cta(ctx, words):
    """n = 64 with 32-item tiles: every k, several orders each, so grids of 1-2 CTAs run both the
    red-list and the bitmap paths (k = 64 .. 33 have up to 31 red entries per CTA)."""
    n = 64
    rng = np.random.default_rng(words)
    host = payload(n, words, seed=5)
    for k in range(n + 1):
        for rep in range(4):
            idx = rng.permutation(n)[:k].astype(np.uint32)
            exp = expect_of(host, idx)
            for cfg, fl in ((rz.LaunchCfg(32, 1, 4, 0, 3), rz.RZ_FORCE_GRID), (rz.LaunchCfg(32, 2, 4, 0, 3), rz.RZ_FORCE_GRID),
                            (rz.LaunchCfg(32, 1, 4, 0, 4), 0), (rz.LaunchCfg(32, 4, 1, 0, 4), 0),
                            (rz.LaunchCfg(32, 1, 1, 0, 5), 0), (rz.LaunchCfg(32, 1, 1, 0, 6), 0)):
                got = run_gpu(ctx, host, idx, cfg=cfg, flags=fl | rz.RZ_SYNC)
                assert np.array_equal(got[: n - k], exp[: n - k]), (words, k, rep, cfg)


def test_back_to_back_calls_leave_scratch_clean(ctx):
    """Bitmap and barrier state are self-cleaning: many calls in a row stay exact."""
    rng = np.random.default_rng(0)
    for it in range(30):
        n = int(rng.integers(1000, 1 << 20))
        k = int(rng.integers(1, n))
        host = payload(n, 1, seed=it)
        idx = workloads.uniform(n, k, seed=it)
        got = run_gpu(ctx, host, idx)
        assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k]), it


def test_split_schedule_back_to_back_and_under_graph_replay(ctx):
    """The split schedule's scan counter is reset by its own pairing grid: calls in a row, and one
    call captured in a CUDA graph replayed several times, stay exact."""
    cfg = rz.LaunchCfg(256, 4, 1, 0, 5)
    rng = np.random.default_rng(3)
    for it in range(10):
        n = int(rng.integers(1 << 12, 1 << 20))
        k = int(rng.integers(1, min(n, 1 << 17)))
        host = payload(n, 1, seed=it)
        idx = workloads.make("red50" if it % 3 == 0 else "uniform", n, k, seed=it)
        got = run_gpu(ctx, host, idx, cfg=cfg)
        assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k]), it
    n, k = 1 << 20, 1 << 15
    host = payload(n, 1, seed=40)
    idx = workloads.uniform(n, k, seed=40)
    exp = expect_of(host, idx)
    d0 = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    d = d0.clone()
    di = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ctx.remove_cfg(d, di, cfg, stream=s)  # first call outside the capture
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            ctx.remove_cfg(d, di, cfg, stream=s)
    for rep in range(3):
        d.copy_(d0)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32).reshape(n, 1)[: n - k], exp[: n - k]), rep
    del g


def test_validation_reports_and_leaves_data_untouched(ctx):
    n, k = 1 << 16, 1000
    host = payload(n, 1)
    idx = workloads.uniform(n, k, seed=1)
    dup = idx.copy()
    dup[10] = dup[500]
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    with pytest.raises(rz.RedzoneError) as e:
        ctx.remove(d, torch.from_numpy(dup.astype(np.int32)).to(DEV), flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
    assert e.value.code == 2
    assert np.array_equal(d.cpu().numpy().view(np.uint32), host)
    bad = idx.copy()
    bad[3] = n + 5
    with pytest.raises(rz.RedzoneError) as e:
        ctx.remove(d, torch.from_numpy(bad.astype(np.int32)).to(DEV), flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
    assert e.value.code == 3
    assert np.array_equal(d.cpu().numpy().view(np.uint32), host)
    # A valid call right after the failures still gives the exact result.
    got = run_gpu(ctx, host, idx, flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


@pytest.mark.parametrize("sched", [4, 5, 6])
def test_validation_on_the_cluster_scan_and_split_schedules(ctx, sched):
    """A failed validation on the cluster-scan schedule (whose CTAs still meet at every cluster
    barrier phase) or the split schedule (whose pairing CTAs still reset the scan's counter)
    leaves the data untouched, and the next call is exact."""
    n, k = 1 << 18, 1 << 14
    host = payload(n, 2, seed=9)
    idx = workloads.uniform(n, k, seed=9)
    cfg = rz.LaunchCfg(256, 4, 1, 0, sched)
    for bad_at, bad_val, code in ((100, None, 2), (7, n + 3, 3)):
        bad = idx.copy()
        bad[bad_at] = bad[bad_at + 1] if bad_val is None else bad_val
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        with pytest.raises(rz.RedzoneError) as e:
            ctx.remove_cfg(d, torch.from_numpy(bad.astype(np.int32)).to(DEV), cfg, flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
        assert e.value.code == code
        assert np.array_equal(d.cpu().numpy().view(np.uint32).reshape(n, 2), host)
    got = run_gpu(ctx, host, idx, cfg=cfg, flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


@pytest.mark.parametrize("block,items", [(128, 1), (256, 2)])
def test_validation_on_the_grid_schedule_with_many_tiles_per_cta(ctx, block, items):
    """The grid schedule with several tiles per CTA (its marking walks each CTA's whole index
    range at once): a duplicate or an out-of-range index under RZ_VALIDATE is reported and leaves
    the data untouched, and the next calls, validated or not, on a ragged k (no whole last tile)
    give the exact result."""
    n, k = 1 << 20, (1 << 17) + 77
    host = payload(n, 1, seed=21)
    idx = workloads.uniform(n, k, seed=21)
    cfg = rz.LaunchCfg(block, items, 1, 0, SCHEDULES["grid"])
    for bad_at, bad_val, code in ((k - 5, None, 2), (k // 2, n + 3, 3)):
        bad = idx.copy()
        bad[bad_at] = bad[bad_at - 1000] if bad_val is None else bad_val
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        with pytest.raises(rz.RedzoneError) as e:
            ctx.remove_cfg(d, torch.from_numpy(bad.astype(np.int32)).to(DEV), cfg, flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
        assert e.value.code == code
        assert np.array_equal(d.cpu().numpy().view(np.uint32), host)
    got = run_gpu(ctx, host, idx, cfg=cfg, flags=rz.RZ_VALIDATE | rz.RZ_SYNC)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])
    got = run_gpu(ctx, host, idx, cfg=cfg)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


def test_out_of_range_without_validation_is_memory_safe(ctx):
    """Bad indices never cause out-of-bounds accesses: an index >= n is ignored, reported."""
    n, k = 1 << 14, 512
    host = payload(n, 1)
    idx = workloads.uniform(n, k, seed=3).astype(np.int64)
    idx[7] = 0xFFFFFF00
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    with pytest.raises(rz.RedzoneError) as e:
        ctx.remove(d, torch.from_numpy(idx.astype(np.uint32).view(np.int32)).to(DEV), flags=rz.RZ_SYNC)
    assert e.value.code == 3


def test_partition_matches_stable_oracle(ctx):
    for words in (1, 2, 4, 8):
        for n, k in [(1000, 10), (1 << 18, 1 << 12), (1 << 20, 1 << 19), (123457, 1)]:
            host = payload(n, words, seed=words)
            idx = workloads.uniform(n, k, seed=n)
            d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
            ctx.partition(d, torch.from_numpy(idx.astype(np.int32)).to(DEV), flags=rz.RZ_SYNC)
            exp = host.copy()
            oracle.stable_remove(exp, idx)
            got = d.cpu().numpy().view(np.uint32)
            assert np.array_equal(got[: n - k], exp[: n - k]), (words, n, k)


def test_partition_many_tiles_per_cta(ctx):
    """Thousands of 32 KB tiles (several per CTA through the stage ring), clustered and uniform
    removals, a ragged end, and back-to-back calls on the same context (map left zero)."""
    cases = [(1, (1 << 24) + 5, "uniform", 1 << 16), (1, 1 << 24, "clustered", 1 << 22),
             (2, (1 << 22) + 3, "tail", 1 << 18), (4, 1 << 21, "uniform", 1 << 20)]
    for words, n, dist, k in cases:
        host = payload(n, words, seed=words + 7)
        idx = workloads.make(dist, n, k, seed=k)
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        ctx.partition(d, torch.from_numpy(idx.astype(np.int32)).to(DEV), flags=rz.RZ_SYNC)
        exp = host.copy()
        oracle.stable_remove(exp, idx)
        got = d.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[: n - k], exp[: n - k]), (words, n, dist, k)


@pytest.mark.parametrize("red", [0, 1, 2, 1023, 1024, 1025, 3000])
@pytest.mark.parametrize("words", [1, 4])
def test_red_list_schedule_around_its_limit(ctx, red, words):
    """Exactly `red` indices in the red zone [n-k, n): up to 1024 of them the grid derives the
    pairing from the published red list, above that it falls back to the bitmap exchange; the
    results are the canonical ones either way (default and 256x4 launch configurations)."""
    n, k = 1 << 20, 1 << 15
    cut = n - k
    rng = np.random.default_rng(red + 17 * words)
    idx = np.concatenate([rng.choice(cut, size=k - red, replace=False),
                          cut + rng.choice(k, size=red, replace=False)]).astype(np.uint32)
    rng.shuffle(idx)
    host = payload(n, words, seed=red)
    exp = expect_of(host, idx)
    for cfg in (None, rz.LaunchCfg(256, 4, 1, 0, 3), rz.LaunchCfg(128, 2, 4, 0, 3), rz.LaunchCfg(256, 4, 1, 0, 4),
                rz.LaunchCfg(128, 2, 4, 0, 4), rz.LaunchCfg(64, 1, 4, 0, 4), rz.LaunchCfg(256, 4, 1, 0, 5),
                rz.LaunchCfg(256, 1, 1, 0, 5), rz.LaunchCfg(256, 1, 1, 0, 6), rz.LaunchCfg(256, 4, 1, 0, 6)):
        got = run_gpu(ctx, host, idx, cfg=cfg)
        assert np.array_equal(got[: n - k], exp[: n - k]), (red, words, cfg)


@pytest.mark.parametrize("red", [255, 256, 257, 1024])
def test_cluster_scan_push_region_limit(ctx, red):
    """All `red` red entries in the first slice of the index list: up to 256 per slice the
    cluster-scan schedule pushes them to every cluster member, above that it ORs the partial maps;
    the results are the canonical ones either way."""
    n, k = 1 << 20, 1 << 15
    cut = n - k
    rng = np.random.default_rng(red)
    idx = np.concatenate([cut + rng.choice(k, size=red, replace=False),
                          rng.choice(cut, size=k - red, replace=False)]).astype(np.uint32)
    host = payload(n, 2, seed=red)
    exp = expect_of(host, idx)
    for cfg in (rz.LaunchCfg(256, 4, 1, 0, 4), rz.LaunchCfg(512, 1, 1, 0, 4)):
        got = run_gpu(ctx, host, idx, cfg=cfg)
        assert np.array_equal(got[: n - k], exp[: n - k]), (red, cfg)


def test_clobber_flag_is_accepted(ctx):
    """RZ_CLOBBER_INDICES (the reference's contract: the removal list may be overwritten) is
    accepted; the result is the canonical one and the list is still left as it was."""
    n, k = 1 << 18, 1 << 13
    host = payload(n, 1, seed=8)
    idx = workloads.uniform(n, k, seed=8)
    got = run_gpu(ctx, host, idx, flags=rz.RZ_SYNC | rz.RZ_CLOBBER_INDICES)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


def test_cluster_scan_with_an_unaligned_index_list(ctx):
    """An index list that does not start on a 16-byte boundary runs on another schedule instead
    (the cluster-scan and scan-all schedules read it in 16-byte units), with the same result."""
    n, k = 1 << 20, 1 << 14
    host = payload(n, 1, seed=4)
    idx = workloads.uniform(n, k, seed=4)
    buf = torch.from_numpy(np.concatenate([[0], idx]).astype(np.int32)).to(DEV)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    for sched in (4, 6):
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        ctx.remove_cfg(d, buf[1:], rz.LaunchCfg(256, 4, 1, 0, sched), flags=rz.RZ_SYNC)
        got = d.cpu().numpy().view(np.uint32).reshape(n, 1)
        assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k]), sched


def test_partition_more_tiles_than_one_scan_chunk(ctx):
    """n = 2^28 + 3 tiles + 77 int32 items: 32,772 tiles of 8192, so the offset scan runs two
    chunks with a carry; checked against a stable keep-mask compaction done by torch."""
    n = (1 << 28) + 3 * 8192 + 77
    k = 1 << 20
    a = torch.arange(n, dtype=torch.int32, device=DEV)
    g = torch.Generator(device=DEV)
    g.manual_seed(7)
    idx = torch.randperm(n, generator=g, device=DEV)[:k].to(torch.int32)
    keep = torch.ones(n, dtype=torch.bool, device=DEV)
    keep[idx.long()] = False
    exp = a[keep]
    ctx.partition(a, idx, flags=rz.RZ_SYNC)
    assert torch.equal(a[: n - k], exp)
    del a, exp, keep
    torch.cuda.empty_cache()


@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_preserve_list_compaction(ctx, words):
    """rz_keep: data[0..m) = old data[keep[j]] for sorted, unsorted, empty and full keep lists
    (reads from [0, m) included); the rest of the array is untouched; an entry >= n is skipped
    and reported."""
    rng = np.random.default_rng(words)
    n = (1 << 18) + 13
    for m, order in [(0, "sorted"), (1, "sorted"), (1000, "sorted"), (1 << 16, "random"), (n // 2, "sorted"),
                     (n, "random")]:
        host = payload(n, words, seed=m + words)
        keep = rng.choice(n, size=m, replace=False).astype(np.uint32)
        if order == "sorted":
            keep.sort()
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        new_len = ctx.keep(d, torch.from_numpy(keep.view(np.int32)).to(DEV), flags=rz.RZ_SYNC)
        assert new_len == m
        got = d.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[:m], host[keep]), (words, m, order)
        assert np.array_equal(got[m:], host[m:])
    keep = np.array([5, n + 7, 9], dtype=np.uint32)
    host = payload(n, words, seed=1)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    with pytest.raises(rz.RedzoneError) as e:
        ctx.keep(d, torch.from_numpy(keep.view(np.int32)).to(DEV), flags=rz.RZ_SYNC)
    assert e.value.code == 3
    got = d.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[0], host[5]) and np.array_equal(got[1], host[1]) and np.array_equal(got[2], host[9])


def test_append_then_remove(ctx):
    """Gains appended at the tail, then removal over the grown list (appended rows removable)."""
    for words, n, g, k in [(1, 1 << 18, 1 << 12, 1 << 13), (4, 5000, 300, 2000), (2, 1 << 16, 0, 100)]:
        cap = n + g + 17
        host = payload(cap, words, seed=n)
        gain = payload(g, words, seed=g + 1) if g else np.zeros((0, words), np.uint32)
        gain[:, 0] = 0xF0000000 + np.arange(g, dtype=np.uint32)
        idx = workloads.uniform(n + g, k, seed=k)
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        dg = torch.from_numpy(gain.view(np.int32).copy()).to(DEV)
        new_len = ctx.append_remove(d, n, dg, torch.from_numpy(idx.astype(np.int32)).to(DEV), flags=rz.RZ_SYNC)
        assert new_len == n + g - k
        grown = np.concatenate([host[:n], gain])
        oracle.remove(grown, idx)
        got = d.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[:new_len], grown[:new_len]), (words, n, g, k)
        assert np.array_equal(got[n + g:], host[n + g:])  # past the grown list: untouched


def test_allocation_failure_is_a_status_and_changes_nothing():
    """Injected allocation failure: with a scratch cap of 0 bytes a fresh context cannot grow its
    scratch, so the call returns RZ_ERR_NO_MEMORY with the data untouched; lifting the cap makes
    the same context work."""
    c = rz.Context(0)
    n, k = 1 << 16, 1 << 12
    host = payload(n, 1, seed=3)
    idx = workloads.uniform(n, k, seed=4)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    di = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    c.set_scratch_limit(0)
    for call in (lambda: c.remove(d, di, flags=rz.RZ_SYNC), lambda: c.partition(d, di, flags=rz.RZ_SYNC),
                 lambda: c.keep(d, di, flags=rz.RZ_SYNC)):
        with pytest.raises(rz.RedzoneError) as e:
            call()
        assert e.value.code == 4  # RZ_ERR_NO_MEMORY
    assert c.scratch_bytes == 0
    assert np.array_equal(d.cpu().numpy().view(np.uint32), host)
    c.set_scratch_limit(None)
    assert c.remove(d, di, flags=rz.RZ_SYNC) == n - k
    assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], expect_of(host, idx)[: n - k])
    assert c.scratch_bytes > 0
    c.close()


def test_bounded_barrier_wait_times_out_with_status(ctx):
    bits = ctx.test_barrier_timeout(spin_limit=2000)
    assert bits & 4
    # The context is usable afterwards.
    host = payload(1 << 16, 1)
    idx = workloads.uniform(1 << 16, 1 << 12, seed=1)
    got = run_gpu(ctx, host, idx)
    assert np.array_equal(got[: (1 << 16) - (1 << 12)], expect_of(host, idx)[: (1 << 16) - (1 << 12)])


def test_host_index_entry_point(ctx):
    n, k = 1 << 20, 1 << 14
    host = payload(n, 1)
    idx = workloads.uniform(n, k, seed=8)
    d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
    pinned = torch.from_numpy(idx.astype(np.int32)).pin_memory()
    new_len = ctx.remove_host_idx(d, pinned)
    assert new_len == n - k
    got = d.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[: n - k], expect_of(host, idx)[: n - k])


def test_reference_shaped_call():
    n, k = 1 << 16, 1 << 10
    a = torch.arange(n, dtype=torch.int32, device=DEV)
    idx = workloads.uniform(n, k, seed=4)
    r = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    new_len = rz.RemoveFromList(a, n, r, k, flags=rz.RZ_SYNC)
    assert new_len == n - k
    e = np.arange(n, dtype=np.int32)
    oracle.remove(e, idx)
    assert np.array_equal(a.cpu().numpy()[: n - k], e[: n - k])


def test_torch_rule_matches_oracle():
    n, k = 1 << 18, 1 << 15
    host = payload(n, 1)
    idx = workloads.red_split(n, k, seed=3, red_percentage=40)
    t = _torch_rule.canonical_prefix(torch.from_numpy(host.view(np.int32)).to(DEV),
                                     torch.from_numpy(idx.astype(np.int64)).to(DEV))
    assert np.array_equal(t.cpu().numpy().view(np.uint32), expect_of(host, idx)[: n - k])


@pytest.mark.parametrize("k_log2,dist", [(16, "uniform"), (24, "tail"), (26, "uniform"), (27, "uniform"), (20, "clustered")])
def test_full_size_n_2_28(ctx, k_log2, dist):
    """n = 2^28 int32 iota (the large-list benchmark size): bit-exact against the torch
    statement of the rule plus isOK_CPU's survivor properties."""
    n, k = 1 << 28, 1 << k_log2
    a = torch.arange(n, dtype=torch.int32, device=DEV)
    idx = workloads.make_torch(dist, n, k, seed=k_log2)
    exp = _torch_rule.canonical_prefix(a, idx)
    ctx.remove(a, idx, flags=rz.RZ_SYNC)
    assert torch.equal(a[: n - k], exp)
    props = _torch_rule.survivor_properties(a[: n - k], n, idx)
    assert all(props.values()), props
    del a, exp
    torch.cuda.empty_cache()


@pytest.mark.parametrize("log2n,log2k,words,dist", [(26, 18, 1, "uniform"), (28, 19, 1, "uniform"),
                                                    (26, 18, 4, "uniform"), (24, 19, 1, "uniform"),
                                                    (26, 18, 1, "tail")])
def test_redlist_schedule_beyond_2e17(ctx, log2n, log2k, words, dist):
    """The grid kernel's red-list schedule for 2^17 < k <= 2^19 (k-bit maps of up to 128 KB in
    shared memory; chosen when k^2/n <= 1024), and the cases that fall back to the bitmap phases
    (more red entries: n = 2^24 with k = 2^19, tail-heavy removals) -- bit-exact against the
    vectorised rule, with every launch configuration of the grid schedule at this size."""
    n, k = 1 << log2n, 1 << log2k
    a0 = torch.zeros((n, words), dtype=torch.int32, device=DEV)
    a0[:, 0] = torch.arange(n, dtype=torch.int32, device=DEV)
    idx = workloads.make_torch(dist, n, k, seed=log2n * 100 + log2k).contiguous()
    exp = _torch_rule.canonical_prefix(a0, idx)
    for cfg in [None, rz.LaunchCfg(896, 4, 2, 0, 0), rz.LaunchCfg(1024, 4, 1, 0, 0), rz.LaunchCfg(512, 8, 2, 0, 0)]:
        a = a0.clone()
        if cfg is None:
            ctx.remove(a, idx, flags=rz.RZ_SYNC)
        else:
            ctx.remove_cfg(a, idx, cfg, flags=rz.RZ_SYNC)
        assert torch.equal(a[: n - k], exp), (log2n, log2k, words, dist, cfg)
        del a
    del a0, exp
    torch.cuda.empty_cache()
