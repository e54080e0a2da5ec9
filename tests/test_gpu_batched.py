"""GPU parity of the batched (one persistent launch, graph-replayed) path against the oracle."""
import ctypes

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


def make_lists(seed, nlists, log2_lo, log2_hi, words, f_hi=0.5):
    n, k = workloads.batched_lists(nlists, seed, log2_lo, log2_hi, 0.001, f_hi)
    rng = np.random.default_rng(seed + 1)
    hosts, idxs = [], []
    for l in range(nlists):
        h = rng.integers(0, 1 << 32, size=(int(n[l]), words), dtype=np.uint64).astype(np.uint32)
        h[:, 0] = np.arange(int(n[l]), dtype=np.uint32)
        hosts.append(h)
        idxs.append(workloads.uniform(int(n[l]), int(k[l]), seed * 100003 + l))
    return hosts, idxs


def to_dev(hosts, idxs):
    return [(torch.from_numpy(h.view(np.int32).copy()).to(DEV), torch.from_numpy(i.astype(np.int32)).to(DEV))
            for h, i in zip(hosts, idxs)]


def expected(hosts, idxs, times=1):
    out = []
    for h, i in zip(hosts, idxs):
        e = h.copy()
        for _ in range(times):
            oracle.remove(e, i)
        out.append(e)
    return out


@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_batched_matches_per_list_oracle(ctx, words):
    hosts, idxs = make_lists(7 + words, 300, 2, 17, words)
    dl = to_dev(hosts, idxs)
    rz.remove_batched(ctx, dl)
    torch.cuda.synchronize()
    for l, (exp, (d, _)) in enumerate(zip(expected(hosts, idxs), dl)):
        n, k = exp.shape[0], idxs[l].size
        got = d.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[: n - k], exp[: n - k]), (words, l, n, k)


@pytest.mark.parametrize("block,items,cps,wave", [(128, 2, 1, 0), (256, 8, 4, 0), (512, 4, 2, 0), (256, 1, 8, 0),
                                                  (128, 2, 1, 1), (256, 8, 4, 6), (512, 4, 2, 2), (256, 2, 4, 6)])
def test_batched_configs_and_graph_replay(ctx, block, items, cps, wave):
    """Every tile/grid choice and both work orders (phase by phase, wavefront with several lags)
    give the same bits, and a second graph replay (on the compacted arrays) equals applying the
    rule twice."""
    hosts, idxs = make_lists(3, 120, 3, 16, 2, f_hi=0.3)
    dl = to_dev(hosts, idxs)
    plan = rz.BatchPlan(ctx, dl, _native.BatchCfg(block, items, cps, 0, wave))
    plan.launch()
    torch.cuda.synchronize()
    assert ctx.sync_status() == 0
    exp1 = expected(hosts, idxs, 1)
    for l, (d, _) in enumerate(dl):
        n, k = exp1[l].shape[0], idxs[l].size
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], exp1[l][: n - k]), (l, "first")
    plan.launch()
    torch.cuda.synchronize()
    exp2 = expected(hosts, idxs, 2)
    for l, (d, _) in enumerate(dl):
        n, k = exp2[l].shape[0], idxs[l].size
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], exp2[l][: n - k]), (l, "replay")
    plan.close()


def test_batched_edge_lists(ctx):
    specs = [(1, 0), (1, 1), (2, 1), (5, 5), (100, 0), (4096, 4095), (3, 2), (70000, 35000), (33, 1)]
    hosts = [np.arange(n, dtype=np.uint32).reshape(n, 1) for n, _ in specs]
    idxs = [workloads.uniform(n, k, n + k) for n, k in specs]
    dl = to_dev(hosts, idxs)
    rz.remove_batched(ctx, dl)
    torch.cuda.synchronize()
    for l, exp in enumerate(expected(hosts, idxs)):
        n, k = specs[l]
        assert np.array_equal(dl[l][0].cpu().numpy().view(np.uint32)[: n - k], exp[: n - k]), specs[l]


def test_batched_large_lists_with_many_chunks(ctx):
    """Lists up to 2^22 items with k up to n/2 (the biggest lists of the 4096-list workload)."""
    hosts, idxs = [], []
    for q, (n, k) in enumerate([(1 << 22, 1 << 21), (3_000_000, 123_457), (1 << 20, 1 << 19), (1 << 18, 10)]):
        hosts.append(np.arange(n, dtype=np.uint64).astype(np.uint32).reshape(n, 1).repeat(2, axis=1))
        idxs.append(workloads.uniform(n, k, q))
    dl = to_dev(hosts, idxs)
    rz.remove_batched(ctx, dl)
    torch.cuda.synchronize()
    for l, exp in enumerate(expected(hosts, idxs)):
        n, k = exp.shape[0], idxs[l].size
        assert np.array_equal(dl[l][0].cpu().numpy().view(np.uint32)[: n - k], exp[: n - k]), l


def test_batched_rejects_misaligned_lists(ctx):
    """A list whose items are not aligned to their width (or whose index list is not 4-byte
    aligned) is refused on the host with RZ_ERR_INVALID_ARG before anything is launched, and
    the context stays usable."""
    raw = torch.zeros(4096 * 2 + 2, dtype=torch.int32, device=DEV)
    idx = torch.arange(0, 4096, 4, dtype=torch.int32, device=DEV)
    arr = (_native.ListDesc * 1)()
    arr[0].data = raw.data_ptr() + 4  # 8-byte items at a 4-byte offset
    arr[0].idx = idx.data_ptr()
    arr[0].n = 4096
    arr[0].k = idx.numel()
    plan = ctypes.c_void_p()
    st = _native.lib.rz_batch_plan_create(ctx.handle, arr, 1, 8, None, ctypes.byref(plan))
    assert st == _native.RZ_ERR_INVALID_ARG
    hosts, idxs = make_lists(3, 8, 10, 14, 2)
    lists = to_dev(hosts, idxs)
    plan = rz.BatchPlan(ctx, lists)
    plan.launch()
    torch.cuda.synchronize()
    assert ctx.sync_status() == 0
    for (d, _), e, i in zip(lists, expected(hosts, idxs), idxs):
        n, k = d.shape[0], i.size
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], e[: n - k])
    plan.close()
