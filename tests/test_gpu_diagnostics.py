"""The measurement aids the benchmark relies on: rz_test_scatter stores exactly the items it is
given at exactly the positions it is given (so the scatter floor times real hole writes), and
rz_test_empty_launch launches the shapes the removals use."""
import numpy as np
import pytest
import torch

import redzone_b200 as rz
from redzone_b200 import _native, workloads

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("words", [1, 2, 4, 8])
def test_scatter_writes_each_position_once(ctx, words):
    n, k = 1 << 18, 5000
    a = torch.full((n, words), -1, dtype=torch.int32, device=DEV)
    pos = workloads.uniform(n, k, seed=words).astype(np.int64)
    pos_with_bad = np.concatenate([pos, [n + 5]]).astype(np.uint32)  # a position >= n is skipped
    ctx.scatter(a, torch.from_numpy(pos_with_bad.view(np.int32)).to(DEV))
    torch.cuda.synchronize()
    got = a.cpu().numpy().view(np.uint32)
    i = np.arange(k, dtype=np.uint32)
    expect_first = np.where(np.arange(words) % 2 == 0, i[:, None], ~i[:, None])
    assert np.array_equal(got[pos], expect_first)
    untouched = np.ones(n, bool)
    untouched[pos] = False
    assert (got[untouched] == 0xFFFFFFFF).all()


def test_empty_launch_shapes(ctx):
    for grid, block, cluster in [(64, 256, 8), (148, 512, 1), (16, 1024, 4)]:
        ctx.empty_launch(grid, block, cluster)
    torch.cuda.synchronize()
    with pytest.raises(rz.RedzoneError) as e:
        ctx.empty_launch(10, 256, 8)  # cluster does not divide the grid
    assert e.value.code == _native.RZ_ERR_INVALID_ARG


def test_thrust_comparator_is_the_stable_remove(ctx):
    import oracle
    for n, k in [(1000, 10), (1 << 20, 1 << 16), (1 << 18, 1 << 17)]:
        idx = workloads.uniform(n, k, seed=n)
        a = torch.arange(n, dtype=torch.int32, device=DEV)
        new_len = ctx.thrust_remove(a, torch.from_numpy(idx.astype(np.int32)).to(DEV))
        torch.cuda.synchronize()
        exp = np.arange(n, dtype=np.uint32)
        oracle.stable_remove(exp, idx)
        assert new_len == n - k
        assert np.array_equal(a.cpu().numpy().view(np.uint32)[: n - k], exp[: n - k])
