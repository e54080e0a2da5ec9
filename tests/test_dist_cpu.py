"""The N > 1 plumbing on CPU: two gloo ranks (one process each) run independent replicas, reduce
their times with max-over-ranks and their work with a sum, and partition batched lists by weight."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from redzone_b200 import dist


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import torch.distributed as tdist

    import oracle
    from redzone_b200 import workloads

    w, r, local = dist.init("gloo", timeout_s=60)
    dist.barrier()
    # Replica: this rank's own seeded list, removed by the CPU restatement.
    n, k = 1 << 14, 1 << 10
    data = np.arange(n, dtype=np.uint32)
    idx = workloads.uniform(n, k, seed=dist.replica_seed(3, r))
    new_len = oracle.remove(data, idx)
    kept_sum = int(data[:new_len].astype(np.int64).sum())
    t = 1.0 + r  # stands in for a measured step time
    res = {"env": [w, r, local], "max": dist.max_over_ranks(t), "sum_k": dist.sum_over_ranks(float(k)),
           "new_len": new_len, "kept_sum": kept_sum, "seed": dist.replica_seed(3, r),
           "shard": dist.shard_by_weight([5, 1, 1, 1, 8, 2, 2], w, r).tolist()}
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)
    dist.barrier()
    tdist.destroy_process_group()


def test_two_gloo_ranks_run_replicas_and_reduce(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, x in enumerate(res):
        assert x["env"] == [2, r, r]
        assert x["max"] == 2.0  # the slowest rank's time
        assert x["sum_k"] == 2.0 * (1 << 10)  # whole-job work
        assert x["new_len"] == (1 << 14) - (1 << 10)
    assert res[0]["seed"] != res[1]["seed"] and res[0]["kept_sum"] != res[1]["kept_sum"]  # distinct replicas
    shards = [x["shard"] for x in res]
    assert sorted(shards[0] + shards[1]) == list(range(7)) and not set(shards[0]) & set(shards[1])


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_by_weight_is_a_balanced_contiguous_partition(world):
    rng = np.random.default_rng(world)
    for trial in range(20):
        w = rng.integers(0, 1000, size=int(rng.integers(0, 300)))
        parts = [dist.shard_by_weight(w, world, r) for r in range(world)]
        allidx = np.concatenate(parts) if parts else np.zeros(0)
        assert sorted(allidx.tolist()) == list(range(len(w)))  # every item exactly once
        for p in parts:
            if len(p):
                assert np.all(np.diff(p) == 1)  # contiguous
        if len(w) and w.sum() > 0:
            heaviest = max(w[p].sum() for p in parts)
            assert heaviest <= w.sum() / world + w.max() + 1e-9
