"""The CPU oracle, pinned: golden vectors from the reference's redzone_CPU, the live compiled
reference (when built here), a vectorised restatement, and exhaustive tiny cases."""
import itertools

import numpy as np
import pytest

import oracle
from redzone_b200 import workloads
from tests import _golden


def test_oracle_matches_reference_golden_vectors():
    n_cases = 0
    for case in _golden.cases():
        a = np.arange(case["n"], dtype=np.int32)
        oracle.remove(a, case["idx"])
        assert _golden.check_prefix(case, a[: case["n"] - case["k"]]), case["id"]
        n_cases += 1
    assert n_cases > 150


@pytest.mark.skipif(oracle.ref_lib() is None, reason="reference CPU path not built on this machine")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    for _ in range(8):
        n = int(rng.integers(2, 5000))
        k = int(rng.integers(1, n))
        dist = ["uniform", "red0", "red50", "red100"][int(rng.integers(0, 4))]
        if dist.startswith("red") and k - (k * int(dist[3:])) // 100 > n - k:
            dist = "uniform"
        idx = workloads.make(dist, n, k, int(rng.integers(0, 1 << 30)))
        a = np.arange(n, dtype=np.int32)
        b = a.copy()
        oracle.remove(a, idx)
        oracle.ref_redzone_cpu(b, idx)
        assert np.array_equal(a[: n - k], b[: n - k]), (n, k, dist)


@pytest.mark.parametrize("w_words", [1, 2, 4, 8])
def test_oracle_matches_numpy_restatement(w_words):
    rng = np.random.default_rng(w_words)
    for _ in range(40):
        n = int(rng.integers(1, 3000))
        k = int(rng.integers(0, n + 1))
        idx = workloads.uniform(n, k, int(rng.integers(0, 1 << 30)))
        a = rng.integers(0, 1 << 31, size=(n, w_words), dtype=np.int64).astype(np.uint32)
        expect = oracle.remove_numpy(a, idx)
        oracle.remove(a, idx)
        assert np.array_equal(a[: n - k], expect)


def test_exhaustive_tiny_lists():
    """Every ordered removal list for n <= 5, against the numpy rule and the reference."""
    ref = oracle.ref_lib()
    count = 0
    for n in range(1, 6):
        for k in range(0, n + 1):
            for idx in itertools.permutations(range(n), k):
                idx = np.array(idx, dtype=np.uint32)
                a = np.arange(n, dtype=np.int32)
                expect = oracle.remove_numpy(a, idx)
                oracle.remove(a, idx)
                assert np.array_equal(a[: n - k], expect)
                if ref is not None and 0 < k < n:
                    b = np.arange(n, dtype=np.int32)
                    oracle.ref_redzone_cpu(b, idx)
                    assert np.array_equal(b[: n - k], expect), (n, idx)
                count += 1
    assert count == sum(
        len(list(itertools.permutations(range(n), k))) for n in range(1, 6) for k in range(n + 1))


def test_survivor_properties():
    """isOK_CPU's checks (DataStruct.hxx:154-191) plus the unmoved-prefix property."""
    n, k = 1 << 16, 5000
    idx = workloads.uniform(n, k, 3)
    a = np.arange(n, dtype=np.int32)
    oracle.remove(a, idx)
    prefix = a[: n - k]
    removed = np.zeros(n, bool)
    removed[idx] = True
    assert (prefix >= 0).all() and (prefix < n).all()
    assert np.unique(prefix).size == prefix.size
    assert not removed[prefix].any()
    untouched = ~removed[: n - k]
    assert np.array_equal(prefix[untouched], np.arange(n - k)[untouched])


def test_stable_remove_and_validate():
    n, k = 4000, 1234
    idx = workloads.uniform(n, k, 9)
    a = np.arange(n, dtype=np.uint32)
    oracle.stable_remove(a, idx)
    keep = np.setdiff1d(np.arange(n), idx)
    assert np.array_equal(a[: n - k], keep)
    assert oracle.validate(n, idx) == 0
    assert oracle.validate(n, np.append(idx, idx[0])) == 2
    assert oracle.validate(n, np.append(idx, n)) == 3


def test_batched_oracle_equals_per_list():
    n, k = workloads.batched_lists(20, seed=1, log2_lo=4, log2_hi=10)
    idx = workloads.batched_indices(n, k, seed=2)
    data_off = np.concatenate([[0], np.cumsum(n)[:-1]])
    idx_off = np.concatenate([[0], np.cumsum(k)[:-1]])
    total = int(n.sum())
    data = np.arange(total, dtype=np.uint64)
    data2 = data.copy()
    oracle.remove_batched(data, 8, idx, data_off, n, idx_off, k)
    for l in range(len(n)):
        seg = data2[data_off[l]: data_off[l] + n[l]]
        oracle.remove(seg, idx[idx_off[l]: idx_off[l] + k[l]])
    assert np.array_equal(data, data2)


def _remove_via_red_entries(a, idx):
    """The formulation the cluster-scan, scan-all, split and produced-list kernels implement,
    restated in numpy: only the red entries (i, idx[i] >= cut) matter. V = {idx[i] - cut}, P = {i};
    a hole idx[i] < cut takes tail item i unless i is in V, in which case it is a destination
    orphan (V \\ P, ranked by position) and takes the tail item of the source orphan (P \\ V,
    ranked by position) of the same rank."""
    n, k = a.shape[0], idx.size
    cut = n - k
    out = a.copy()
    if k == 0 or k == n:
        return out
    idx = idx.astype(np.int64)
    red = idx >= cut
    V = np.zeros(k, bool)
    V[idx[red] - cut] = True
    P = red
    src_orphans = np.flatnonzero(P & ~V)          # positions, ascending
    dst_rank = np.cumsum(V & ~P) - 1               # rank of each destination orphan
    tail = a[cut:].copy()
    for i in range(k):
        if P[i]:
            continue
        if not V[i]:
            out[idx[i]] = tail[i]
        else:
            out[idx[i]] = tail[src_orphans[dst_rank[i]]]
    return out


@pytest.mark.parametrize("dist", ["uniform", "clustered", "tail", "red0", "red50", "red100"])
def test_red_entry_formulation_equals_the_canonical_rule(dist):
    rng = np.random.default_rng(["uniform", "clustered", "tail", "red0", "red50", "red100"].index(dist))
    cases = 0
    for _ in range(200):
        n = int(rng.integers(20, 4000))
        k = int(rng.integers(1, max(2, n // 10))) if dist == "tail" else int(rng.integers(1, n))
        if dist.startswith("red") and k - (k * int(dist[3:])) // 100 > n - k:
            continue
        if dist == "clustered" and k < 256:
            continue
        idx = workloads.make(dist, n, k, int(rng.integers(0, 1 << 30)))
        a = rng.integers(0, 1 << 31, size=(n, 2), dtype=np.int64).astype(np.uint32)
        expect = a.copy()
        oracle.remove(expect, idx)
        got = _remove_via_red_entries(a, idx)
        assert np.array_equal(got[: n - k], expect[: n - k]), (dist, n, k)
        cases += 1
    assert cases > 20
