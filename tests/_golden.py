"""Access to the committed golden vectors made from the reference's redzone_CPU."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

from redzone_b200 import workloads

GOLDEN = Path(__file__).resolve().parent / "golden" / "redzone_cpu_golden.npz"
DISTS = ["uniform", "clustered", "tail", "red0", "red25", "red50", "red75", "red100"]


def sha(a: np.ndarray) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def cases(max_n: int | None = None):
    """Yield dicts with n, k, seed, dist, idx and either prefix or prefix_sha."""
    d = np.load(GOLDEN)
    c = 0
    while f"c{c}_meta" in d.files:
        n, k, seed, dcode = (int(x) for x in d[f"c{c}_meta"])
        if max_n is None or n <= max_n:
            dist = DISTS[dcode]
            case = dict(n=n, k=k, seed=seed, dist=dist, id=c)
            if f"c{c}_idx" in d.files:
                case["idx"] = d[f"c{c}_idx"]
                case["prefix"] = d[f"c{c}_prefix"]
            else:
                idx = workloads.make(dist, n, k, seed)
                assert sha(idx.astype("<u4")) == d[f"c{c}_idx_sha256"].tobytes(), "index generator drifted"
                case["idx"] = idx
                case["prefix_sha"] = d[f"c{c}_sha256"].tobytes()
            yield case
        c += 1


def check_prefix(case, prefix: np.ndarray) -> bool:
    p = np.ascontiguousarray(prefix.astype("<i4"))
    if "prefix" in case:
        return np.array_equal(p, case["prefix"])
    return sha(p) == case["prefix_sha"]
