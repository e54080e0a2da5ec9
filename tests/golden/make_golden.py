"""Generate golden vectors from the reference's own CPU Redzone (redzone_CPU, Redzone_CPU.hxx:150).

The reference ships no golden vectors or known-answer tests. This script runs the reference's
``redzone_CPU``, compiled from its sources by ``oracle/Makefile`` (``oracle/_ref``), on seeded
iota int32 inputs and stores the resulting surviving prefix. The fixtures are committed, so the
tests need neither the reference sources nor the compiled reference.

Output: ``tests/golden/redzone_cpu_golden.npz`` holding, per case c, ``c{c}_meta`` =
[n, k, seed, dist code] and either ``c{c}_idx`` (uint32) with ``c{c}_prefix`` (int32) for
n <= 4096, or, for larger n, ``c{c}_idx_sha256`` (SHA-256 of the regenerated little-endian
uint32 indices) with ``c{c}_sha256`` (SHA-256 of the little-endian int32 prefix).

Run: ``python tests/golden/make_golden.py`` (needs oracle/_ref/librz_ref_cpu.so).
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from redzone_b200 import workloads  # noqa: E402

DISTS = ["uniform", "clustered", "tail", "red0", "red25", "red50", "red75", "red100"]
OUT = Path(__file__).resolve().parent / "redzone_cpu_golden.npz"


def feasible(n, k, dist):
    if dist.startswith("red"):
        red_k = (k * int(dist[3:])) // 100
        return k - red_k <= n - k
    if dist == "tail":
        return k <= n // 10
    if dist == "clustered":
        return k % 256 == 0
    return True


def cases():
    return [c for c in _all_cases() if feasible(c[0], c[1], c[3])]


def _all_cases():
    out = []
    seed = 100
    for n in [2, 3, 5, 8, 17, 64, 100, 257, 1000, 4096]:
        for k in sorted({1, 2, n // 3, n // 2, n - 1}):
            if k < 1 or k >= n:
                continue
            for dist in ["uniform", "red0", "red100", "red50"]:
                out.append((n, k, seed, dist))
                seed += 1
    for n, k in [(1 << 12, 1 << 8), (1 << 12, 1 << 11), (1 << 14, 3000), (1 << 16, 1 << 10)]:
        for dist in DISTS:
            if dist == "tail" and k > n // 10:
                continue
            if dist == "clustered" and k % 256:
                continue
            out.append((n, k, seed, dist))
            seed += 1
    # The single-list configuration of the reference's headline benchmark (n=2^20, k=2^14).
    for s in range(3):
        out.append((1 << 20, 1 << 14, s, "uniform"))
    out.append((1 << 20, 1 << 19, 11, "uniform"))
    out.append((1 << 20, 1 << 16, 12, "tail"))
    out.append((1 << 20, 1 << 16, 13, "clustered"))
    return out


def main():
    L = oracle.ref_lib()
    if L is None:
        raise SystemExit("build the reference CPU path first: make -C oracle ref")
    arrays = {}
    for c, (n, k, seed, dist) in enumerate(cases()):
        idx = workloads.make(dist, n, k, seed)
        a = np.arange(n, dtype=np.int32)
        oracle.ref_redzone_cpu(a, idx)
        prefix = a[: n - k]
        arrays[f"c{c}_meta"] = np.array([n, k, seed, DISTS.index(dist)], dtype=np.int64)
        if n <= 1 << 12:
            arrays[f"c{c}_idx"] = idx.astype(np.uint32)
            arrays[f"c{c}_prefix"] = prefix.copy()
        else:
            # Large cases: the indices are regenerated from (dist, n, k, seed); their hash guards
            # against generator drift.
            arrays[f"c{c}_idx_sha256"] = np.frombuffer(hashlib.sha256(idx.astype("<u4").tobytes()).digest(), np.uint8)
            arrays[f"c{c}_sha256"] = np.frombuffer(hashlib.sha256(prefix.astype("<i4").tobytes()).digest(), np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} with {len(cases())} cases, {OUT.stat().st_size} bytes")


if __name__ == "__main__":
    main()
