"""Seeded synthetic removal workloads (the reference's benchmark inputs, reproducibly).

The reference draws k distinct removal indices by a partial Fisher-Yates shuffle seeded from
``std::random_device`` (DataStruct.hxx:73-133), so its runs cannot be repeated. Here every
generator takes an explicit seed. Distributions:

* ``uniform``   k distinct indices uniform over [0, n), in draw order (unsorted).
* ``clustered`` k/256 runs of 256 consecutive indices at uniformly random non-overlapping
                starts, index order shuffled.
* ``tail``      k distinct indices uniform over the last 10% of the list, [n - n//10, n).
* ``red<p>``    the reference's red% split (DataStruct.hxx:97-122): round-down(k*p/100) indices
                in the red zone [n-k, n), the rest in [0, n-k).

All functions return uint32 numpy arrays; ``*_torch`` variants generate on a torch device.
"""
from __future__ import annotations

import math

import numpy as np

DISTRIBUTIONS = ("uniform", "clustered", "tail")


def _distinct(rng: np.random.Generator, lo: int, hi: int, k: int) -> np.ndarray:
    """k distinct values from [lo, hi) in random order."""
    span = hi - lo
    if k > span:
        raise ValueError(f"cannot draw {k} distinct values from a range of {span}")
    if k == 0:
        return np.zeros(0, dtype=np.uint32)
    if k * 4 <= span:
        out = rng.choice(span, size=k, replace=False)
    else:
        out = rng.permutation(span)[:k]
    return (out + lo).astype(np.uint32)


def uniform(n: int, k: int, seed: int) -> np.ndarray:
    return _distinct(np.random.default_rng(seed), 0, n, k)


def clustered(n: int, k: int, seed: int, run: int = 256) -> np.ndarray:
    rng = np.random.default_rng(seed)
    m, rem = divmod(k, run)
    lens = [run] * m + ([rem] if rem else [])
    total_len = sum(lens)
    free = n - total_len
    if free < 0:
        raise ValueError("runs do not fit")
    # Sorted gaps: start_j = y_j + (sum of earlier run lengths) with y sorted in [0, free].
    y = np.sort(rng.integers(0, free + 1, size=len(lens)))
    order = rng.permutation(len(lens))  # which run length goes where (only the short one moves)
    lens = np.asarray(lens, dtype=np.int64)[order]
    starts = y + np.concatenate([[0], np.cumsum(lens)[:-1]])
    idx = np.concatenate([np.arange(s, s + L, dtype=np.int64) for s, L in zip(starts, lens)]) if lens.size else np.zeros(0, np.int64)
    rng.shuffle(idx)
    return idx.astype(np.uint32)


def tail(n: int, k: int, seed: int, frac: float = 0.1) -> np.ndarray:
    lo = n - int(n * frac)
    return _distinct(np.random.default_rng(seed), lo, n, k)


def red_split(n: int, k: int, seed: int, red_percentage: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    red_k = (k * red_percentage) // 100
    green = _distinct(rng, 0, n - k, k - red_k)
    red = _distinct(rng, n - k, n, red_k)
    return np.concatenate([green, red]).astype(np.uint32)


def make(dist: str, n: int, k: int, seed: int) -> np.ndarray:
    if dist == "uniform":
        return uniform(n, k, seed)
    if dist == "clustered":
        return clustered(n, k, seed)
    if dist == "tail":
        return tail(n, k, seed)
    if dist.startswith("red"):
        return red_split(n, k, seed, int(dist[3:]))
    raise ValueError(f"unknown distribution {dist!r}")


def make_torch(dist: str, n: int, k: int, seed: int, device="cuda"):
    """Same distributions generated with torch (fast at n = 2^28); not bit-identical to numpy."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if dist == "uniform":
        if k * 8 <= n:
            # Oversample, deduplicate in draw order, trim (expected few collisions).
            need = k
            out = torch.empty(0, dtype=torch.int64, device=device)
            while out.numel() < need:
                cand = torch.randint(0, n, (int((need - out.numel()) * 1.1) + 64,), generator=g, device=device)
                allv = torch.cat([out, cand])
                uniq, inv = torch.unique(allv, return_inverse=True)
                first = torch.full((uniq.numel(),), allv.numel(), dtype=torch.int64, device=device)
                first.scatter_reduce_(0, inv, torch.arange(allv.numel(), device=device), reduce="amin")
                keep = torch.zeros(allv.numel(), dtype=torch.bool, device=device)
                keep[first] = True
                out = allv[keep]
            out = out[:need]
        else:
            out = torch.randperm(n, generator=g, device=device)[:k]
        return out.to(torch.int32)
    if dist == "tail":
        lo = n - n // 10
        return (torch.randperm(n - lo, generator=g, device=device)[:k] + lo).to(torch.int32)
    if dist == "clustered":
        run = 256
        m, rem = divmod(k, run)
        if rem:
            raise ValueError("clustered torch generator needs k % 256 == 0")
        free = n - k
        y = torch.sort(torch.randint(0, free + 1, (m,), generator=g, device=device)).values
        starts = y + torch.arange(m, device=device) * run
        idx = (starts[:, None] + torch.arange(run, device=device)[None, :]).reshape(-1)
        perm = torch.randperm(idx.numel(), generator=g, device=device)
        return idx[perm].to(torch.int32)
    raise ValueError(f"unknown distribution {dist!r}")


# ---- batched workload: thousands of uneven lists ----------------------------------------------
def batched_lists(nlists: int, seed: int, log2_lo: float = 8.0, log2_hi: float = 22.0,
                  f_lo: float = 0.001, f_hi: float = 0.5):
    """Per-list (n, k): n = round(2^U(lo, hi)), k = round(f*n), f ~ U(f_lo, f_hi)."""
    rng = np.random.default_rng(seed)
    n = np.rint(np.exp2(rng.uniform(log2_lo, log2_hi, size=nlists))).astype(np.int64)
    f = rng.uniform(f_lo, f_hi, size=nlists)
    k = np.minimum(np.rint(f * n).astype(np.int64), n)
    return n, k


def batched_indices(n: np.ndarray, k: np.ndarray, seed: int) -> np.ndarray:
    """Concatenated per-list uniform removal indices (list-local positions)."""
    rng = np.random.default_rng(seed)
    parts = [_distinct(rng, 0, int(ni), int(ki)) for ni, ki in zip(n, k)]
    return np.concatenate(parts) if parts else np.zeros(0, np.uint32)


def expected_batched_elements(log2_lo: float = 8.0, log2_hi: float = 22.0) -> float:
    """E[2^U(lo,hi)] per list, = (2^hi - 2^lo) / ((hi - lo) ln 2)."""
    return (2.0 ** log2_hi - 2.0 ** log2_lo) / ((log2_hi - log2_lo) * math.log(2.0))
