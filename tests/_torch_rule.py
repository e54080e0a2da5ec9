"""Vectorised torch statement of the canonical Redzone result, for checking full-size runs on the
GPU where the C oracle would be slow. It is checked against the C oracle in the GPU tests."""
from __future__ import annotations

import torch


def canonical_prefix(a: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
    """Surviving prefix [0, n-k) that Redzone must produce from items `a` and removals `idx`."""
    n, k = a.shape[0], idx.numel()
    cut = n - k
    if k == 0 or k == n:
        return a[:cut].clone()
    idx = idx.to(torch.int64)
    red = torch.zeros(k, dtype=torch.bool, device=a.device)
    m = idx >= cut
    red[idx[m] - cut] = True
    sv, dv = ~red, idx < cut
    out = a[:cut].clone()
    src = a[cut:]
    both = sv & dv
    out[idx[both]] = src[both]
    out[idx[dv & ~sv]] = src[sv & ~dv]
    return out


def survivor_properties(prefix: torch.Tensor, n: int, idx: torch.Tensor) -> dict:
    """isOK_CPU's checks (DataStruct.hxx:154-191) for iota int32 payloads, plus 'unmoved'."""
    cut = prefix.shape[0]
    removed = torch.zeros(n, dtype=torch.bool, device=prefix.device)
    removed[idx.to(torch.int64)] = True
    p = prefix.to(torch.int64)
    in_range = bool(((p >= 0) & (p < n)).all())
    distinct = bool(torch.unique(p).numel() == cut)
    none_removed = bool(not removed[p.clamp(0, n - 1)].any())
    keep_below = ~removed[:cut]
    unmoved = bool((p[keep_below] == torch.arange(cut, device=p.device)[keep_below]).all())
    return dict(in_range=in_range, distinct=distinct, none_removed=none_removed, unmoved=unmoved)
