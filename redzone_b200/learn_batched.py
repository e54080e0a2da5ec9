"""Learned configuration of the batched kernel: data from its own timings, GPU training, regret
against exhaustive autotuning.

The batched kernel (``rz_batch_plan_*``) runs a mix of lists in one launch; its configuration
(block x items x CTAs per SM x work order, ``rz_batch_config_space``) decides tile size, which
lists run whole in one CTA, grid size and how a list's phases are spaced in the work queue. The
best choice depends on the mix. The same FP32 MLP as the single-list predictor (``rz_mlp_*``, own
forward / backward / Adam kernels) is trained here to pick it from 12 features of the mix
(``rz_batch_features``, computed from the list sizes alone).

Pipeline (``python -m redzone_b200.learn_batched collect|train``; ``train`` also evaluates):

* ``collect``: seeded list mixes (list count, size range, removal-fraction range and payload
  width drawn per mix; one family is the 4096-list benchmark workload scaled down). For each mix:
  its features and the median time of every configuration (one graph-replayed launch per run,
  256 MiB L2 scrub before each run).
* ``train``: soft targets over the configurations (those within a few percent of the fastest get
  most of the mass); Adam on the GPU through ``rz_mlp_train``.
* evaluation (end of ``train``): on held-out seeds, regret = time of the predicted configuration
  / time of the exhaustively best one - 1, against the built-in default configuration (the method
  without the network) and the best single fixed configuration.

``attach_default(ctx)`` loads the shipped weights (``redzone_b200/data/batch_predictor.npz``) so
that ``rz_batch_plan_create(..., cfg=NULL)`` uses the network's choice.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import statistics
import sys
import time
from pathlib import Path

import numpy as np

from . import _native
from .learn import N_IN, N_OUT, Mlp, _fp

DATA = Path(__file__).resolve().parent / "data"
SCRUB_BYTES = 256 << 20
MAX_ITEMS = 1 << 28  # a mix holds at most this many items (4x that for the benchmark's own family)
DEFAULT_WAVE = 4     # the built-in default's work order (kDefaultWave)


def config_space() -> list[tuple[int, int, int, int]]:
    """(block, items, CTAs per SM, wave) in the library's order; class index = position."""
    n = _native.lib.rz_batch_config_space(None, 0)
    out = (_native.BatchCfg * n)()
    _native.lib.rz_batch_config_space(out, n)
    return [(c.block, c.items, c.ctas_per_sm, c.wave) for c in out]


def n_cfg() -> int:
    return int(_native.lib.rz_batch_config_space(None, 0))


def features(lists_or_sizes, w: int) -> np.ndarray:
    """The 12 mix features from (data, idx) tensor pairs or from (n, k) pairs."""
    pairs = [(int(d.shape[0]), int(i.numel())) if hasattr(d, "shape") else (int(d), int(i))
             for d, i in lists_or_sizes]
    arr = (_native.ListDesc * len(pairs))()
    for q, (n, k) in enumerate(pairs):
        arr[q].n, arr[q].k = n, k
    f = np.zeros(N_IN, np.float32)
    st = _native.lib.rz_batch_features(arr, len(pairs), w, _fp(f))
    if st != 0:
        raise RuntimeError(f"rz_batch_features: status {st}")
    return f


MAX_TILES_PER_LIST = 1024  # a list of the batched kernel spans at most this many tiles


def default_cfg(w: int, kmax: int = 0) -> tuple[int, int, int, int]:
    """The configuration rz_batch_plan_create uses without a predictor or table: 512 x 4 x 4 CTAs
    per SM in wavefront order (256 x 4 x 4 for 32-byte items), with items and then block raised
    until the longest list (kmax removals) fits the tile limit."""
    block, items, wave = (256 if w >= 32 else 512), 4, DEFAULT_WAVE
    while block * items * MAX_TILES_PER_LIST < kmax:
        if items < 8:
            items *= 2
        elif block < 512:
            block *= 2
        else:
            break
    return (block, items, 4, wave)


def default_class(ctx, w: int, kmax: int = 0) -> int:
    """Class of the default configuration (``default_cfg``) in the configuration space."""
    return config_space().index(default_cfg(w, kmax))


def kmax_of(features_row) -> int:
    """The largest k of a mix, recovered from its feature 11 (log2(1 + max k) / 24)."""
    return int(round(2.0 ** (24.0 * float(features_row[11])) - 1.0))


def draw_mix(rng: np.random.Generator) -> dict:
    """One seeded list mix: sizes n = round(2^U(lo, hi)), k = round(f n) with f ~ U(f_lo, f_hi)."""
    cap_items = MAX_ITEMS
    if rng.random() < 0.25:  # the benchmark workload's family, up to about half its size
        nl, lo, hi, f_lo, f_hi = int(rng.choice([256, 512, 1024, 2048])), 8.0, 22.0, 0.001, 0.5
        cap_items = 4 * MAX_ITEMS
    else:
        nl = int(round(2 ** rng.uniform(5, 12)))
        lo = rng.uniform(6, 16)
        hi = rng.uniform(lo + 1, 22)
        f_lo = 10 ** rng.uniform(-3, -1.3)
        f_hi = rng.uniform(min(0.5, 2 * f_lo), 0.5)
    w = int(rng.choice([4, 8, 16, 32], p=[.25, .4, .25, .1]))
    n = np.rint(np.exp2(rng.uniform(lo, hi, size=nl))).astype(np.int64)
    f = rng.uniform(f_lo, f_hi, size=nl)
    k = np.minimum(np.rint(f * n).astype(np.int64), n)
    cap = cap_items * 8 // max(w, 8)
    keep = np.cumsum(n) <= cap
    keep[0] = True
    return {"n": n[keep], "k": k[keep], "w": w, "seed": int(rng.integers(0, 1 << 62)),
            "family": [nl, lo, hi, f_lo, f_hi]}


def build_lists(mix: dict, dev):
    """The mix's lists on the device: payload items (w bytes, first word = index) and seeded
    distinct removal indices per list."""
    import torch

    n, k, w = mix["n"], mix["k"], mix["w"]
    words = w // 4
    buf = torch.zeros((int(n.sum()), words), dtype=torch.int32, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(mix["seed"] & ((1 << 62) - 1))
    lists, off = [], 0
    for ni, ki in zip(n.tolist(), k.tolist()):
        seg = buf[off: off + ni]
        seg[:, 0] = torch.arange(ni, dtype=torch.int32, device=dev)
        idx = torch.randperm(ni, generator=g, device=dev)[:ki].to(torch.int32)
        lists.append((seg, idx))
        off += ni
    return buf, lists


def time_configs(ctx, lists, reps: int, scrub) -> np.ndarray:
    """Median ms of one graph-replayed launch for every configuration (inf where a configuration
    cannot plan the mix)."""
    import torch
    import redzone_b200 as rz

    space = config_space()
    stream = torch.cuda.current_stream()
    out = np.full(len(space), np.inf, np.float32)
    for q, (b, i, c, wave) in enumerate(space):
        try:
            plan = rz.BatchPlan(ctx, lists, _native.BatchCfg(b, i, c, 0, wave))
        except rz.RedzoneError:
            continue
        plan.launch()
        ts = []
        for r in range(reps):
            scrub.fill_(r & 255)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.launch()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        plan.close()
        out[q] = statistics.median(ts)
    st = ctx.sync_status()
    if st != 0:
        raise RuntimeError(f"batched timing run reported device status {st}")
    return out


def collect(ctx, count: int, seed: int, reps: int = 3, log_every: int = 25):
    """Features, per-configuration times and a description of `count` seeded mixes."""
    import torch

    dev = torch.device("cuda", ctx.device)
    scrub = torch.empty(SCRUB_BYTES, dtype=torch.uint8, device=dev)
    rng = np.random.default_rng(seed)
    X = np.zeros((count, N_IN), np.float32)
    T = np.zeros((count, n_cfg()), np.float32)
    meta = np.zeros((count, 4), np.float64)  # lists, total n, total k, w
    t0 = time.time()
    for q in range(count):
        mix = draw_mix(rng)
        buf, lists = build_lists(mix, dev)
        X[q] = features(lists, mix["w"])
        T[q] = time_configs(ctx, lists, reps, scrub)
        meta[q] = (len(lists), float(mix["n"].sum()), float(mix["k"].sum()), mix["w"])
        del buf, lists
        if log_every and (q + 1) % log_every == 0:
            print(f"collected {q + 1}/{count} mixes in {time.time() - t0:.0f}s", file=sys.stderr, flush=True)
    return X, T, meta


def soft_targets(times: np.ndarray, tau: float = 0.03) -> np.ndarray:
    """(N, configurations) ms -> (N, 64) network targets: a distribution over the configurations in
    the first columns, zero elsewhere (the last column is the unused partition bit)."""
    t = np.asarray(times, np.float64)
    best = np.nanmin(np.where(np.isfinite(t), t, np.nan), axis=1, keepdims=True)
    z = np.where(np.isfinite(t), -(t / best - 1.0) / tau, -np.inf)
    z -= z.max(1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(1, keepdims=True)
    out = np.zeros((t.shape[0], N_OUT), np.float32)
    out[:, : t.shape[1]] = p
    return out


def feasible_mask(X: np.ndarray) -> np.ndarray:
    """(mixes, configurations): the configurations whose tile lets the longest list of the mix
    (from its feature 11) fit in the batched kernel's tile limit -- the library's prediction only
    considers those."""
    space = np.array(config_space())
    tile_cap = space[:, 0].astype(np.int64) * space[:, 1] * MAX_TILES_PER_LIST
    kmax = np.array([kmax_of(x) for x in X], np.int64)
    return tile_cap[None, :] >= kmax[:, None]


def choose(logits: np.ndarray, X: np.ndarray) -> np.ndarray:
    """The library's choice from network outputs: the best feasible configuration."""
    o = np.where(feasible_mask(X), logits[:, : n_cfg()], -np.inf)
    return o.argmax(1)


def predict(m: Mlp, X: np.ndarray) -> np.ndarray:
    return choose(m.forward(X), X)


def evaluate(pred: np.ndarray, T: np.ndarray, default_cls: np.ndarray) -> dict:
    """Regret of the predictions against the exhaustive best, of the default and of the best
    single fixed configuration."""
    t = np.where(np.isfinite(T), T, np.nan).astype(np.float64)
    best = np.nanmin(t, axis=1)
    rows = np.arange(t.shape[0])
    t_pred = t[rows, pred]
    t_def = t[rows, default_cls]
    fixed = np.nanmean(t / best[:, None], axis=0)
    fixed_q = int(np.nanargmin(fixed))
    t_fixed = t[rows, fixed_q]
    both = np.isfinite(t_def) & np.isfinite(t_pred)
    return {
        "mixes": int(t.shape[0]),
        "regret_mean": float(np.nanmean(t_pred / best - 1)),
        "regret_median": float(np.nanmedian(t_pred / best - 1)),
        "within_5pct": float(np.nanmean(t_pred <= 1.05 * best)),
        "default_regret_mean": float(np.nanmean(t_def / best - 1)),
        "best_fixed_cfg": list(config_space()[fixed_q]),
        "best_fixed_regret_mean": float(np.nanmean(t_fixed / best - 1)),
        "default_infeasible": int(np.sum(~np.isfinite(T[rows, default_cls]))),
        # total time over the mixes both can run
        "speedup_vs_default_total_time": float(t_def[both].sum() / t_pred[both].sum()),
        "infeasible_predictions": int(np.sum(~np.isfinite(T[rows, pred]))),
    }


def attach_default(ctx) -> Mlp | None:
    """Load the shipped list-mix predictor into `ctx` (rz_set_batch_predictor), if present."""
    path = DATA / "batch_predictor.npz"
    if not path.exists():
        return None
    m = Mlp(ctx)
    m.load(path)
    m.attach_batched()
    return m


def detach(ctx) -> None:
    _native.lib.rz_set_batch_predictor(ctx.handle, None)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m redzone_b200.learn_batched")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=200)
    c.add_argument("--seed", type=int, default=0)
    c.add_argument("--reps", type=int, default=3, help="timed launches per configuration (median)")
    c.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", nargs="+", required=True)
    t.add_argument("--heldout", nargs="+", required=True)
    t.add_argument("--epochs", type=int, default=300)
    t.add_argument("--tau", type=float, default=0.03)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--out", required=True)
    t.add_argument("--report", default=None)
    t.add_argument("--fixture", default=None, help="also write the held-out features, times and default classes")
    args = ap.parse_args(argv)
    import redzone_b200 as rz

    ctx = rz.Context(0)
    if args.cmd == "collect":
        X, T, meta = collect(ctx, args.count, args.seed, reps=args.reps)
        np.savez_compressed(args.out, X=X, T=T, meta=meta, seed=args.seed, reps=args.reps,
                            space=np.array(config_space(), np.int32))
        print(json.dumps({"collected": int(X.shape[0]), "reps": args.reps, "out": args.out}))
        return
    parts = [np.load(p) for p in args.data]
    X = np.concatenate([p["X"] for p in parts])
    T = np.concatenate([p["T"] for p in parts])
    hold = [np.load(p) for p in args.heldout]
    Xh = np.concatenate([p["X"] for p in hold])
    Th = np.concatenate([p["T"] for p in hold])
    Mh = np.concatenate([p["meta"] for p in hold])
    m = Mlp(ctx, seed=3)
    t0 = time.time()
    loss = m.train(X, soft_targets(T, args.tau), epochs=args.epochs, batch=min(256, X.shape[0]), lr=args.lr)
    train_s = time.time() - t0
    pred = predict(m, Xh)
    dcls = np.array([default_class(ctx, int(row[3]), kmax_of(x)) for row, x in zip(Mh, Xh)])
    rep = evaluate(pred, Th, dcls)
    rep.update({"train_mixes": int(X.shape[0]), "final_loss": loss, "train_seconds": train_s,
                "epochs": args.epochs, "tau": args.tau, "lr": args.lr,
                "train_seeds": [int(p["seed"]) for p in parts], "heldout_seeds": [int(p["seed"]) for p in hold]})
    m.save(args.out)
    if args.fixture:
        np.savez_compressed(args.fixture, X=Xh, T=Th, meta=Mh, default_cls=dcls.astype(np.int32),
                            heldout_seeds=np.array(rep["heldout_seeds"]), space=np.array(config_space(), np.int32))
    print(json.dumps(rep))
    if args.report:
        Path(args.report).write_text(json.dumps(rep, indent=1))


if __name__ == "__main__":
    main()
