"""Learned launch-configuration predictor: data from the kernels' own timings, GPU training,
regret against exhaustive autotuning.

Pipeline (``python -m redzone_b200.learn collect|train``; ``train`` also evaluates):

* ``collect``: seeded removal instances drawn as mixes of the two single-list benchmark
  configurations (n = 2^20 and n = 2^28, plus intermediate sizes; int32 and 16-byte payloads;
  uniform, clustered and tail-heavy indices). For each: the 12 features from the GPU feature
  kernel (``rz_mlp_features``) and the time of every one of the 63 launch configurations plus the
  partition path (``rz_autotune_single``, CUDA events, L2 flushed between runs).
* ``train``: soft targets (configurations within a few percent of the fastest get most of the
  mass) and the partition bit; Adam on the GPU through ``rz_mlp_train``.
* evaluation (end of ``train``): on held-out seeds, regret = time of the predicted
  configuration / time of the best one - 1 (the best one taken from the exhaustive autotune table);
  compared with the fixed default configuration (``rz_default_cfg``), i.e. the method without
  the network.

``Mlp`` wraps the C-ABI network; ``attach_default(ctx)`` loads the shipped weights
(``redzone_b200/data/predictor.npz``) into a context for ``rz_remove(..., RZ_USE_PREDICTOR)``.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

from . import _native
from ._native import LaunchCfg

N_IN, N_OUT, N_CFG = 12, 64, 63
SCHED_AUTO, SCHED_CSCAN, SCHED_SPLIT, SCHED_SCANALL = 0, 4, 5, 6
DATA = Path(__file__).resolve().parent / "data"
_FP = ctypes.POINTER(ctypes.c_float)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def config_space() -> list[tuple[int, int, int, int]]:
    """(block, items, grid scale, schedule) in the library's canonical order (class index =
    position): 48 points with the schedule chosen by k, then 8 cluster-scan, 4 scan-all and 3
    split launches."""
    grid = [(b, i, g, SCHED_AUTO) for b in (128, 256, 512, 1024) for i in (1, 2, 4, 8) for g in (1, 2, 4)]
    cscan = [(b, i, 2, SCHED_CSCAN) for b, i in ((128, 2), (128, 4), (256, 1), (256, 2), (256, 4), (256, 8),
                                                  (512, 2), (512, 4))]
    scanall = [(256, i, 2, SCHED_SCANALL) for i in (1, 2, 4, 8)]
    split = [(256, i, 2, SCHED_SPLIT) for i in (1, 2, 4)]
    return grid + cscan + scanall + split


class Mlp:
    """The library's FP32 MLP (rz_mlp_*), trained and run by its own CUDA kernels."""

    def __init__(self, ctx, seed: int = 0):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(_native.lib.rz_mlp_create(ctx.handle, seed, ctypes.byref(h)), "rz_mlp_create")
        self.handle = h
        self.nparams = _native.lib.rz_mlp_param_count()

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, np.float32)
        self.ctx._check(_native.lib.rz_mlp_get_params(self.handle, _fp(p), self.nparams), "rz_mlp_get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self.ctx._check(_native.lib.rz_mlp_set_params(self.handle, _fp(p), self.nparams), "rz_mlp_set_params")

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros((x.shape[0], N_OUT), np.float32)
        self.ctx._check(_native.lib.rz_mlp_forward(self.handle, _fp(x), x.shape[0], _fp(out)), "rz_mlp_forward")
        return out

    def gradients(self, x, t) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_float(0)
        self.ctx._check(_native.lib.rz_mlp_gradients(self.handle, _fp(x), _fp(t), x.shape[0], _fp(g),
                                                     ctypes.byref(loss)), "rz_mlp_gradients")
        return float(loss.value), g

    def train(self, x, t, epochs=40, batch=512, lr=2e-3, seed=0) -> float:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = ctypes.c_float(0)
        self.ctx._check(_native.lib.rz_mlp_train(self.handle, _fp(x), _fp(t), x.shape[0], epochs, batch, lr, seed,
                                                 ctypes.byref(loss)), "rz_mlp_train")
        return float(loss.value)

    def predict(self, x) -> tuple[np.ndarray, np.ndarray]:
        """(class index, partition bit) per row of x."""
        o = self.forward(x)
        return o[:, :N_CFG].argmax(1), (o[:, N_CFG] > 0).astype(np.int32)

    def attach(self) -> None:
        """Make rz_remove(..., RZ_USE_PREDICTOR) use this network."""
        self.ctx._check(_native.lib.rz_set_predictor(self.ctx.handle, self.handle), "rz_set_predictor")
        self._attached = "single"

    def attach_batched(self) -> None:
        """Make batched plans created without a configuration use this network."""
        self.ctx._check(_native.lib.rz_set_batch_predictor(self.ctx.handle, self.handle), "rz_set_batch_predictor")
        self._attached = "batched"

    def save(self, path) -> None:
        np.savez_compressed(path, params=self.params())

    def load(self, path) -> None:
        self.set_params(np.load(path)["params"])

    def close(self):
        if getattr(self, "handle", None):
            # Destroying the network detaches it from the context (rz_mlp_destroy).
            _native.lib.rz_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def attach_default(ctx) -> Mlp | None:
    """Load the shipped predictor weights into `ctx`, if the package carries them."""
    path = DATA / "predictor.npz"
    if not path.exists():
        return None
    m = Mlp(ctx)
    m.load(path)
    m.attach()
    return m


# ---- training data ------------------------------------------------------------------------------
def soft_targets(times: np.ndarray, tau: float = 0.03) -> np.ndarray:
    """times: (N, 64) ms for the 63 configurations and the partition path -> (N, 64) targets."""
    t = np.asarray(times, np.float64)
    cfg = t[:, :N_CFG]
    best = cfg.min(1, keepdims=True)
    z = -(cfg / best - 1.0) / tau
    z -= z.max(1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(1, keepdims=True)
    bit = (t[:, N_CFG] < best[:, 0]).astype(np.float64)
    return np.concatenate([p, bit[:, None]], axis=1).astype(np.float32)


def draw_instance(rng: np.random.Generator, klog: tuple[float, float] | None = None) -> tuple[int, int, int, str]:
    """(n, k, w, distribution): mixes of the n = 2^20 (k = 2^14) and n = 2^28 (k sweep, int32 and
    16-byte items) configurations, with intermediate list sizes for coverage. k reaches 2^24, where
    the O(n) partition overtakes the O(k) removal at n = 2^28. With `klog` = (lo, hi), only
    instances with log2 k in [lo, hi) are kept (the same distribution, restricted)."""
    while True:
        n, k, w, dist = _draw_instance(rng)
        if klog is None or klog[0] <= math.log2(max(k, 1)) < klog[1]:
            return n, k, w, dist


def _draw_instance(rng: np.random.Generator) -> tuple[int, int, int, str]:
    if rng.random() < 0.15:
        n, k = 1 << 20, 1 << 14
    else:
        n = 1 << int(rng.choice([16, 18, 20, 22, 24, 26, 28], p=[.08, .1, .14, .14, .16, .14, .24]))
        hi = min(math.log2(n) - 1, 24.0)
        k = int(round(2 ** rng.uniform(8.0, hi)))
    w = int(rng.choice([4, 16]))
    dist = str(rng.choice(["uniform", "clustered", "tail"], p=[.6, .2, .2]))
    if dist == "clustered":
        k = max(256, (k // 256) * 256)
    if dist == "tail" and k > n // 10:
        dist = "uniform"
    return n, min(k, n // 2), w, dist


def collect(ctx, count: int, seed: int, reps: int = 1, log_every: int = 500,
            klog: tuple[float, float] | None = None):
    """Features and 64 timings for `count` seeded instances (timing rewrites a scratch array)."""
    import torch
    from . import workloads

    dev = torch.device("cuda", ctx.device)
    buf = torch.zeros((1 << 28) * 4, dtype=torch.int32, device=dev)  # room for n = 2^28 x 16 bytes
    rng = np.random.default_rng(seed)
    X = np.zeros((count, N_IN), np.float32)
    T = np.zeros((count, N_OUT), np.float32)
    meta = np.zeros((count, 4), np.int64)
    entries = (_native.TuneEntry * N_OUT)()
    nent = ctypes.c_int32(0)
    space = {c: q for q, c in enumerate(config_space())}
    t0 = time.time()
    for q in range(count):
        n, k, w, dist = draw_instance(rng, klog)
        idx = workloads.make_torch(dist, n, k, seed=int(rng.integers(0, 1 << 62))).contiguous()
        data = buf[: n * (w // 4)].view(n, w // 4)
        f = np.zeros(N_IN, np.float32)
        ctx._check(_native.lib.rz_mlp_features(ctx.handle, ctypes.c_void_p(idx.data_ptr()), n, k, w, _fp(f)),
                   "rz_mlp_features")
        ctx._check(_native.lib.rz_autotune_single(ctx.handle, ctypes.c_void_p(data.data_ptr()), n, w,
                                                  ctypes.c_void_p(idx.data_ptr()), k, reps, entries, N_OUT,
                                                  ctypes.byref(nent)), "rz_autotune_single")
        for e in entries[: nent.value]:
            if e.cfg.use_partition:
                T[q, N_CFG] = e.ms
            else:
                T[q, space[(e.cfg.block, e.cfg.items, e.cfg.ctas_per_sm, e.cfg.schedule)]] = e.ms
        X[q] = f
        meta[q] = (n, k, w, ["uniform", "clustered", "tail"].index(dist))
        if log_every and (q + 1) % log_every == 0:
            print(f"collected {q + 1}/{count} in {time.time() - t0:.0f}s", file=sys.stderr, flush=True)
    del buf
    return X, T, meta


def default_class(ctx, n, k, w) -> int:
    c = LaunchCfg()
    ctx._check(_native.lib.rz_default_cfg(ctx.handle, int(n), int(k), int(w), ctypes.byref(c)), "rz_default_cfg")
    space = config_space()
    key = (c.block, c.items, c.ctas_per_sm, c.schedule)
    if key in space:
        return space.index(key)
    # The default's block may be clamped; pick the nearest class of the same schedule family with
    # the same items and grid.
    fam = c.schedule if c.schedule in (SCHED_CSCAN, SCHED_SPLIT, SCHED_SCANALL) else SCHED_AUTO
    return min(range(N_CFG), key=lambda q: (space[q][3] != fam, space[q][1] != c.items,
                                            space[q][2] != c.ctas_per_sm, abs(space[q][0] - c.block)))


def evaluate(pred_cls, pred_bit, T, default_cls) -> dict:
    """Regret of the predictions against the exhaustive best, and of the fixed default."""
    cfg = T[:, :N_CFG].astype(np.float64)
    part = T[:, N_CFG].astype(np.float64)
    best = np.minimum(cfg.min(1), part)
    rows = np.arange(T.shape[0])
    t_pred = np.where(pred_bit == 1, part, cfg[rows, pred_cls])
    t_pred_cfg = cfg[rows, pred_cls]
    t_def = cfg[rows, default_cls]
    best_cfg = cfg.min(1)
    return {
        "instances": int(T.shape[0]),
        "regret_mean": float(np.mean(t_pred / best - 1)),
        "regret_median": float(np.median(t_pred / best - 1)),
        "within_5pct": float(np.mean(t_pred <= 1.05 * best)),
        "config_regret_mean": float(np.mean(t_pred_cfg / best_cfg - 1)),
        "default_regret_mean": float(np.mean(t_def / best - 1)),
        "default_config_regret_mean": float(np.mean(t_def / best_cfg - 1)),
        "speedup_vs_default_total_time": float(t_def.sum() / t_pred.sum()),
        "bit_accuracy": float(np.mean(pred_bit == (part < best_cfg))),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m redzone_b200.learn")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=1000)
    c.add_argument("--seed", type=int, default=0)
    c.add_argument("--out", required=True)
    c.add_argument("--reps", type=int, default=1, help="timed runs per configuration (median)")
    c.add_argument("--klog", type=float, nargs=2, default=None,
                   help="keep only instances with log2 k in [lo, hi) (re-timing a range after a kernel change)")
    t = sub.add_parser("train")
    t.add_argument("--data", nargs="+", required=True)
    t.add_argument("--stale", nargs="*", default=[],
                   help="data files timed before a kernel change; their rows with log2 k in --stale-klog are dropped")
    t.add_argument("--stale-klog", type=float, nargs=2, default=None)
    t.add_argument("--heldout", nargs="+", required=True)
    t.add_argument("--epochs", type=int, default=60)
    t.add_argument("--tau", type=float, default=0.05, help="soft-target temperature (relative time)")
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--out", required=True)
    t.add_argument("--report", default=None)
    t.add_argument("--fixture", default=None,
                   help="also write the first --fixture-count held-out rows (features, timings, default class)")
    t.add_argument("--fixture-count", type=int, default=1000)
    e = sub.add_parser("evaluate", help="regret of saved weights on held-out data")
    e.add_argument("--weights", required=True)
    e.add_argument("--heldout", nargs="+", required=True)
    args = ap.parse_args(argv)
    import redzone_b200 as rz

    ctx = rz.Context(0)
    if args.cmd == "evaluate":
        hold = [np.load(p) for p in args.heldout]
        Xh = np.concatenate([p["X"] for p in hold])
        Th = np.concatenate([p["T"] for p in hold])
        Mh = np.concatenate([p["meta"] for p in hold])
        m = Mlp(ctx)
        m.load(args.weights)
        cls, bit = m.predict(Xh)
        dcls = np.array([default_class(ctx, *row[:3]) for row in Mh])
        rep = evaluate(cls, bit, Th, dcls)
        rep.update({"weights": args.weights, "heldout_seeds": [int(p["seed"]) for p in hold]})
        print(json.dumps(rep))
        return
    if args.cmd == "collect":
        X, T, meta = collect(ctx, args.count, args.seed, reps=args.reps, klog=args.klog)
        np.savez_compressed(args.out, X=X, T=T, meta=meta, seed=args.seed, reps=args.reps)
        print(json.dumps({"collected": int(X.shape[0]), "reps": args.reps, "out": args.out}))
        return
    parts = [np.load(p) for p in args.data]
    keep = []
    for path, p in zip(args.data, parts):
        rows = np.ones(p["X"].shape[0], bool)
        if path in args.stale and args.stale_klog:
            lk = np.log2(np.maximum(p["meta"][:, 1], 1))
            rows = ~((lk >= args.stale_klog[0]) & (lk < args.stale_klog[1]))
        keep.append(rows)
    X = np.concatenate([p["X"][r] for p, r in zip(parts, keep)])
    T = np.concatenate([p["T"][r] for p, r in zip(parts, keep)])
    hold = [np.load(p) for p in args.heldout]
    Xh = np.concatenate([p["X"] for p in hold])
    Th = np.concatenate([p["T"] for p in hold])
    Mh = np.concatenate([p["meta"] for p in hold])
    m = Mlp(ctx, seed=1)
    t0 = time.time()
    loss = m.train(X, soft_targets(T, args.tau), epochs=args.epochs, lr=args.lr)
    train_s = time.time() - t0
    cls, bit = m.predict(Xh)
    dcls = np.array([default_class(ctx, *row[:3]) for row in Mh])
    rep = evaluate(cls, bit, Th, dcls)
    rep.update({"train_instances": int(X.shape[0]), "heldout_instances": int(Xh.shape[0]), "final_loss": loss,
                "dropped_stale_instances": int(sum((~r).sum() for r in keep)),
                "train_seconds": train_s, "epochs": args.epochs, "tau": args.tau, "lr": args.lr,
                "train_seeds": [int(p["seed"]) for p in parts], "heldout_seeds": [int(p["seed"]) for p in hold]})
    m.save(args.out)
    if args.fixture:
        q = slice(0, min(args.fixture_count, Xh.shape[0]))
        np.savez_compressed(args.fixture, X=Xh[q], T=Th[q], meta=Mh[q], default_cls=dcls[q].astype(np.int32),
                            heldout_seeds=np.array(rep["heldout_seeds"]))
    print(json.dumps(rep))
    if args.report:
        Path(args.report).write_text(json.dumps(rep, indent=1))


if __name__ == "__main__":
    main()
