"""The predictor's CPU oracle, pinned: its analytic gradient against central finite differences."""
import numpy as np

from oracle import mlp_ref


def random_batch(seed, nb=16):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, mlp_ref.N_PARAMS)
    x = rng.uniform(0, 1, (nb, mlp_ref.N_IN))
    t = rng.uniform(0, 1, (nb, mlp_ref.N_OUT))
    t[:, : mlp_ref.N_CFG] /= t[:, : mlp_ref.N_CFG].sum(1, keepdims=True)
    t[:, mlp_ref.N_CFG] = rng.integers(0, 2, nb)
    return p, x, t


def test_analytic_gradient_matches_finite_differences():
    p, x, t = random_batch(0)
    _, g = mlp_ref.loss_and_grad(p, x, t)
    rng = np.random.default_rng(1)
    # Every bias and a sample of weights from each layer.
    probe = np.concatenate([np.arange(mlp_ref.OFF_B1, mlp_ref.OFF_W2), np.arange(mlp_ref.OFF_B2, mlp_ref.OFF_W3),
                            np.arange(mlp_ref.OFF_B3, mlp_ref.N_PARAMS),
                            rng.integers(mlp_ref.OFF_W1, mlp_ref.OFF_B1, 40),
                            rng.integers(mlp_ref.OFF_W2, mlp_ref.OFF_B2, 40),
                            rng.integers(mlp_ref.OFF_W3, mlp_ref.OFF_B3, 40)])
    h = 1e-6
    for q in probe:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (mlp_ref.loss_and_grad(pp, x, t)[0] - mlp_ref.loss_and_grad(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 + 1e-4 * abs(fd), (q, fd, g[q])


def test_features_of_known_patterns():
    n, k = 1 << 20, 4096
    run = np.arange(1000, 1000 + k, dtype=np.uint32)  # one run of 4096
    f = mlp_ref.features(run, n, k, 4)
    assert f[11] == 1.0 and f[7] == 0.0
    tail = np.arange(n - k, n, dtype=np.uint32)
    assert mlp_ref.features(tail, n, k, 4)[6] == 1.0
    spaced = np.arange(0, n, n // k, dtype=np.uint32)[:k]
    fs = mlp_ref.features(spaced, n, k, 16)
    assert fs[7] == 1.0 and abs(fs[4] - 1.0 / 8) < 1e-9 and fs[5] < 1e-12 and fs[3] == 0.5


# ---- the shipped predictor on held-out instances (CPU: the oracle's forward pass) ----------------
from pathlib import Path  # noqa: E402

ROOT = Path(__file__).resolve().parent.parent
WEIGHTS = ROOT / "redzone_b200" / "data" / "predictor.npz"
HELDOUT = ROOT / "tests" / "golden" / "predictor_heldout.npz"


def _regret(cls, T):
    cfg = T[:, : mlp_ref.N_CFG].astype(np.float64)
    best = np.minimum(cfg.min(1), T[:, mlp_ref.N_CFG].astype(np.float64))
    return cfg[np.arange(T.shape[0]), cls] / best - 1.0


def test_shipped_predictor_beats_the_method_without_it():
    """Held-out seeds, timings of all 63 configurations + partition measured on a B200 (median of
    5 runs each): the network's choice is within 5 % of the exhaustive best on average, and better
    than the fixed default configuration and than the best single configuration for all inputs."""
    p = np.load(WEIGHTS)["params"].astype(np.float64)
    h = np.load(HELDOUT)
    X, T, dcls = h["X"].astype(np.float64), h["T"], h["default_cls"]
    _, _, out = mlp_ref.forward(p, X)
    cls = out[:, : mlp_ref.N_CFG].argmax(1)
    reg = _regret(cls, T)
    reg_default = _regret(dcls, T)
    fixed = min(range(mlp_ref.N_CFG), key=lambda c: _regret(np.full(len(T), c), T).mean())
    reg_fixed = _regret(np.full(len(T), fixed), T)
    assert reg.mean() <= 0.05, reg.mean()
    assert reg.mean() < reg_default.mean() and reg.mean() < reg_fixed.mean()
