"""The list-mix predictor's host side, no GPU: its features equal a numpy statement of their
definition, and its configuration space is the one the training code and the autotuner use."""
import numpy as np

from redzone_b200 import _native, learn_batched


def _features_numpy(n, k, w):
    n = np.asarray(n, np.float64)
    k = np.asarray(k, np.float64)
    lg = np.log2(1 + n)
    tk = k.sum()
    return np.array([
        np.log2(len(n)) / 16, np.log2(1 + n.sum()) / 36, np.log2(1 + tk) / 36, tk / n.sum(), w / 32,
        lg.mean() / 32, lg.std() / 8, (k / n).mean(),
        k[k <= 256].sum() / tk, k[k <= 1024].sum() / tk, k[k <= 4096].sum() / tk, np.log2(1 + k.max()) / 24,
    ], np.float32)


def test_mix_features_match_their_definition():
    from redzone_b200 import workloads
    for seed, nl, w in [(0, 4096, 8), (1, 37, 4), (2, 512, 16)]:
        n, k = workloads.batched_lists(nl, seed=seed)
        got = learn_batched.features(list(zip(n.tolist(), k.tolist())), w)
        np.testing.assert_allclose(got, _features_numpy(n, k, w), rtol=1e-5, atol=1e-6)


def test_batch_config_space():
    space = learn_batched.config_space()
    assert len(space) == learn_batched.n_cfg() == 54 <= 63  # the network's 63 class outputs
    assert len(set(space)) == len(space)
    assert {b for b, _, _, _ in space} == {128, 256, 512}
    assert {i for _, i, _, _ in space} == {2, 4, 8}
    assert {c for _, _, c, _ in space} == {1, 2, 4}
    assert {wv for _, _, _, wv in space} == {0, learn_batched.DEFAULT_WAVE}
    for w in (4, 8, 16):
        assert space[learn_batched.default_class(None, w)] == (512, 4, 4, learn_batched.DEFAULT_WAVE)
    assert space[learn_batched.default_class(None, 32)] == (256, 4, 4, learn_batched.DEFAULT_WAVE)


def test_soft_targets_ignore_infeasible_configurations():
    T = np.array([[1.0, 1.01, np.inf] + [2.0] * 51], np.float32)
    t = learn_batched.soft_targets(T, tau=0.03)
    assert t.shape == (1, 64)
    assert abs(t[0].sum() - 1) < 1e-5 and t[0, 2] == 0 and t[0, 54:].sum() == 0
    assert t[0, 0] > t[0, 1] > t[0, 3]


def test_shipped_batch_predictor_beats_the_method_without_it():
    """Held-out list mixes, every configuration timed on a B200 (median of 5 launches): the
    network's choice (CPU oracle forward of the shipped weights, best configuration among those
    whose tile fits the mix's longest list, as the library chooses) is within 5 % of the exhaustive
    best on average, better than the default configuration (the method without the network) and
    than the best single fixed configuration."""
    from pathlib import Path
    from oracle import mlp_ref
    root = Path(__file__).resolve().parent.parent
    p = np.load(root / "redzone_b200" / "data" / "batch_predictor.npz")["params"].astype(np.float64)
    h = np.load(root / "tests" / "golden" / "batch_predictor_heldout.npz")
    assert [tuple(x) for x in h["space"]] == learn_batched.config_space()
    _, _, out = mlp_ref.forward(p, h["X"].astype(np.float64))
    pred = learn_batched.choose(out, h["X"])
    rep = learn_batched.evaluate(pred, h["T"], h["default_cls"])
    assert rep["infeasible_predictions"] == 0 and rep["default_infeasible"] == 0
    assert rep["regret_mean"] <= 0.05, rep
    assert rep["regret_mean"] < rep["default_regret_mean"] and rep["regret_mean"] < rep["best_fixed_regret_mean"]
