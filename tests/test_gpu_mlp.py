"""GPU checks of the learned predictor's hand-written kernels against the CPU oracle."""
import ctypes
import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from oracle import mlp_ref
from redzone_b200 import learn, workloads

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def batch(seed, nb):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (nb, mlp_ref.N_IN)).astype(np.float32)
    t = rng.uniform(0, 1, (nb, mlp_ref.N_OUT)).astype(np.float32)
    t[:, : mlp_ref.N_CFG] /= t[:, : mlp_ref.N_CFG].sum(1, keepdims=True)
    t[:, mlp_ref.N_CFG] = rng.integers(0, 2, nb)
    return x, t


@pytest.mark.parametrize("nb", [1, 37, 512])
def test_gradients_match_cpu_oracle(ctx, nb):
    m = learn.Mlp(ctx, seed=3)
    p = np.random.default_rng(nb).normal(0, 0.25, m.nparams).astype(np.float32)
    m.set_params(p)
    x, t = batch(nb, nb)
    loss, g = m.gradients(x, t)
    ref_loss, ref_g = mlp_ref.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    np.testing.assert_allclose(g, ref_g, rtol=2e-3, atol=2e-6)
    m.close()


def test_forward_matches_cpu_oracle(ctx):
    m = learn.Mlp(ctx, seed=5)
    p = m.params()
    x, _ = batch(9, 300)
    out = m.forward(x)
    _, _, ref = mlp_ref.forward(p.astype(np.float64), x.astype(np.float64))
    np.testing.assert_allclose(out, ref, rtol=1e-4, atol=1e-5)
    m.close()


@pytest.mark.parametrize("dist,n,k,w", [("uniform", 1 << 20, 1 << 14, 4), ("clustered", 1 << 22, 1 << 12, 16),
                                        ("tail", 1 << 24, 1 << 16, 4), ("uniform", 5000, 77, 8),
                                        ("uniform", 1 << 16, 1 << 15, 32)])
def test_feature_kernel_matches_cpu_oracle(ctx, dist, n, k, w):
    idx = workloads.make(dist, n, k, seed=k)
    d = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    f = np.zeros(12, np.float32)
    import ctypes
    from redzone_b200 import _native
    st = _native.lib.rz_mlp_features(ctx.handle, ctypes.c_void_p(d.data_ptr()), n, k, w,
                                     f.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert st == 0
    np.testing.assert_allclose(f, mlp_ref.features(idx, n, k, w), rtol=1e-4, atol=1e-5)


def test_training_on_the_gpu_learns_a_separable_task(ctx):
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, (4000, 12)).astype(np.float32)
    label = (x[:, 0] * 7).astype(int) * 9 + (x[:, 1] * 9).astype(int)  # 63 classes on a grid
    t = np.zeros((4000, mlp_ref.N_OUT), np.float32)
    t[np.arange(4000), label] = 1.0
    t[:, mlp_ref.N_CFG] = (x[:, 2] > 0.5)
    m = learn.Mlp(ctx, seed=2)
    before = m.gradients(x[:512], t[:512])[0]
    after = m.train(x, t, epochs=60, batch=256, lr=3e-3, seed=1)
    assert after < 0.5 * before
    cls, bit = m.predict(x)
    assert np.mean(cls == label) > 0.8 and np.mean(bit == t[:, mlp_ref.N_CFG]) > 0.95
    m.close()


def test_predicted_configuration_keeps_results_bit_exact(ctx):
    m = learn.Mlp(ctx, seed=11)
    m.attach()
    for n, k in [(1 << 20, 1 << 14), (1 << 18, 1 << 16), (1 << 16, 300)]:
        host = np.arange(n, dtype=np.uint32)
        idx = workloads.uniform(n, k, seed=n + k)
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        ctx.remove(d, torch.from_numpy(idx.astype(np.int32)).to(DEV), flags=rz.RZ_USE_PREDICTOR | rz.RZ_SYNC)
        exp = host.copy()
        oracle.remove(exp, idx)
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], exp[: n - k])
    m.close()


def test_shipped_predictor_on_the_gpu_matches_the_oracle_and_its_regret(ctx):
    """The shipped weights run through the library's own forward kernel: predictions agree with the
    CPU oracle (up to near-ties) and keep the held-out regret within 5 % of exhaustive autotune."""
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    p = np.load(root / "redzone_b200" / "data" / "predictor.npz")["params"]
    h = np.load(root / "tests" / "golden" / "predictor_heldout.npz")
    X, T, dcls = h["X"], h["T"], h["default_cls"]
    m = learn.Mlp(ctx)
    m.set_params(p)
    cls, bit = m.predict(X)
    _, _, ref = mlp_ref.forward(p.astype(np.float64), X.astype(np.float64))
    agree = cls == ref[:, : mlp_ref.N_CFG].argmax(1)
    assert agree.mean() > 0.99
    rep = learn.evaluate(cls, bit, T, dcls)
    assert rep["regret_mean"] <= 0.05 and rep["regret_mean"] < rep["default_regret_mean"]
    m.close()


def test_attached_predictor_is_used_and_falls_back(ctx):
    """rz_remove with RZ_USE_PREDICTOR runs the network's configuration; without a network
    attached the same flag falls back to the tables / defaults. Results are bit-exact either way."""
    n, k = 1 << 20, 1 << 14
    host = np.arange(n, dtype=np.uint32)
    idx = workloads.uniform(n, k, seed=5)
    exp = host.copy()
    oracle.remove(exp, idx)
    d_idx = torch.from_numpy(idx.astype(np.int32)).to(DEV)
    for attach in (True, False):
        c = rz.Context(0)
        m = learn.attach_default(c) if attach else None
        assert (m is not None) == attach
        cfg = rz.LaunchCfg()
        st = rz._native.lib.rz_predict_cfg(c.handle, ctypes.c_void_p(d_idx.data_ptr()), n, k, 4, ctypes.byref(cfg))
        if attach:
            assert st == 0
            p = np.load(learn.DATA / "predictor.npz")["params"].astype(np.float64)
            _, _, o = mlp_ref.forward(p, mlp_ref.features(idx, n, k, 4)[None, :].astype(np.float64))
            q = learn.config_space().index((cfg.block, cfg.items, cfg.ctas_per_sm, cfg.schedule))
            assert o[0, q] >= o[0, : mlp_ref.N_CFG].max() - 1e-3  # the oracle's choice, up to a near-tie
        else:
            assert st == rz._native.RZ_ERR_UNSUPPORTED  # no network: rz_remove falls back to the tables
        d = torch.from_numpy(host.view(np.int32).copy()).to(DEV)
        c.remove(d, torch.from_numpy(idx.astype(np.int32)).to(DEV), flags=rz.RZ_USE_PREDICTOR | rz.RZ_SYNC)
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], exp[: n - k])
        if m is not None:
            m.close()
        c.close()
