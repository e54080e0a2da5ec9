"""GPU checks of the learned predictor's hand-written kernels against the CPU oracle."""
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
    label = (x[:, 0] * 6).astype(int) * 8 + (x[:, 1] * 8).astype(int)  # 48 classes on a grid
    t = np.zeros((4000, 49), np.float32)
    t[np.arange(4000), label] = 1.0
    t[:, 48] = (x[:, 2] > 0.5)
    m = learn.Mlp(ctx, seed=2)
    before = m.gradients(x[:512], t[:512])[0]
    after = m.train(x, t, epochs=60, batch=256, lr=3e-3, seed=1)
    assert after < 0.5 * before
    cls, bit = m.predict(x)
    assert np.mean(cls == label) > 0.8 and np.mean(bit == t[:, 48]) > 0.95
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
