"""The list-mix predictor on the GPU: the library's forward kernel agrees with the CPU oracle on
the shipped weights, keeps the held-out regret of the oracle, and a plan created with the
predictor attached (configuration chosen by the network) gives every list the canonical result."""
import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import redzone_b200 as rz
from oracle import mlp_ref
from redzone_b200 import _native, learn, learn_batched, workloads

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
ROOT = Path(__file__).resolve().parent.parent
WEIGHTS = ROOT / "redzone_b200" / "data" / "batch_predictor.npz"
HELDOUT = ROOT / "tests" / "golden" / "batch_predictor_heldout.npz"


@pytest.fixture(scope="module")
def ctx():
    c = rz.Context(0)
    yield c
    c.close()


def test_library_forward_matches_oracle_and_regret(ctx):
    p = np.load(WEIGHTS)["params"]
    h = np.load(HELDOUT)
    X, T, dcls = h["X"], h["T"], h["default_cls"]
    m = learn.Mlp(ctx)
    m.set_params(p)
    pred = learn_batched.predict(m, X)
    _, _, ref = mlp_ref.forward(p.astype(np.float64), X.astype(np.float64))
    assert np.mean(pred == learn_batched.choose(ref, X)) > 0.97  # near-ties may flip in FP32
    rep = learn_batched.evaluate(pred, T, dcls)
    assert rep["regret_mean"] <= 0.05 and rep["infeasible_predictions"] == 0
    m.close()


def _mix(seed, nl, w):
    n, k = workloads.batched_lists(nl, seed=seed, log2_hi=16.0)
    rng = np.random.default_rng(seed)
    hosts, idxs = [], []
    for ni, ki in zip(n.tolist(), k.tolist()):
        h = rng.integers(0, 1 << 32, size=(ni, w // 4), dtype=np.uint64).astype(np.uint32)
        hosts.append(h)
        idxs.append(workloads.uniform(ni, ki, seed=int(rng.integers(1 << 30))))
    return hosts, idxs


@pytest.mark.parametrize("w", [4, 8, 16])
def test_attached_predictor_picks_the_oracle_choice_and_results_are_exact(ctx, w):
    hosts, idxs = _mix(7 + w, 96, w)
    lists = [(torch.from_numpy(h.view(np.int32).copy()).to(DEV), torch.from_numpy(i.astype(np.int32)).to(DEV))
             for h, i in zip(hosts, idxs)]
    m = learn_batched.attach_default(ctx)
    assert m is not None
    cfg = _native.BatchCfg()
    descs = rz.list_descs(lists)
    assert _native.lib.rz_predict_batch_cfg(ctx.handle, descs, len(lists), w, ctypes.byref(cfg)) == 0
    p = np.load(WEIGHTS)["params"].astype(np.float64)
    f = learn_batched.features(lists, w)
    _, _, o = mlp_ref.forward(p, f[None, :].astype(np.float64))
    q = learn_batched.config_space().index((cfg.block, cfg.items, cfg.ctas_per_sm, cfg.wave))
    feas = learn_batched.feasible_mask(f[None, :])[0]
    assert feas[q] and o[0, q] >= o[0, : learn_batched.n_cfg()][feas].max() - 1e-3
    plan = rz.BatchPlan(ctx, lists)  # no configuration: the attached network chooses
    info = plan.info()
    assert (info["block"], info["items"]) == (cfg.block, cfg.items) or info["block"] < cfg.block
    plan.launch()
    torch.cuda.synchronize()
    assert ctx.sync_status() == 0
    for (d, _), h, i in zip(lists, hosts, idxs):
        exp = h.copy()
        oracle.remove(exp, i)
        n, k = h.shape[0], i.size
        assert np.array_equal(d.cpu().numpy().view(np.uint32)[: n - k], exp[: n - k])
    plan.close()
    m.close()
    # Detached: no prediction, plans fall back to the table / default.
    assert _native.lib.rz_predict_batch_cfg(ctx.handle, descs, len(lists), w, ctypes.byref(cfg)) == \
        _native.RZ_ERR_UNSUPPORTED
