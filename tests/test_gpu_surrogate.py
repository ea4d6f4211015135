"""GPU checks of the learned surrogate: the tcgen05 BF16 GEMM against numpy,
the network's gradients against the CPU oracle (oracle/mlp.py, which is
itself checked against finite differences), training, inference."""
import numpy as np
import pytest

from bd_aging_b200 import lib as B
from oracle import mlp as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 128, 256), (300, 200, 520), (4096, 256, 256),
                                   (256, 256, 4096), (1, 17, 8)])
def test_umma_gemm_matches_numpy(m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.normal(size=(m, k))
    b = rng.normal(size=(n, k))
    c = B.umma_gemm_bf16(M.bf16_bits(a), M.bf16_bits(b))
    ref = M.to_bf16(a) @ M.to_bf16(b).T
    # FP32 accumulation of exact BF16 products
    scale = np.abs(M.to_bf16(a)) @ np.abs(M.to_bf16(b)).T
    assert np.all(np.abs(c - ref) <= 1e-5 * scale + 1e-6)


def _net(width, depth, batch, seed=3, n_in=5, n_out=34):
    s = B.Surrogate(n_in=n_in, n_out=n_out, width=width, depth=depth, batch=batch, seed=seed)
    rng = np.random.default_rng(seed)
    layers = [(rng.normal(0, 1 / np.sqrt(k), (nn, k)), rng.normal(0, 0.2, nn)) for nn, k in s.sizes()]
    s.set_params(M.flatten(layers).astype(np.float32))
    layers = M.unflatten(s.get_params().astype(np.float64), s.sizes())
    x = rng.normal(size=(batch, n_in))
    t = rng.normal(size=(batch, n_out))
    return s, layers, x, t


@pytest.mark.parametrize("width,depth,batch", [(64, 2, 256), (192, 3, 512), (256, 4, 4096)])
def test_gradients_match_oracle(width, depth, batch):
    s, layers, x, t = _net(width, depth, batch)
    g, loss = s.gradients(x.astype(np.float32), t.astype(np.float32))
    lo, grads, _ = M.loss_and_grad(layers, x.astype(np.float32), t.astype(np.float32), bf16=True)
    go = M.flatten(grads)
    # BF16 storage of activations and dZ: agreement to a few BF16 ulps overall
    assert abs(loss - lo) <= 1e-3 * lo
    cos = float(g @ go / (np.linalg.norm(g) * np.linalg.norm(go)))
    assert cos > 0.9999, cos
    assert np.max(np.abs(g - go)) <= 2e-2 * np.max(np.abs(go))
    # and the exact FP64 network (no BF16 rounding) agrees in direction
    _, g64, _ = M.loss_and_grad(layers, x, t, bf16=False)
    g64 = M.flatten(g64)
    assert float(g @ g64 / (np.linalg.norm(g) * np.linalg.norm(g64))) > 0.999


def test_predict_matches_oracle():
    s, layers, x, _ = _net(256, 4, 4096, seed=9)
    xs = x[:5000 % 4096 + 900]
    y = s.predict(xs.astype(np.float32))
    yo = M.predict(layers, xs.astype(np.float32), bf16=True)
    assert np.max(np.abs(y - yo)) <= 2e-2 * np.max(np.abs(yo))


def test_training_fits_a_smooth_function():
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, size=(20000, 5)).astype(np.float32)
    w = rng.normal(size=(5, 34))
    y = np.tanh(x @ w * 0.7).astype(np.float32) + 0.1 * np.sin(3 * x[:, :1])
    s = B.Surrogate(batch=4096, seed=11)
    s.set_data(x, y)
    first = s.train(1, lr=1e-3)
    last = s.train(400, lr=1e-3)
    assert last < 0.05 * first, (first, last)
    xt = rng.uniform(-1, 1, size=(3000, 5)).astype(np.float32)
    yt = np.tanh(xt @ w * 0.7) + 0.1 * np.sin(3 * xt[:, :1])
    err = np.sqrt(np.mean((s.predict(xt) - yt) ** 2))
    assert err < 0.1, err


def test_proposals_beat_a_uniform_grid():
    """Ablation: with the same number of simulated temperatures, surrogate
    proposals locate the F_s = 0.5 crossing closer to the dense-sweep truth
    than a uniform grid does."""
    from bd_aging_b200 import surrogate as S
    r = S.crossing_study(budget=6, truth_points=24)
    assert 0.05 < r["t_star"] < 1.0, r
    assert r["err_surrogate"] < r["err_grid"], r
    assert r["err_surrogate"] < 0.05, r


def test_held_out_fs_error_below_0_02():
    """Trained on about 1e5 samples of one ragged batched engine run (256
    replicas: N in [500, 8000], phi in [0.50, 0.60], T_final in [0.05, 1.0],
    dt = 1e-5, 16 waiting times x 8 lags x 3 wave numbers), the surrogate
    predicts F_s of plain N = 4000 runs at fixed settings it has not seen
    (phi in {0.525, 0.575} x T_final in {0.2, 0.45, 0.7, 0.9}, 4 seeds
    averaged) within 0.02 on average."""
    from bd_aging_b200 import surrogate as S
    X, Y = S.build_batched_dataset(replicas=256, seed=11)
    assert len(X) > 90000
    model = S.SurrogateModel(seed=3)
    model.fit(X, Y, steps=4000, lr=1e-3)
    mean_err, max_err, n = S.held_out_batched_fs_error(model)
    model.close()
    assert n > 1000
    assert mean_err < 0.02, (mean_err, max_err)
