"""The surrogate's CPU oracle (oracle/mlp.py): analytic FP64 gradients
against central finite differences; BF16 rounding helper against torch."""
import numpy as np
import torch

from oracle import mlp as M


def test_fp64_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    sizes = M.sizes_of(5, 7, 16, 3)
    layers = [(rng.normal(0, 1 / np.sqrt(k), (n, k)), rng.normal(0, 0.1, n)) for n, k in sizes]
    x = rng.normal(size=(32, 5))
    t = rng.normal(size=(32, 7))
    loss, grads, _ = M.loss_and_grad(layers, x, t)
    g = M.flatten(grads)
    idx = rng.choice(len(g), 60, replace=False)
    fd = M.finite_difference(layers, x, t, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-6, atol=1e-9)


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).normal(size=10000) * np.logspace(-6, 6, 10000)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(M.to_bf16(x), ref)
    bits = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    np.testing.assert_array_equal(M.bf16_bits(x), bits)
