"""The float64 reference of the differentiable form against central finite
differences of its relaxed forward (CPU)."""

import numpy as np
import torch

import lif_reference as ref
from nemo_b200.lif import LIFNetwork, rate_loss


def _tiny():
    net = LIFNetwork.random(24, 6, 8, 3, seed=2, checkpoint=5, bin_steps=5, device="cpu", kappa=10.0)
    return net


def test_relaxed_reference_gradient_matches_finite_differences():
    net = _tiny()
    rng = np.random.default_rng(0)
    T, B = 30, 3
    ins = rng.random((T, 8, B)) < 0.2
    w0 = torch.tensor(rng.normal(0, 0.6, net.synapses), dtype=torch.float64)
    target = torch.tensor(20 + 10 * np.sin(np.arange(T // 5)), dtype=torch.float64)

    def loss(w):
        return rate_loss(ref.counts(net, w, ins, B, relaxed=True), net.n, net.bin_steps, target)

    w = w0.clone().requires_grad_(True)
    loss(w).backward()
    g = w.grad.numpy()
    eps = 1e-6
    for k in rng.choice(net.synapses, size=12, replace=False):
        e = torch.zeros_like(w0)
        e[k] = eps
        fd = (loss(w0 + e) - loss(w0 - e)).item() / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-4 * abs(fd), (k, fd, g[k])
