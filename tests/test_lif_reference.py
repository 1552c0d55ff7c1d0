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


def test_segment_recomputation_gives_the_same_gradient():
    """counts(..., segment=K) recomputes each K-step segment in the backward
    pass (torch.utils.checkpoint): same counts and same gradient as keeping
    every step, in exact (pinned spikes) and relaxed mode, on a trial subset
    taken by indexing the trial axis."""
    net = _tiny()
    rng = np.random.default_rng(3)
    T, B = 30, 4
    ins = rng.random((T, 8, B)) < 0.3
    spikes = rng.random((T, net.n, B)) < 0.1
    sub = [3, 1]
    target = torch.tensor(20 + 10 * np.sin(np.arange(T // 5)), dtype=torch.float64)
    w0 = torch.tensor(rng.normal(0, 0.6, net.synapses), dtype=torch.float64)
    for relaxed in (False, True):
        grads = []
        for segment in (None, 7):
            w = w0.clone().requires_grad_(True)
            c = ref.counts(net, w, ins[:, :, sub], len(sub), relaxed=relaxed,
                           spikes=None if relaxed else spikes[:, :, sub], segment=segment)
            rate_loss(c, net.n, net.bin_steps, target).backward()
            grads.append((c.detach().numpy(), w.grad.numpy()))
        assert np.array_equal(grads[0][0], grads[1][0])
        assert np.allclose(grads[0][1], grads[1][1], rtol=1e-12, atol=1e-15)
        assert np.abs(grads[0][1]).max() > 0
