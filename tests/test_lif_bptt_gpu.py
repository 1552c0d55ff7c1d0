"""The differentiable form on the GPU: the adjoint kernel's gradients against
the float64 PyTorch reference (exact spikes pinned to the kernel's forward;
relaxed model), against finite differences of the relaxed forward, invariance
under the checkpoint interval, and the exactness of the spiking forward."""

import numpy as np
import pytest
import torch

import lif_reference as ref
from nemo_b200.lif import LIFNetwork, lif_backward, lif_bptt, lif_forward, poisson_bits, rate_loss, \
    sinusoid_target

pytestmark = pytest.mark.gpu

N, C, FAN, INFAN, T, B, BIN = 300, 40, 30, 10, 120, 8, 10


def _setup(checkpoint=25, seed=1):
    net = LIFNetwork.random(N, FAN, C, INFAN, seed=seed, checkpoint=checkpoint, bin_steps=BIN)
    w = net.initial_weights(seed=seed, scale_rec=0.35, scale_in=1.2)
    bits, spikes = poisson_bits(T, C, B, rate_hz=60.0, seed=seed)
    target = sinusoid_target(T // BIN, BIN)
    return net, w, bits, spikes, target


def _spikes_from_bits(s_bits, trials):
    words = s_bits.cpu().numpy().view(np.uint32)
    return np.stack([(words >> np.uint32(b)) & 1 for b in range(trials)], axis=2).astype(bool)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_exact_adjoint_matches_float64_reference():
    net, w, bits, ins, target = _setup()
    wg = w.clone().requires_grad_(True)
    counts = lif_bptt(wg, bits, net, B)
    assert counts.sum().item() > 0, "the network must spike"
    loss = rate_loss(counts, net.n, BIN, target)
    loss.backward()
    # the reference differentiates the same spike trains
    _, saved = lif_forward(net, w, bits, B)
    spikes = _spikes_from_bits(saved[0], B)
    w64 = torch.tensor(w.cpu().numpy().astype(np.float64), requires_grad=True)
    c64 = ref.counts(net, w64, ins, B, spikes=spikes)
    assert np.array_equal(c64.detach().numpy(), counts.detach().cpu().numpy().astype(np.float64))
    rate_loss(c64, net.n, BIN, target.cpu().double()).backward()
    g, g64 = wg.grad.cpu().numpy().astype(np.float64), w64.grad.numpy()
    assert np.abs(g64).max() > 0
    assert _rel(g, g64) <= 1e-3
    big = np.abs(g64) > 1e-3 * np.abs(g64).max()
    assert np.all(np.abs(g[big] - g64[big]) <= 1e-3 * np.abs(g64[big]) + 1e-6 * np.abs(g64).max())


def test_forward_spikes_are_exact():
    """Wherever the float64 membrane potential is clearly away from the
    threshold, the kernel's float32 spike decision is the same."""
    net, w, bits, ins, _ = _setup(seed=3)
    _, saved = lif_forward(net, w, bits, B)
    spikes = _spikes_from_bits(saved[0], B)
    # recompute u in float64 along the kernel's own spike trains
    pre = torch.as_tensor(net.pres)
    tgt = torch.as_tensor(net.targets)
    rec = pre < net.n
    w64 = torch.tensor(w.cpu().numpy().astype(np.float64))
    v = torch.zeros(B, net.n, dtype=torch.float64)
    prev = torch.zeros(B, net.n, dtype=torch.float64)
    checked = 0
    for t in range(T):
        x = torch.zeros(B, pre.numel(), dtype=torch.float64)
        x[:, rec] = prev[:, pre[rec]]
        x[:, ~rec] = torch.as_tensor(ins[t][pre[~rec] - net.n].T.astype(np.float64))
        u = net.beta * v + torch.zeros(B, net.n, dtype=torch.float64).index_add(1, tgt, x * w64)
        s = torch.as_tensor(spikes[t].T.astype(np.float64))
        clear = (u - net.theta).abs() > 1e-4
        assert torch.equal((u >= net.theta)[clear], (s > 0)[clear]), t
        checked += int(clear.sum())
        v = u - net.theta * s
        prev = s
    assert checked > 0.99 * T * B * net.n


def test_relaxed_adjoint_matches_finite_differences():
    net, w, bits, ins, target = _setup(seed=5)
    wg = w.clone().requires_grad_(True)
    loss = rate_loss(lif_bptt(wg, bits, net, B, True), net.n, BIN, target)
    loss.backward()
    g = wg.grad.cpu().numpy().astype(np.float64)
    tgt64 = target.cpu().double()

    def loss64(wv):
        return rate_loss(ref.counts(net, wv, ins, B, relaxed=True), net.n, BIN, tgt64)

    w64 = torch.tensor(w.cpu().numpy().astype(np.float64), requires_grad=True)
    loss64(w64).backward()
    assert _rel(g, w64.grad.numpy()) <= 1e-3
    rng = np.random.default_rng(0)
    base = torch.tensor(w.cpu().numpy().astype(np.float64))
    eps = 1e-5
    order = np.argsort(-np.abs(w64.grad.numpy()))
    for k in list(order[:6]) + list(rng.choice(net.synapses, size=6, replace=False)):
        e = torch.zeros_like(base)
        e[k] = eps
        fd = (loss64(base + e) - loss64(base - e)).item() / (2 * eps)
        assert abs(g[k] - fd) <= 1e-3 * abs(fd) + 1e-6 * np.abs(g).max(), (k, g[k], fd)


def test_checkpoint_interval_does_not_change_the_gradient():
    """Recomputing from checkpoints reproduces u exactly; only the grouping
    of the weight-gradient sums over steps follows the segments, so the
    gradients agree to float32 rounding, and each is reproducible."""
    grads = []
    for K in (T, 25, 7, 7):
        net, w, bits, _, target = _setup(checkpoint=K, seed=9)
        counts, saved = lif_forward(net, w, bits, B)
        dcounts = torch.full_like(counts, 0.01) * torch.arange(counts.shape[1], device=counts.device)
        grads.append(lif_backward(net, w, bits, B, saved, dcounts).cpu().numpy())
    assert np.array_equal(grads[2], grads[3])
    for g in grads[1:]:
        assert np.allclose(g, grads[0], rtol=1e-5, atol=1e-6 * np.abs(grads[0]).max())
