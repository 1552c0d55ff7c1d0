"""A plain-PyTorch float64 restatement of the discrete LIF network of
nemo_b200/csrc/lif_bptt.cu -- the oracle of the differentiable form (no
reference implementation exists; used by the tests and by bench.py's CPU
baseline of the BPTT line, never by the product): the same model, with the
spike's derivative replaced by the same fast-sigmoid surrogate through
torch.autograd, so that its gradient is the reference for the adjoint kernel.

Exact mode takes the spike trains as given (normally the kernel's own
forward), so that both sides differentiate the same trajectory; relaxed mode
uses the relaxed spike r(u - theta) = (u - theta) / (1 + kappa |u - theta|),
whose true gradient the adjoint computes in its relaxed mode."""

import numpy as np
import torch


class _Spike(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, s, theta, kappa):
        ctx.save_for_backward(u)
        ctx.theta, ctx.kappa = theta, kappa
        return s

    @staticmethod
    def backward(ctx, g):
        (u,) = ctx.saved_tensors
        a = 1.0 + ctx.kappa * (u - ctx.theta).abs()
        return g / (a * a), None, None, None


def counts(net, w, in_spikes, trials, relaxed=False, spikes=None):
    """Spike counts [trials][bins] in float64. w: float64 tensor (synapse
    order of net); in_spikes: bool [T][C][trials]; spikes: bool [T][N][trials]
    (exact mode; None: thresholds computed here)."""
    n, T = net.n, in_spikes.shape[0]
    pre = torch.as_tensor(net.pres)
    tgt = torch.as_tensor(net.targets)
    rec = pre < n
    inp = ~rec
    beta, theta, kappa = net.beta, net.theta, net.kappa
    B = trials
    v = torch.zeros(B, n, dtype=torch.float64)
    s_prev = torch.zeros(B, n, dtype=torch.float64)
    bins = T // net.bin_steps
    out = []
    acc = torch.zeros(B, dtype=torch.float64)
    ins = torch.as_tensor(in_spikes[:, :, :trials].astype(np.float64))
    for t in range(T):
        x = torch.zeros(B, pre.numel(), dtype=torch.float64)
        x[:, rec] = s_prev[:, pre[rec]]
        x[:, inp] = ins[t][pre[inp] - n].T
        I = torch.zeros(B, n, dtype=torch.float64).index_add(1, tgt, x * w)
        u = beta * v + I
        if relaxed:
            d = u - theta
            s = d / (1.0 + kappa * d.abs())
        else:
            given = (u >= theta).double() if spikes is None else \
                torch.as_tensor(spikes[t].T.astype(np.float64))
            s = _Spike.apply(u, given, theta, kappa)
        v = u - theta * s
        acc = acc + s.sum(1)
        if (t + 1) % net.bin_steps == 0:
            out.append(acc)
            acc = torch.zeros(B, dtype=torch.float64)
        s_prev = s
    return torch.stack(out, 1)
