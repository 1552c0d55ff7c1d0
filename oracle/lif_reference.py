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


def counts(net, w, in_spikes, trials, relaxed=False, spikes=None, segment=None):
    """Spike counts [trials][bins] in float64. w: float64 tensor (synapse
    order of net); in_spikes: bool [T][C][>= trials]; spikes: bool
    [T][N][>= trials] (exact mode; None: thresholds computed here); only the
    first `trials` trials are used. segment: recompute the steps of each
    segment of this many steps in the backward pass instead of keeping them
    (torch.utils.checkpoint), for networks whose per-step tensors do not all
    fit in memory; the values are the same."""
    import torch.utils.checkpoint as ckpt
    n, T = net.n, in_spikes.shape[0]
    pre = torch.as_tensor(net.pres)
    tgt = torch.as_tensor(net.targets)
    rec = torch.nonzero(pre < n).flatten()
    inp = torch.nonzero(pre >= n).flatten()
    pre_rec, tgt_rec = pre[rec], tgt[rec]
    pre_inp, tgt_inp = pre[inp] - n, tgt[inp]
    beta, theta, kappa = net.beta, net.theta, net.kappa
    B = trials

    def run(t0, t1, w, v, s_prev):
        """steps [t0, t1) from state (v, s_prev): the new state and the
        population spike sums of each step [t1 - t0][B]"""
        w_rec, w_inp = w[rec], w[inp]
        sums = []
        for t in range(t0, t1):
            ins = torch.as_tensor(in_spikes[t][:, :trials].T.astype(np.float64))     # [B][C]
            I = torch.zeros(B, n, dtype=torch.float64).index_add(1, tgt_rec, s_prev[:, pre_rec] * w_rec)
            I = I.index_add(1, tgt_inp, ins[:, pre_inp] * w_inp)
            u = beta * v + I
            if relaxed:
                d = u - theta
                s = d / (1.0 + kappa * d.abs())
            else:
                given = (u >= theta).double() if spikes is None else \
                    torch.as_tensor(spikes[t][:, :trials].T.astype(np.float64))
                s = _Spike.apply(u, given, theta, kappa)
            v = u - theta * s
            sums.append(s.sum(1))
            s_prev = s
        return v, s_prev, torch.stack(sums)

    v = torch.zeros(B, n, dtype=torch.float64)
    s_prev = torch.zeros(B, n, dtype=torch.float64)
    seg = T if segment is None else int(segment)
    parts = []
    for t0 in range(0, T, seg):
        t1 = min(T, t0 + seg)
        if segment is None:
            v, s_prev, sums = run(t0, t1, w, v, s_prev)
        else:
            v, s_prev, sums = ckpt.checkpoint(run, t0, t1, w, v, s_prev, use_reentrant=False)
        parts.append(sums)
    per_step = torch.cat(parts)                   # [T][B]
    return per_step.reshape(T // net.bin_steps, net.bin_steps, B).sum(1).T
