"""The differentiable form: a recurrent network of discrete leaky
integrate-and-fire neurons whose backpropagation-through-time gradient is
computed by the hand-written adjoint kernels of libnemo_b200
(``nemo_b200_lif_forward`` / ``nemo_b200_lif_backward``, model in
``nemo_b200/csrc/lif_bptt.cu``), exposed as a ``torch.autograd.Function``.

The forward is the exact spiking network (Heaviside threshold); only the
backward replaces the threshold's derivative by the fast-sigmoid surrogate
1 / (1 + kappa |u - theta|)^2. State is checkpointed every ``checkpoint``
steps and recomputed between checkpoints in the backward. Up to 32 trials run
per call (one GPU lane each).

PyTorch provides device memory and the stream; the computation is the
library's."""

import ctypes
import math

import numpy as np

from .nemo import Library

P = ctypes.POINTER


class LifNetStruct(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("C", ctypes.c_int), ("B", ctypes.c_int), ("T", ctypes.c_int),
                ("K", ctypes.c_int), ("bin_steps", ctypes.c_int),
                ("beta", ctypes.c_float), ("theta", ctypes.c_float), ("kappa", ctypes.c_float),
                ("rowptr", ctypes.c_void_p), ("pre", ctypes.c_void_p), ("colptr", ctypes.c_void_p),
                ("post", ctypes.c_void_p), ("wpos", ctypes.c_void_p), ("nnz_rec", ctypes.c_int)]


def _bind(lib):
    d = lib.dll
    if getattr(d, "_lif_bound", False):
        return d
    d.nemo_b200_lif_work_bytes.restype = ctypes.c_size_t
    d.nemo_b200_lif_work_bytes.argtypes = [P(LifNetStruct)]
    d.nemo_b200_lif_forward.restype = ctypes.c_int
    d.nemo_b200_lif_forward.argtypes = [P(LifNetStruct), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
    d.nemo_b200_lif_backward.restype = ctypes.c_int
    d.nemo_b200_lif_backward.argtypes = [P(LifNetStruct), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    d.nemo_b200_lif_error.restype = ctypes.c_char_p
    d._lif_bound = True
    return d


class LIFNetwork:
    """Connectivity (fixed) and model constants of the network. ``targets``
    and ``pres`` list the synapses: synapse k goes from presynaptic unit
    ``pres[k]`` (< n: a neuron, arriving one step later; >= n: input channel
    pres[k] - n, same step) to neuron ``targets[k]``. The weights are the
    trainable tensor, in the order of ``synapse_order`` (by target)."""

    def __init__(self, n, n_in, targets, pres, tau_m=20.0, theta=1.0, kappa=10.0, checkpoint=50,
                 bin_steps=10, device="cuda"):
        import torch
        self.n, self.n_in = int(n), int(n_in)
        targets = np.asarray(targets, np.int64)
        pres = np.asarray(pres, np.int64)
        order = np.lexsort((np.arange(targets.size), targets))   # by target, stable
        self.synapse_order = order
        self.targets = targets[order]
        self.pres = pres[order]
        rowptr = np.zeros(n + 1, np.int64)
        np.add.at(rowptr, self.targets + 1, 1)
        rowptr = np.cumsum(rowptr)
        rec = np.nonzero(self.pres < n)[0]
        corder = rec[np.lexsort((rec, self.pres[rec]))]            # recurrent, by source
        colptr = np.zeros(n + 1, np.int64)
        np.add.at(colptr, self.pres[corder] + 1, 1)
        colptr = np.cumsum(colptr)
        self.beta = float(np.float32(1.0) - np.float32(1.0) / np.float32(tau_m))
        self.theta, self.kappa = float(theta), float(kappa)
        self.checkpoint, self.bin_steps = int(checkpoint), int(bin_steps)
        self.device = device
        to = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.int32), device=device)
        self._rowptr, self._pre = to(rowptr), to(self.pres)
        self._colptr, self._post, self._wpos = to(colptr), to(self.targets[corder]), to(corder)
        self.lib = Library()
        _bind(self.lib)

    @property
    def synapses(self):
        return self.targets.size

    @classmethod
    def random(cls, n, fan_in, n_in, in_fan_in, seed=0, **kw):
        """n neurons, each with fan_in recurrent synapses from random other
        neurons and in_fan_in synapses from random input channels."""
        rng = np.random.default_rng(seed)
        tgt = np.repeat(np.arange(n), fan_in + in_fan_in)
        pre = np.empty(tgt.size, np.int64)
        for i in range(n):
            src = rng.choice(n - 1, size=fan_in, replace=False)
            src = src + (src >= i)
            chan = rng.choice(n_in, size=in_fan_in, replace=False) + n
            pre[i * (fan_in + in_fan_in):(i + 1) * (fan_in + in_fan_in)] = np.concatenate([src, chan])
        net = cls(n, n_in, tgt, pre, **kw)
        return net

    def initial_weights(self, seed=0, scale_rec=None, scale_in=None):
        """float32 weights ~N(0, 1/sqrt(fan-in)) per kind, in synapse order."""
        import torch
        rng = np.random.default_rng(seed)
        rec = self.pres < self.n
        fan_rec = max(1, int(np.round(rec.sum() / self.n)))
        fan_in = max(1, int(np.round((~rec).sum() / self.n)))
        sr = scale_rec if scale_rec is not None else 1.0 / math.sqrt(fan_rec)
        si = scale_in if scale_in is not None else 1.0 / math.sqrt(fan_in)
        w = np.where(rec, rng.normal(0.0, sr, self.synapses), rng.normal(0.0, si, self.synapses))
        return torch.tensor(w.astype(np.float32), device=self.device)

    def struct(self, trials, steps):
        if steps % self.bin_steps:
            raise ValueError("steps must be a whole number of bins")
        return LifNetStruct(self.n, self.n_in, int(trials), int(steps), self.checkpoint, self.bin_steps,
                            self.beta, self.theta, self.kappa,
                            self._rowptr.data_ptr(), self._pre.data_ptr(), self._colptr.data_ptr(),
                            self._post.data_ptr(), self._wpos.data_ptr(), int(self._post.numel()))


def _check(lib, status):
    if status != 0:
        raise RuntimeError("nemo_b200_lif: " + lib.dll.nemo_b200_lif_error().decode())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def lif_forward(net, w, in_bits, trials, relaxed=False):
    """Run the forward; returns (counts [trials][bins], saved tensors)."""
    import torch
    steps = in_bits.shape[0]
    st = net.struct(trials, steps)
    dev = w.device
    n = net.n
    s_bits = torch.zeros((steps, n), dtype=torch.int32, device=dev)
    s_float = torch.zeros((steps, n, 32) if relaxed else (1,), dtype=torch.float32, device=dev)
    ck = (steps + net.checkpoint - 1) // net.checkpoint
    v_ckpt = torch.zeros((ck, n, 32), dtype=torch.float32, device=dev)
    counts = torch.zeros((trials, steps // net.bin_steps), dtype=torch.float32, device=dev)
    work = torch.empty(net.lib.dll.nemo_b200_lif_work_bytes(ctypes.byref(st)) // 4, dtype=torch.float32,
                       device=dev)
    _check(net.lib, net.lib.dll.nemo_b200_lif_forward(
        ctypes.byref(st), w.data_ptr(), in_bits.data_ptr(), int(relaxed), s_bits.data_ptr(), s_float.data_ptr(),
        v_ckpt.data_ptr(), counts.data_ptr(), work.data_ptr(), _stream()))
    return counts, (s_bits, s_float, v_ckpt, work)


def lif_backward(net, w, in_bits, trials, saved, dcounts, relaxed=False):
    """dL/dw for dL/dcounts from a forward's saved tensors."""
    import torch
    s_bits, s_float, v_ckpt, work = saved
    st = net.struct(trials, in_bits.shape[0])
    dw = torch.zeros_like(w)
    dcounts = dcounts.contiguous().to(torch.float32)
    _check(net.lib, net.lib.dll.nemo_b200_lif_backward(
        ctypes.byref(st), w.data_ptr(), in_bits.data_ptr(), int(relaxed), s_bits.data_ptr(), s_float.data_ptr(),
        v_ckpt.data_ptr(), dcounts.data_ptr(), dw.data_ptr(), work.data_ptr(), _stream()))
    return dw


def _function():
    import torch

    class LIFBPTT(torch.autograd.Function):
        """counts = LIFBPTT.apply(w, in_bits, net, trials, relaxed): spike
        counts per trial and bin of the network run on the input spikes; the
        gradient w.r.t. w comes from the adjoint kernel."""

        @staticmethod
        def forward(ctx, w, in_bits, net, trials, relaxed=False):
            w = w.contiguous()
            counts, saved = lif_forward(net, w, in_bits, trials, relaxed)
            ctx.net, ctx.trials, ctx.relaxed = net, trials, relaxed
            ctx.saved = saved
            ctx.save_for_backward(w, in_bits)
            return counts

        @staticmethod
        def backward(ctx, dcounts):
            w, in_bits = ctx.saved_tensors
            dw = lif_backward(ctx.net, w, in_bits, ctx.trials, ctx.saved, dcounts, ctx.relaxed)
            ctx.saved = None
            return dw, None, None, None, None

    return LIFBPTT


_FN = None


def lif_bptt(w, in_bits, net, trials, relaxed=False):
    """Differentiable spike counts [trials][bins] (see LIFBPTT)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(w, in_bits, net, trials, relaxed)


def poisson_bits(steps, channels, trials, rate_hz, seed=0, device="cuda", dt_ms=1.0):
    """Input spikes [steps][channels] as int32 words, bit b = trial b."""
    import torch
    rng = np.random.default_rng(seed)
    p = rate_hz * dt_ms / 1000.0
    spikes = rng.random((steps, channels, trials)) < p
    words = np.zeros((steps, channels), np.uint64)
    for b in range(trials):
        words |= spikes[:, :, b].astype(np.uint64) << np.uint64(b)
    return torch.tensor(words.astype(np.uint32).view(np.int32), device=device), spikes


def rate_loss(counts, n, bin_steps, target_hz, dt_ms=1.0):
    """Mean squared error (Hz^2) between the population rate of each bin
    (spikes per neuron per second) and the target rate of the bin."""
    rate = counts / (n * bin_steps * dt_ms / 1000.0)
    return ((rate - target_hz) ** 2).mean()


def sinusoid_target(bins, bin_steps, mean_hz=20.0, amp_hz=10.0, freq_hz=4.0, dt_ms=1.0, device="cuda"):
    """Target rate at the bin centres: mean + amp sin(2 pi f t)."""
    import torch
    t = (np.arange(bins) + 0.5) * bin_steps * dt_ms / 1000.0
    return torch.tensor(mean_hz + amp_hz * np.sin(2 * np.pi * freq_hz * t), dtype=torch.float32, device=device)
