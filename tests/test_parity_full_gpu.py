"""Bit-exact parity at the sizes of the benchmark configurations, every cycle
against the oracle (the reference CPU backend restated), through the C ABI:

* the 1e8-synapse STDP network the headline benchmark runs (100,000
  Izhikevich neurons, 1000 synapses each, delays U{1..20}, excitatory
  synapses plastic, seed 1): 3 x (100 cycles in one device-resident launch,
  then applyStdp(1.0)); the fired list of every cycle and every plastic
  weight after every applyStdp;
* the 50,000-neuron mixed network (Izhikevich, IF_curr_exp, QIF, HH) with
  its Bernoulli(0.005) firing stimulus through nemo_step: the fired list of
  each of 200 cycles and the membrane potentials after them;
* the batched form: all 256 networks of sizes log-uniform in [500, 20000]
  in one simulation, 100 cycles replayed from a CUDA graph: every
  instance's fired list of every cycle against its own oracle run;
* the differentiable form at its configuration (10,000 LIF neurons, 200
  recurrent + 50 input synapses each, 32 trials of 500 steps): the spiking
  forward against float64, the adjoint's gradient of a trial subset's loss
  against the float64 PyTorch reference, and the relaxed adjoint against
  central finite differences of the float64 relaxed forward.

The reference benchmark's protocol is src/examples/common.cpp:13-121; the
order of one cycle is cpu/Simulation.cpp:95-111. Each test prints its
figures (run pytest with -s to see them)."""

import time

import numpy as np
import pytest
import torch

import lif_reference as ref
from nemo_b200 import netgen
from nemo_b200.lif import LIFNetwork, lif_backward, lif_forward, poisson_bits, rate_loss, sinusoid_target
from nemo_b200.nemo import Configuration, Library, Network, Simulation

pytestmark = pytest.mark.gpu


def _build(spec, lib, oracle, stdp=None):
    net = spec.build(Network(lib))
    conf = Configuration(lib)
    if stdp is not None:
        pre, post, limits = stdp
        conf.set_stdp_function(pre, post, *limits)
    if oracle:
        conf.set_cpu_backend()
    sim = Simulation(net, conf)
    del net
    return sim


def _weights_equal(g, o, sources, per_source, chunk=8000):
    """Every weight of the synapses of `sources` (ids (s << 32) | k, k <
    per_source) on both simulations: (mismatches, synapses compared, a
    digest of the B200 weights' bits)."""
    bad = total = 0
    digest = np.uint64(0)
    k = np.arange(per_source, dtype=np.uint64)
    for c0 in range(0, sources.size, chunk):
        src = sources[c0:c0 + chunk].astype(np.uint64)
        ids = ((src[:, None] << np.uint64(32)) | k[None, :]).ravel()
        a = g.get_weights(ids).view(np.uint32)
        b = o.get_weights(ids).view(np.uint32)
        bad += int(np.count_nonzero(a != b))
        total += ids.size
        digest = np.uint64((int(digest) * 1000003 + int(a.astype(np.uint64).sum())) % (1 << 64))
    return bad, total, int(digest)


def test_headline_stdp_network_full_size(oracle_lib):
    n, m = 100000, 1000
    spec = netgen.izhikevich_random(n, m, dmax=20, seed=1, stdp=True)
    nexc = int(n * 0.8)
    pre, post = netgen.standard_stdp()
    stdp = (pre, post, (0.0, 1.0, 0.0, -1.0))
    t0 = time.perf_counter()
    g = _build(spec, Library(), False, stdp)
    o = _build(spec, oracle_lib, True, stdp)
    del spec
    build_s = time.perf_counter() - t0
    plastic_sources = np.arange(nexc, dtype=np.uint64)
    cycle = 0
    fired_total = 0
    for epoch in range(3):
        counts = g.run(100)
        for k in range(100):
            want = o.step()
            got = g.fired_at(cycle + k)
            assert got.size == counts[k]
            assert np.array_equal(got, want), "epoch %d cycle %d: %d fired on the B200, %d in the oracle" % (
                epoch, cycle + k, got.size, want.size)
            fired_total += want.size
        cycle += 100
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
        bad, compared, digest = _weights_equal(g, o, plastic_sources, m)
        assert bad == 0, "epoch %d: %d of %d plastic weights differ" % (epoch, bad, compared)
        print("headline network: epoch %d, cycles %d..%d bit-exact, %d plastic weights equal (digest %016x)"
              % (epoch, cycle - 100, cycle - 1, compared, digest))
    assert fired_total > 300 * 100
    print("headline network: %d cycles, %d firings, 3 applyStdp, build %.1f s" % (cycle, fired_total, build_s))


def test_mixed_network_full_size(oracle_lib):
    spec = netgen.mixed_plugins(seed=2)
    n = spec.neuron_count
    rng = np.random.default_rng(5)
    g = _build(spec, Library(), False)
    o = _build(spec, oracle_lib, True)
    fired = 0
    for c in range(200):
        stim = np.nonzero(rng.random(n) < 0.005)[0].astype(np.uint32)
        a, b = g.step(fstim=stim), o.step(fstim=stim)
        assert np.array_equal(a, b), "cycle %d: %d fired on the B200, %d in the oracle" % (c, a.size, b.size)
        fired += a.size
    sample = np.arange(0, n, 97)
    va = np.array([np.float32(g.get_membrane_potential(int(i))).view(np.uint32) for i in sample])
    vb = np.array([np.float32(o.get_membrane_potential(int(i))).view(np.uint32) for i in sample])
    assert np.array_equal(va, vb)
    print("mixed network: %d neurons, 200 cycles bit-exact, %d firings, %d membrane potentials equal"
          % (n, fired, sample.size))


def test_batched_form_all_instances(oracle_lib):
    """The benchmark's 256 networks (sizes, seeds and noise scales as in the
    batched benchmark) in one simulation, 100 cycles as one CUDA-graph
    replay; each instance against its own oracle simulation."""
    from test_batch_gpu import Batch
    count, cycles = 256, 100
    sizes = netgen.batched_sizes(count, 500, 20000, seed=3)
    sig = np.random.default_rng(4).uniform(3.0, 7.0, size=count)
    specs = [netgen.izhikevich_random(int(sizes[j]), 100, dmax=20, seed=1000 + j, sigma_exc=float(sig[j]),
                                      sigma_inh=float(0.4 * sig[j])) for j in range(count)]
    lib = Library()
    batch = Batch(lib, specs)
    batch.nets = [None] * count   # the networks' host copies are not needed after construction
    oracles = [_build(s, oracle_lib, True) for s in specs]
    del specs
    batch.run_graph(cycles, cycles)
    fired = 0
    for c in range(cycles):
        per = batch.fired(c)
        for j in range(count):
            want = oracles[j].step()
            assert np.array_equal(per[j], want), "instance %d (%d neurons), cycle %d" % (j, sizes[j], c)
            fired += want.size
    assert fired > cycles * count
    print("batched form: %d instances (%d neurons), %d cycles bit-exact per instance, %d firings"
          % (count, int(sizes.sum()), cycles, fired))


# the differentiable form's configuration (its benchmark)
LIF_N, LIF_FAN, LIF_C, LIF_INFAN, LIF_T, LIF_B, LIF_BIN = 10000, 200, 500, 50, 500, 32, 10


def _lif_setup():
    net = LIFNetwork.random(LIF_N, LIF_FAN, LIF_C, LIF_INFAN, seed=7, checkpoint=50, bin_steps=LIF_BIN, kappa=10.0)
    w = net.initial_weights(seed=7, scale_in=0.35)
    bits, ins = poisson_bits(LIF_T, LIF_C, LIF_B, rate_hz=10.0, seed=8)
    target = sinusoid_target(LIF_T // LIF_BIN, LIF_BIN)
    return net, w, bits, ins, target


def _spikes(s_bits, trials):
    words = s_bits.cpu().numpy().view(np.uint32)
    return np.stack([(words >> np.uint32(b)) & 1 for b in range(trials)], axis=2).astype(bool)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _subset_grad(net, w, bits, target, trials, relaxed):
    """The adjoint's gradient of the loss over `trials` only, computed in the
    32-trial launch (the other trials' count gradients are 0)."""
    counts, saved = lif_forward(net, w, bits, LIF_B, relaxed)
    c = counts.detach().clone().requires_grad_(True)
    rate_loss(c[trials], net.n, LIF_BIN, target).backward()
    return counts, saved, lif_backward(net, w, bits, LIF_B, saved, c.grad, relaxed).cpu().numpy().astype(np.float64)


def test_bptt_full_size_exact_forward_and_gradient():
    net, w, bits, ins, target = _lif_setup()
    sub = [3, 20]
    counts, saved, g = _subset_grad(net, w, bits, target, sub, False)
    spikes = _spikes(saved[0], LIF_B)
    rate = counts.sum().item() / (LIF_B * LIF_N * LIF_T / 1000.0)
    assert 1.0 < rate < 200.0, rate
    # the float64 reference differentiates the same spike trains of the
    # subset: equal counts, gradient within 1e-3
    cnet = LIFNetwork.random(LIF_N, LIF_FAN, LIF_C, LIF_INFAN, seed=7, checkpoint=50, bin_steps=LIF_BIN, kappa=10.0,
                             device="cpu")
    w64 = torch.tensor(w.cpu().numpy().astype(np.float64), requires_grad=True)
    c64 = ref.counts(cnet, w64, ins[:, :, sub], len(sub), spikes=spikes[:, :, sub], segment=50)
    assert np.array_equal(c64.detach().numpy(), counts[sub].cpu().numpy().astype(np.float64))
    rate_loss(c64, LIF_N, LIF_BIN, target.cpu().double()).backward()
    g64 = w64.grad.numpy()
    assert np.abs(g64).max() > 0
    rel = _rel(g, g64)
    assert rel <= 1e-3, rel
    # the spiking forward: wherever the float64 membrane potential of the
    # subset is clearly away from the threshold, the same spike decision
    pre = torch.as_tensor(cnet.pres)
    tgt = torch.as_tensor(cnet.targets)
    rec = torch.nonzero(pre < LIF_N).flatten()
    inp = torch.nonzero(pre >= LIF_N).flatten()
    w64d = w64.detach()
    v = torch.zeros(len(sub), LIF_N, dtype=torch.float64)
    prev = torch.zeros_like(v)
    checked = disagree = 0
    for t in range(LIF_T):
        x_in = torch.as_tensor(ins[t][:, sub].T.astype(np.float64))
        u = net.beta * v + torch.zeros_like(v).index_add(1, tgt[rec], prev[:, pre[rec]] * w64d[rec]) \
            .index_add(1, tgt[inp], x_in[:, pre[inp] - LIF_N] * w64d[inp])
        s = torch.as_tensor(spikes[t][:, sub].T.astype(np.float64))
        clear = (u - net.theta).abs() > 1e-4
        disagree += int(((u >= net.theta) != (s > 0))[clear].sum())
        checked += int(clear.sum())
        v = u - net.theta * s
        prev = s
    assert disagree == 0
    assert checked > 0.99 * LIF_T * len(sub) * LIF_N
    print("BPTT %d neurons x %d trials x %d steps: rate %.2f Hz; trials %s: spike decisions equal float64 on %d "
          "of %d (step, neuron, trial), gradient rel. error %.2e vs float64"
          % (LIF_N, LIF_B, LIF_T, rate, sub, checked, LIF_T * len(sub) * LIF_N, rel))


def test_bptt_full_size_relaxed_gradient_and_finite_differences():
    net, w, bits, ins, target = _lif_setup()
    sub = [11]
    _, _, g = _subset_grad(net, w, bits, target, sub, True)
    cnet = LIFNetwork.random(LIF_N, LIF_FAN, LIF_C, LIF_INFAN, seed=7, checkpoint=50, bin_steps=LIF_BIN, kappa=10.0,
                             device="cpu")
    tgt64 = target.cpu().double()

    def loss64(wv, segment=None):
        return rate_loss(ref.counts(cnet, wv, ins[:, :, sub], len(sub), relaxed=True, segment=segment),
                         LIF_N, LIF_BIN, tgt64)

    w64 = torch.tensor(w.cpu().numpy().astype(np.float64), requires_grad=True)
    loss64(w64, segment=50).backward()
    g64 = w64.grad.numpy()
    rel = _rel(g, g64)
    assert rel <= 1e-3, rel
    base = torch.tensor(w.cpu().numpy().astype(np.float64))
    eps = 1e-5
    rng = np.random.default_rng(0)
    order = np.argsort(-np.abs(g64))
    worst = 0.0
    with torch.no_grad():
        for k in list(order[:2]) + list(rng.choice(net.synapses, size=2, replace=False)):
            e = torch.zeros_like(base)
            e[k] = eps
            fd = (loss64(base + e) - loss64(base - e)).item() / (2 * eps)
            err = abs(g[k] - fd)
            assert err <= 1e-3 * abs(fd) + 1e-6 * np.abs(g).max(), (k, g[k], fd)
            worst = max(worst, err / max(abs(fd), 1e-30))
    print("BPTT relaxed, trial %s: gradient rel. error %.2e vs float64 autograd; 4 central differences, worst "
          "rel. error %.2e" % (sub, rel, worst))
