"""The sharded simulation on one GPU: `world` shards of one network, each a
simulation of its own (own stream and device memory) run in turn every
cycle, their fired words exchanged in the process. Every cycle's firing
equals the oracle's unsharded simulation, and so do the fixed-point weights
after STDP. No kernel waits on another: each shard's launches complete on
their own."""

import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, NemoError, Network, ShardedSimulation, Simulation

pytestmark = pytest.mark.gpu

LIMITS = (0.0, 1.0, 0.0, -1.0)


def _shards(spec, world, stdp=None):
    lib = Library()
    net = spec.build(Network(lib))
    shards = []
    for rank in range(world):
        conf = Configuration(lib)
        if stdp is not None:
            conf.set_stdp_function(stdp[0], stdp[1], *LIMITS)
        shards.append(ShardedSimulation(net, conf, rank, world))
    return net, shards


def _oracle(spec, oracle_lib, stdp=None):
    net = spec.build(Network(oracle_lib))
    conf = Configuration(oracle_lib)
    if stdp is not None:
        conf.set_stdp_function(stdp[0], stdp[1], *LIMITS)
    conf.set_cpu_backend()
    return net, Simulation(net, conf)


def _cycle(shards, fstim=(), istim=()):
    """One cycle of every shard: local updates, the in-process exchange (the
    shards in rank order cover the warps in order), delivery."""
    words = np.concatenate([s.step_local(fstim, istim) for s in shards])
    assert words.size == shards[0].total_words
    fired = [s.deliver(words) for s in shards]
    for f in fired[1:]:
        assert np.array_equal(f, fired[0])
    return fired[0]


@pytest.mark.parametrize("world", [1, 2, 3])
def test_sharded_stdp_network(oracle_lib, world):
    """Izhikevich network with thalamic noise and exponential STDP on the
    excitatory synapses, applyStdp every 100 cycles: identical firing, and
    every synapse's weight, read on the shard that holds it, identical."""
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=4, stdp=True)
    stdp = netgen.standard_stdp()
    net, shards = _shards(spec, world, stdp)
    onet, o = _oracle(spec, oracle_lib, stdp)
    total = 0
    for epoch in range(3):
        for c in range(100):
            a, b = _cycle(shards), o.step()
            assert np.array_equal(a, b), "epoch %d cycle %d" % (epoch, c)
            total += a.size
        for s in shards:
            s.apply_stdp(1.0)
        o.apply_stdp(1.0)
    assert total > 300
    for src in range(0, 2000, 7):
        expected = {int(sid): o.get_synapse_weight(int(sid)) for sid in o.get_synapses_from(src)}
        got = {}
        for s in shards:
            for sid in s.get_synapses_from(src):
                assert int(sid) not in got
                got[int(sid)] = s.get_synapse_weight(int(sid))
        assert got == expected, src


def test_sharded_mixed_models_with_stimulus(oracle_lib):
    """Izhikevich, IF_curr_exp, QIF and Hodgkin-Huxley populations (eight
    device lanes per HH neuron) over three shards, with firing and current
    stimulus every cycle given to every shard (each applies its own
    neurons' entries): identical firing every cycle."""
    spec = netgen.mixed_plugins(n_iz=700, n_lif=500, n_qif=300, n_hh=61, m=60, dmax=10, seed=5)
    n = spec.neuron_count
    net, shards = _shards(spec, 3)
    onet, o = _oracle(spec, oracle_lib)
    rng = np.random.default_rng(3)
    total = 0
    for c in range(120):
        fstim = np.nonzero(rng.random(n) < 0.01)[0]
        ii = np.nonzero(rng.random(n) < 0.02)[0]
        istim = [(int(i), float(rng.normal(5, 5))) for i in ii]
        a, b = _cycle(shards, fstim, istim), o.step(fstim=fstim, istim=istim)
        assert np.array_equal(a, b), "cycle %d" % c
        total += a.size
    assert total > 0


def test_shard_protocol_errors():
    """A shard runs only through step_local + deliver, in that order."""
    spec = netgen.izhikevich_random(300, 20, dmax=5, seed=1)
    net, shards = _shards(spec, 2)
    s = shards[0]
    with pytest.raises(NemoError):
        Simulation.step(s)
    with pytest.raises(NemoError):
        s.deliver(np.zeros(s.total_words, np.uint32))
    s.step_local()
    with pytest.raises(NemoError):
        s.step_local()
    with pytest.raises(ValueError):
        s.deliver(np.zeros(s.total_words + 1, np.uint32))


@pytest.mark.parametrize("world", [1, 3])
def test_sharded_device_exchange(oracle_lib, world):
    """The device-resident exchange (nemo_b200_shard_step_async /
    _deliver_async): each shard's words go to a CUDA tensor, the cycle's
    words of all shards are concatenated on the current stream (as the NCCL
    all-gather does across processes), and delivery reads them there; no word
    crosses to host memory and nothing waits on the host inside a cycle. The
    firing of every cycle, read afterwards with fired_at, and the weights
    after STDP equal the oracle's."""
    import torch
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=4, stdp=True)
    stdp = netgen.standard_stdp()
    net, shards = _shards(spec, world, stdp)
    onet, o = _oracle(spec, oracle_lib, stdp)
    stream = torch.cuda.current_stream().cuda_stream
    cycle = 0
    for epoch in range(2):
        for c in range(100):
            locals_ = []
            for s in shards:
                local = torch.empty(s.words, dtype=torch.int32, device="cuda")
                s.lib.call("nemo_b200_shard_step_async", s.handle, None, 0, None, None, 0, local.data_ptr(), stream)
                locals_.append(local)
            all_words = torch.cat(locals_)
            for s in shards:
                s.lib.call("nemo_b200_shard_deliver_async", s.handle, all_words.data_ptr(), stream)
            for s in shards:
                s._in_flight = (locals_, all_words)
            cycle += 1
        for s in shards:
            s.stream_wait()
        for k in range(cycle - 100, cycle):
            want = o.step()
            for s in shards:
                assert np.array_equal(s.fired_at(k), want), "cycle %d" % k
        for s in shards:
            s.apply_stdp(1.0)
        o.apply_stdp(1.0)
    for src in range(0, 2000, 13):
        expected = {int(sid): o.get_synapse_weight(int(sid)) for sid in o.get_synapses_from(src)}
        got = {}
        for s in shards:
            for sid in s.get_synapses_from(src):
                got[int(sid)] = s.get_synapse_weight(int(sid))
        assert got == expected, src
