"""Known-answer tests of the reference (src/test/test.cpp, src/test/stdp.cpp,
src/test/networks.cpp), run against the oracle on the CPU and against the B200
library on the GPU (the ``lib`` fixture)."""

import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import NemoError, Network, Simulation

from conftest import configuration


def make_sim(lib, spec, stdp=False, conf=None):
    net = spec.build(Network(lib))
    conf = conf or configuration(lib, stdp)
    return net, Simulation(net, conf)


def add_excitatory(net, t, idx, sigma=0.0):
    """src/test/utils.cpp:106-113"""
    r = np.float32(0.5)
    b = np.float32(0.25) - np.float32(0.05) * r
    v = np.float32(-65.0)
    net.add_neuron(t, idx, np.float32(0.02) + np.float32(0.08) * r, b, v, 2.0, sigma, b * v, v)


# ---- neuron count: src/test/test.cpp:155-177 (network construction only,
# so both libraries run it on the host) ----

@pytest.mark.parametrize("which", ["oracle", "b200"])
@pytest.mark.parametrize("start,step", [(0, 1), (1000, 1), (0, 5), (1000, 5)])
def test_neuron_count(which, start, step):
    from conftest import ensure_oracle
    from nemo_b200.nemo import Library
    lib = Library(ensure_oracle()) if which == "oracle" else Library()
    net = Network(lib)
    for i in range(2000):
        net.add_neuron_iz(start + i * step, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7)
    assert net.neuron_count() == 2000


# ---- ring networks: src/test/test.cpp:302-328, 474-490 ----

@pytest.mark.parametrize("ncount,delay", [(1000, 1), (1024, 1), (2000, 1), (4000, 1), (2000, 20), (2000, 63)])
def test_ring(lib, ncount, delay):
    _, sim = make_sim(lib, netgen.ring(ncount, delay=delay))
    sim.step(fstim=[0])
    duration = ncount * 5 // 2
    for ms in range(1, duration):
        fired = sim.step()
        if delay == 1:
            assert list(fired) == [ms % ncount]
        elif ms % delay == 0:
            assert list(fired) == [(ms // delay) % ncount]
        else:
            assert len(fired) == 0


def test_double_ring(lib):
    """src/test/test.cpp:331-367: output order within a cycle is ascending."""
    ncount = 512
    net = Network(lib)
    a = netgen.ring(ncount, 0, delay=1)
    b = netgen.ring(ncount, ncount, delay=2)
    a.build(net)
    b.build(net)
    sim = Simulation(net, configuration(lib))
    sim.step(fstim=[0, ncount])
    for ms in range(1, ncount * 5 // 2):
        fired = list(sim.step())
        if ms % 2 == 0:
            assert fired == [ms % ncount, ncount + (ms // 2) % ncount]
        else:
            assert fired == [ms % ncount]


def test_max_delay_64_delivers_nothing(lib):
    """With a 64 ms synapse the reference's valid-spike mask is built with a
    64-bit shift by 64, which x86-64 evaluates modulo 64 (src/nemo/cpu/
    Simulation.cpp:264): no spike is ever delivered."""
    spec = netgen.ring(100, delay=1)
    spec.delay[-1] = 64
    _, sim = make_sim(lib, spec)
    sim.step(fstim=[0])
    for _ in range(10):
        assert len(sim.step()) == 0


# ---- stimulus: src/test/test.cpp:208-298 ----

def test_firing_stimulus(lib):
    ncount, cycles = 3000, 1000
    net = Network(lib)
    t = net.add_neuron_type("Izhikevich")
    add_excitatory(net, t, np.arange(ncount))
    sim = Simulation(net, configuration(lib))
    rng = np.random.default_rng(1)
    for _ in range(cycles):
        fstim = np.nonzero(rng.random(ncount) < 10.0 / ncount)[0]
        fired = sim.step(fstim=fstim)
        assert list(fired) == sorted(fstim.tolist())


def test_current_stimulus(lib):
    ncount = 1500
    _, sim = make_sim(lib, netgen.ring(ncount))
    sim.step(istim=[(5, 0.001), (8, 0.001), (0, 1000.0), (100, 0.001), (1, 0.001)])
    for ms in range(1, ncount * 2):
        assert list(sim.step()) == [ms % ncount]


def test_invalid_current_stimulus(lib):
    ncount = 1000
    _, sim = make_sim(lib, netgen.ring(ncount))
    sim.step()
    sim.step()
    with pytest.raises(NemoError) as e:
        sim.step(istim=[(ncount + 1, 0.5)])
    assert e.value.status == 6


def test_invalid_firing_stimulus(lib):
    _, sim = make_sim(lib, netgen.ring(100))
    with pytest.raises(NemoError) as e:
        sim.step(fstim=[1000])
    assert e.value.status == 6


# ---- fixed-point saturation: src/test/test.cpp:417-472 ----

def test_fixed_point_saturation(lib):
    net = Network(lib)
    iz = net.add_neuron_type("Izhikevich")
    INPUT0, INPUT1, OUT_SAT, OUT_REF, OUT_WEAK, N = range(6)
    params = [0.02, 0.2, -65.0, 8.0, 0.0, -13.0, -65.0]
    for n in range(N):
        net.add_neuron(iz, n, *params)
    net.add_synapse(INPUT0, OUT_REF, 1, 1024.0, False)
    net.add_synapse(INPUT1, OUT_REF, 1, 1024.0, False)
    net.add_synapse(INPUT0, OUT_WEAK, 1, 1000.0, False)
    net.add_synapse(INPUT1, OUT_WEAK, 1, 1000.0, False)
    net.add_synapse(INPUT0, OUT_SAT, 1, 1100.0, False)
    net.add_synapse(INPUT1, OUT_SAT, 1, 1100.0, False)
    sim = Simulation(net, configuration(lib))
    assert len(sim.step(fstim=[INPUT0, INPUT1])) == 2
    assert len(sim.step()) == 3
    u_ref = sim.get_neuron_state(OUT_REF, 0)
    u_weak = sim.get_neuron_state(OUT_WEAK, 0)
    u_sat = sim.get_neuron_state(OUT_SAT, 0)
    assert abs(u_ref - u_weak) > 1e-5
    assert abs(u_ref - u_sat) < 1e-5


def test_fixed_point_overflow_rejected(lib):
    net = Network(lib)
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, 0, 0.02, 0.2, -65.0, 8.0, 0.0, -13.0, -65.0)
    net.add_synapse(0, 0, 1, 4096.0, False)
    with pytest.raises(NemoError):
        Simulation(net, configuration(lib))


# ---- networks without outgoing synapses / invalid targets: src/test/networks.cpp ----

@pytest.mark.parametrize("contiguous", [True, False])
@pytest.mark.parametrize("stdp", [False, True])
def test_no_outgoing(lib, contiguous, stdp):
    ncount = 200
    idx = lambda i: i if contiguous else 50 + 3 * i
    net = Network(lib)
    t = net.add_neuron_type("Izhikevich")
    for i in range(ncount):
        add_excitatory(net, t, idx(i))
    src, tgt = [], []
    for i in range(ncount):
        if not (50 <= i < 150):
            src += [idx(i)] * ncount
            tgt += [idx(j) for j in range(ncount)]
    net.add_synapse(np.array(src), np.array(tgt), 1, 2.0, stdp)
    sim = Simulation(net, configuration(lib, stdp))
    for t_ in range(20):
        sim.step(fstim=[idx(i) for i in range(ncount) if idx(i) // 8 == t_])


def test_invalid_target(lib):
    net = Network(lib)
    t = net.add_neuron_type("Izhikevich")
    add_excitatory(net, t, np.arange(10))
    net.add_synapse(0, 20, 1, 1.0, False)
    # constructors report failure as NULL plus nemo_strerror (no status code)
    with pytest.raises(NemoError, match="Non-existing neuron index 20"):
        Simulation(net, configuration(lib))


def test_empty_network_rejected(lib):
    with pytest.raises(NemoError, match="empty network"):
        Simulation(Network(lib), configuration(lib))


def test_network_without_synapses(lib):
    """src/test/test.cpp:140-151,193-205"""
    for start in (0, 1):
        net = Network(lib)
        for n in range(start, start + 4):
            net.add_neuron_iz(n, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7)
        sim = Simulation(net, configuration(lib))
        sim.step()


# ---- index mapping: src/test/test.cpp:522-560 ----

@pytest.mark.parametrize("n0,nstep", [(1, 1), (1000000, 1), (1, 4), (1000000, 4)])
def test_non_contiguous_indices(lib, n0, nstep):
    ncount, seconds = 1000, 2

    def run(first):
        _, sim = make_sim(lib, netgen.ring(ncount, first, nstep=nstep))
        out = []
        for ms in range(seconds * 1000):
            fired = sim.step(fstim=[first] if ms == 0 else [])
            out += [(ms, int(f)) for f in fired]
        return out

    r0 = run(0)
    r1 = run(n0)
    assert len(r0) == seconds * ncount == len(r1)
    assert [(c, f) for c, f in r0] == [(c, f - n0) for c, f in r1]


# ---- neuron type mixture: src/test/test.cpp:379-414 ----

@pytest.mark.parametrize("iz_first", [True, False])
@pytest.mark.parametrize("others", [0, 1, 1000, 1023, 1025])
def test_neuron_type_mixture(lib, iz_first, others):
    szRing = 1024
    net = Network(lib)
    ring = netgen.ring(szRing)
    if iz_first:
        ring.build(net)
    poisson = net.add_neuron_type("PoissonSource")
    if others:
        net.add_neuron(poisson, np.arange(szRing, szRing + others), np.full(others, 0.001, np.float32))
    if not iz_first:
        ring.build(net)
    sim = Simulation(net, configuration(lib))
    sim.step(fstim=[0])
    for ms in range(1, 1000):
        fired = sorted(sim.step())
        assert len(fired) > 0
        assert fired[0] == ms % szRing
        if len(fired) > 1:
            assert fired[1] >= szRing


# ---- queries: src/test/test.cpp:564-659, 741-968 ----

def test_get_synapses(lib):
    spec = netgen.izhikevich_random(300, 50, dmax=20, seed=3, stdp=True)
    net, sim = make_sim(lib, spec, stdp=True)
    for src in range(300):
        s_ids = sim.get_synapses_from(src)
        n_ids = net.get_synapses_from(src)
        assert list(s_ids) == list(n_ids)
        for sid in s_ids[:10]:
            assert sim.get_synapse_target(sid) == net.get_synapse_target(sid)
            assert sim.get_synapse_delay(sid) == net.get_synapse_delay(sid)
            assert sim.get_synapse_plastic(sid) == net.get_synapse_plastic(sid)
            assert sim.get_synapse_source(sid) == src
    n0 = 1000000
    net, sim = make_sim(lib, netgen.ring(1500, n0))
    for src in range(n0, n0 + 1500):
        ids = sim.get_synapses_from(src)
        assert len(ids) == 1
        assert sim.get_synapse_target(ids[0]) == net.get_synapse_target(ids[0])


def test_write_only_synapses(lib):
    conf = configuration(lib)
    conf.set_write_only_synapses()
    net = netgen.ring(10, plastic=True).build(Network(lib))
    sim = Simulation(net, conf)
    sim.step()
    with pytest.raises(NemoError):
        sim.get_synapses_from(0)
    with pytest.raises(NemoError):
        sim.get_synapse_weight((1 << 32) | 0)


def test_synapses_from_unconnected(lib):
    net = Network(lib)
    for n in range(4):
        net.add_neuron_iz(n, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7)
    sim = Simulation(net, configuration(lib))
    sim.step()
    with pytest.raises(NemoError):
        sim.get_synapses_from(4)
    assert len(sim.get_synapses_from(3)) == 0


def test_vprobe(lib):
    net = Network(lib)
    v0 = -65.0
    net.add_neuron_iz(0, 0.02, 0.2, -65.0 + 15.0 * 0.25, 8.0 - 6.0 * 0.25, 0.2 * -65.0, v0, 5.0)
    sim = Simulation(net, configuration(lib))
    assert sim.get_membrane_potential(0) == v0


def test_duplicate_neuron(lib):
    net = Network(lib)
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, 0, *([0.0] * 7))
    with pytest.raises(NemoError):
        net.add_neuron(iz, 0, *([0.0] * 7))


def test_set_neuron(lib):
    """src/test/test.cpp:772-850: setters on the network and the simulation."""
    a, b, c, d, u, v, s = 0.02, 0.2, -65.0 + 15.0 * 0.25, 8.0 - 6.0 * 0.25, 0.2 * -65.0, -65.0, 5.0
    net = Network(lib)
    net.add_neuron_iz(0, a, b, c, d, u, v, s)
    net.add_neuron_iz(1, a, b, c, d, u, v, s)
    with pytest.raises(NemoError):
        net.set_neuron(2, a, b, c, d, s, u, v)
    net.set_neuron(0, a, b, c, d, s, u, v)
    assert net.get_neuron_parameter(0, 0) == np.float32(a)
    assert net.get_neuron_state(0, 1) == np.float32(v)
    with pytest.raises(NemoError):
        net.get_neuron_state(0, 2)
    with pytest.raises(NemoError):
        net.get_neuron_parameter(0, 5)
    net.set_neuron_parameter(1, 2, -50.0)
    assert net.get_neuron_parameter(1, 2) == -50.0
    sim = Simulation(net, configuration(lib))
    assert sim.get_neuron_parameter(1, 2) == -50.0
    assert sim.get_neuron_state(0, 0) == np.float32(u)
    sim.set_neuron_state(0, 1, -70.0)
    assert sim.get_membrane_potential(0) == -70.0
    sim.set_neuron_parameter(0, 4, 0.0)
    assert sim.get_neuron_parameter(0, 4) == 0.0
    sim.set_neuron(1, 0.1, 0.2, -60.0, 6.0, 0.0, -12.0, -60.0)
    assert sim.get_neuron_state(1, 0) == np.float32(-12.0)
    sim.step()
    with pytest.raises(NemoError):
        sim.set_neuron(1, 0.1, 0.2)
    with pytest.raises(NemoError):
        sim.get_neuron_state(7, 0)


def test_timers(lib):
    _, sim = make_sim(lib, netgen.ring(100))
    for _ in range(10):
        sim.step()
    assert sim.elapsed_simulation() == 10
    sim.reset_timer()
    assert sim.elapsed_simulation() == 0
    sim.step()
    assert sim.elapsed_simulation() == 1


# ---- STDP: src/test/stdp.cpp ----

GROUP = 2 * 768
INIT_WEIGHT = 5.0


def _dw_pre(dt):
    return np.float32(1.0) * np.exp(np.float32(dt) / np.float32(20.0))


def _dw_post(dt):
    return np.float32(-0.8) * np.exp(np.float32(-dt) / np.float32(20.0))


def _stdp_delay(local):
    return 1 + (local % 20)


def _stdp_network(lib, noise):
    """src/test/stdp.cpp:125-170"""
    net = Network(lib)
    t = net.add_neuron_type("Izhikevich")
    add_excitatory(net, t, np.arange(2 * GROUP))
    local = np.arange(GROUP)
    net.add_synapse(local, GROUP + local, _stdp_delay(local), INIT_WEIGHT, True)
    if noise:
        ls, lt = np.meshgrid(np.arange(GROUP), np.arange(GROUP), indexing="ij")
        mask = ls != lt
        ls, lt = ls[mask], lt[mask]
        net.add_synapse(ls, GROUP + lt, _stdp_delay(lt + ls), -0.00001, (lt & 1).astype(np.uint8))
    return net


def _stdp_conf(lib):
    from nemo_b200.nemo import Configuration
    conf = Configuration(lib)
    pre = np.array([_dw_pre(-i) for i in range(20)], np.float32)
    post = np.array([_dw_post(i) for i in range(20)], np.float32)
    conf.set_stdp_function(pre, post, -0.5, 2 * INIT_WEIGHT)
    if "oracle" in lib.path:
        conf.set_cpu_backend()
    return conf


def _verify_weights(sim, epoch, reward):
    checked = 0
    for local in range(GROUP):
        for sid in sim.get_synapses_from(local):
            target = sim.get_synapse_target(sid)
            if local != target % GROUP:
                continue
            delay = sim.get_synapse_delay(sid)
            assert delay == _stdp_delay(target % GROUP)
            assert sim.get_synapse_plastic(sid)
            dt = -(10 - int(delay))
            dw = _dw_post(dt - 1) if dt > 0 else _dw_pre(dt)
            expected = INIT_WEIGHT + epoch * reward * dw
            actual = sim.get_synapse_weight(sid)
            assert abs(expected - actual) <= abs(expected) * 1e-5  # 0.001 percent
            checked += 1
    assert checked == GROUP


@pytest.mark.parametrize("noise,reward", [(False, 1.0), (True, 1.0), (False, 0.8), (True, 0.9)])
def test_stdp_analytic(lib, noise, reward):
    net = _stdp_network(lib, noise)
    sim = Simulation(net, _stdp_conf(lib))
    _verify_weights(sim, 0, reward)
    for epoch in range(1, 5):
        for ms in range(100):
            fstim = []
            if ms == 10:
                fstim = list(range(GROUP))
            elif ms == 20:
                fstim = list(range(GROUP, 2 * GROUP))
            sim.step(fstim=fstim)
        sim.apply_stdp(reward)
        _verify_weights(sim, epoch, reward)


def test_apply_stdp_without_stdp_fails(lib):
    _, sim = make_sim(lib, netgen.ring(10, plastic=True))
    sim.step()
    with pytest.raises(NemoError):
        sim.apply_stdp(1.0)


def test_stdp_reward_rounding(lib):
    _, sim = make_sim(lib, netgen.ring(10, plastic=True), stdp=True)
    sim.step()
    with pytest.raises(NemoError) as e:
        sim.apply_stdp(1e-9)
    assert e.value.status == 6
    sim.apply_stdp(0.0)


def test_stdp_all_static(lib):
    spec = netgen.izhikevich_random(1000, 100, dmax=1, seed=5, stdp=False)
    _, sim = make_sim(lib, spec, stdp=True)
    for _ in range(2):
        for _ in range(200):
            sim.step()
        sim.apply_stdp(1.0)


def test_stdp_configuration_limits(oracle_lib):
    from nemo_b200.nemo import Configuration
    pre = np.exp(-np.arange(20, dtype=np.float32) / 20).astype(np.float32)
    post = pre.copy()
    conf = Configuration(oracle_lib)
    bad = [(-0.01, 1.0, -0.01, -1.0), (0.01, -1.0, -0.01, -1.0), (-0.01, -1.0, -0.01, -1.0),
           (0.01, 1.0, 0.01, -1.0), (0.01, 1.0, -0.01, 1.0), (0.01, 1.0, 0.01, 1.0),
           (1.0, 0.01, -0.01, -1.0), (0.01, 1.0, -1.0, -0.01)]
    for limits in bad:
        with pytest.raises(NemoError):
            conf.set_stdp_function(pre, post, *limits)
    long = np.ones(35, np.float32)
    with pytest.raises(NemoError):
        conf.set_stdp_function(long, long, 0.01, 1.0, -0.01, -1.0)


@pytest.mark.parametrize("stdp", [True, False])
def test_stdp_dynamic_window_length(lib, stdp):
    from nemo_b200.nemo import Configuration
    conf = Configuration(lib)
    if "oracle" in lib.path:
        conf.set_cpu_backend()
    if stdp:
        w = np.exp(-np.arange(31, dtype=np.float32) / 31).astype(np.float32)
        conf.set_stdp_function(w, w, 0.01, 1.0, -0.01, -1.0)
    net = Network(lib)
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, 0, *([0.0] * 7))
    net.add_neuron(iz, 1, *([0.0] * 7))
    net.add_synapse(0, 1, 34, 1.0, stdp)
    if stdp:
        with pytest.raises(NemoError):
            Simulation(net, conf)
    else:
        Simulation(net, conf)


def test_high_firing(lib):
    """src/test/test.cpp:703-735: every neuron forced to fire every cycle."""
    spec = netgen.izhikevich_random(1000, 1000, dmax=20, seed=2)
    _, sim = make_sim(lib, spec)
    everyone = np.arange(1000)
    for _ in range(50):
        assert len(sim.step(fstim=everyone)) == 1000
