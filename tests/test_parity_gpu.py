"""Parity of the B200 library with the oracle on the same seeded networks:
bit-exact firing traces per cycle, bit-exact neuron state (float bits) and
bit-exact fixed-point weights after STDP. Everything here runs the sm_100a
kernels through the C ABI."""

import ctypes

import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, Network, Simulation

pytestmark = pytest.mark.gpu


def _pair(spec, oracle_lib, stdp=None, write_only=False):
    sims = []
    for lib in (Library(), oracle_lib):
        net = spec.build(Network(lib))
        conf = Configuration(lib)
        if stdp is not None:
            pre, post, limits = stdp
            conf.set_stdp_function(pre, post, *limits)
        if write_only:
            conf.set_write_only_synapses()
        if lib is oracle_lib:
            conf.set_cpu_backend()
        sims.append((net, Simulation(net, conf)))
    return sims[0], sims[1]


def _state_bits(sim, spec, var):
    return np.array([np.float32(sim.get_neuron_state(int(i), var)).view(np.uint32)
                     for p in spec.populations for i in p.idx], dtype=np.uint32)


def test_libm_exhaustive(oracle_lib):
    """The device noise path reproduces host glibc sinf/logf on all 83886081
    reachable inputs."""
    lib = Library()
    net = netgen.ring(32).build(Network(lib))
    sim = Simulation(net, Configuration(lib))
    mism = ctypes.c_uint64(99)
    lib.dll.nemo_b200_libm_check.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    lib.call("nemo_b200_libm_check", sim.handle, ctypes.byref(mism))
    assert mism.value == 0


def test_nrand_probe_matches_glibc():
    lib = Library()
    net = netgen.ring(32).build(Network(lib))
    sim = Simulation(net, Configuration(lib))
    rng = np.random.default_rng(0)
    u1 = rng.integers(0, 2**32, 20000, dtype=np.uint64).astype(np.uint32)
    u2 = rng.integers(0, 2**32, 20000, dtype=np.uint64).astype(np.uint32)
    edges = np.array([0, 1, 2**24 - 1, 2**24, 2**24 + 1, 2**31, 2**32 - 129, 2**32 - 128, 2**32 - 1], np.uint32)
    u1 = np.concatenate([u1, edges, edges[::-1]])
    u2 = np.concatenate([u2, edges[::-1], edges])
    out = np.empty(u1.size, np.float32)
    P = ctypes.POINTER
    lib.dll.nemo_b200_nrand_probe.argtypes = [ctypes.c_void_p, P(ctypes.c_uint32), P(ctypes.c_uint32),
                                              P(ctypes.c_float), ctypes.c_size_t]
    lib.call("nemo_b200_nrand_probe", sim.handle, u1.ctypes.data_as(P(ctypes.c_uint32)),
             u2.ctypes.data_as(P(ctypes.c_uint32)), out.ctypes.data_as(P(ctypes.c_float)), u1.size)
    libm = ctypes.CDLL("libm.so.6")
    libm.sinf.restype = libm.logf.restype = libm.sqrtf.restype = ctypes.c_float
    libm.sinf.argtypes = libm.logf.argtypes = libm.sqrtf.argtypes = [ctypes.c_float]
    C = np.float32(1.4629180792671596810513378043098e-9)
    S = np.float32(0.00000000023283064365386962890625)
    for k in range(u1.size):
        a = np.float32(np.float32(u1[k]) * C)
        b = np.float32(np.float32(u2[k]) * S)
        r = np.float32(libm.sqrtf(np.float32(np.float32(-2) * np.float32(libm.logf(np.float32(np.float32(1) - b))))))
        expected = np.float32(np.float32(libm.sinf(a)) * r)
        assert np.float32(out[k]).view(np.uint32) == expected.view(np.uint32) or (np.isnan(out[k]) and np.isnan(expected)), k


@pytest.mark.parametrize("n,m,cycles,seed", [(1000, 100, 1000, 1), (3000, 50, 300, 2)])
def test_izhikevich_random_network(oracle_lib, n, m, cycles, seed):
    """The 1000-neuron benchmark network (thalamic noise sigma 5/2, 100
    synapses per neuron, delays 1..20): identical firing every cycle and
    identical u, v bits at the end."""
    spec = netgen.izhikevich_random(n, m, dmax=20, seed=seed)
    (_, g), (_, o) = _pair(spec, oracle_lib)
    total = 0
    for c in range(cycles):
        a, b = g.step(), o.step()
        assert np.array_equal(a, b), "cycle %d" % c
        total += a.size
    assert total > cycles  # the network is active
    assert np.array_equal(_state_bits(g, spec, 0), _state_bits(o, spec, 0))
    assert np.array_equal(_state_bits(g, spec, 1), _state_bits(o, spec, 1))


def test_stdp_network_weights(oracle_lib):
    """Exponential STDP on excitatory synapses, applyStdp every 100 cycles:
    identical firing and identical fixed-point weights of every synapse."""
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=4, stdp=True)
    pre, post = netgen.standard_stdp()
    (gn, g), (on, o) = _pair(spec, oracle_lib, stdp=(pre, post, (0.0, 1.0, 0.0, -1.0)))
    for epoch in range(4):
        for c in range(100):
            a, b = g.step(), o.step()
            assert np.array_equal(a, b), "epoch %d cycle %d" % (epoch, c)
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
    for src in range(0, 2000, 7):
        for sid in g.get_synapses_from(src):
            assert g.get_synapse_weight(sid) == o.get_synapse_weight(sid)


def test_autotuned_shape_keeps_results(oracle_lib):
    """The autotuner's trials (block sizes x STDP run lengths) are ordinary
    cycles and the shape it keeps changes no result: firing every cycle and
    every weight after applyStdp equal the oracle's, which runs the same
    cycles."""
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=8, stdp=True)
    pre, post = netgen.standard_stdp()
    (gn, g), (on, o) = _pair(spec, oracle_lib, stdp=(pre, post, (0.0, 1.0, 0.0, -1.0)))
    lib = g.lib
    lib.dll.nemo_b200_autotune_shape.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.POINTER(ctypes.c_uint),
                                                 ctypes.POINTER(ctypes.c_uint), ctypes.c_double * 6]
    for c in range(50):
        assert np.array_equal(g.step(), o.step()), c
    threads, run = ctypes.c_uint(), ctypes.c_uint()
    ms = (ctypes.c_double * 6)()
    trial = 10
    lib.call("nemo_b200_autotune_shape", g.handle, trial, ctypes.byref(threads), ctypes.byref(run), ms)
    assert threads.value in (256, 512, 1024) and run.value in (64, 128)
    assert all(x > 0 for x in ms)
    # two rounds over 3 block sizes x 2 run lengths
    first = 50
    for c in range(first, first + 12 * trial):
        assert np.array_equal(g.fired_at(c), o.step()), c
    for epoch in range(2):
        for c in range(100):
            assert np.array_equal(g.step(), o.step()), (epoch, c)
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
    for src in range(0, 2000, 7):
        for sid in g.get_synapses_from(src):
            assert g.get_synapse_weight(sid) == o.get_synapse_weight(sid)


def test_stdp_clamps_out_of_bound_weights(oracle_lib):
    """Excitatory weights up to 0.5 with an STDP bound of 0.3: the first
    applyStdp clamps every plastic weight, those with a zero accumulator
    included (after it, synapses with a zero accumulator are left alone);
    every weight equals the oracle's after each apply."""
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=6, stdp=True)
    pre, post = netgen.standard_stdp()
    (gn, g), (on, o) = _pair(spec, oracle_lib, stdp=(pre, post, (0.0, 0.3, 0.0, -1.0)))
    sources = range(0, 2000, 11)
    for epoch in range(3):
        for c in range(50):
            a, b = g.step(), o.step()
            assert np.array_equal(a, b), "epoch %d cycle %d" % (epoch, c)
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
        clamped = 0
        for src in sources:
            for sid in g.get_synapses_from(src):
                wg = g.get_synapse_weight(sid)
                assert wg == o.get_synapse_weight(sid), (epoch, src, sid)
                clamped += abs(wg - 0.3) < 2e-6   # the bound in Q11.20
        assert clamped > 0


def test_expf_exhaustive():
    """The Hodgkin-Huxley model's device expf reproduces host glibc expf on
    every float in [-104, 89]."""
    lib = Library()
    net = netgen.ring(32).build(Network(lib))
    sim = Simulation(net, Configuration(lib))
    mism = ctypes.c_uint64(99)
    lib.dll.nemo_b200_expf_check.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    lib.call("nemo_b200_expf_check", sim.handle, ctypes.byref(mism))
    assert mism.value == 0


def test_hh_constant_divisions_exhaustive():
    """The Hodgkin-Huxley model divides -(v + 65) by 20, 80 and 18 with an
    FMA-corrected product: equal to correctly rounded division on every float
    of magnitude at least 2^-100 and on the zeros (v + 65 is zero or at least
    2^-17 in magnitude)."""
    lib = Library()
    mism = (ctypes.c_uint64 * 3)(9, 9, 9)
    lib.dll.nemo_b200_hh_division_check.argtypes = [ctypes.c_uint64 * 3]
    lib.call("nemo_b200_hh_division_check", mism)
    assert list(mism) == [0, 0, 0]


def _hh_network(n, m, seed):
    rng = np.random.default_rng(seed)
    f32 = np.float32
    vals = [-65.0, 0.3177, 0.0529, 0.5961, 0.0]
    spec = netgen.NetSpec([netgen.Population("HH", np.arange(n, dtype=np.uint32),
                                             [np.full(n, x, f32) for x in vals])])
    spec.source = np.repeat(np.arange(n, dtype=np.uint32), m)
    spec.target = rng.integers(0, n, n * m, dtype=np.uint32)
    spec.delay = rng.integers(1, 6, n * m, dtype=np.uint32)
    spec.weight = (rng.random(n * m, dtype=f32) * f32(0.3)).astype(f32)
    spec.plastic = np.zeros(n * m, np.uint8)
    return spec


def test_hodgkin_huxley_network(oracle_lib):
    """A network of Hodgkin-Huxley neurons alone (simulation index base 0,
    where the reference plugin is well defined) driven by current stimulus:
    identical firing every cycle and identical v, n, m, h, dir bits. 157
    neurons take eight lanes each: the last warp is partly empty."""
    n = 157
    spec = _hh_network(n, 20, seed=8)
    (_, g), (_, o) = _pair(spec, oracle_lib)
    rng = np.random.default_rng(1)
    total = 0
    for c in range(60):
        ii = np.nonzero(rng.random(n) < 0.3)[0]
        istim = [(int(i), float(rng.uniform(5, 25))) for i in ii]
        a, b = g.step(istim=istim), o.step(istim=istim)
        assert np.array_equal(a, b), "cycle %d" % c
        total += a.size
    assert total > 0
    for var in range(5):
        assert np.array_equal(_state_bits(g, spec, var), _state_bits(o, spec, var)), var


def test_mixed_models_with_stimulus(oracle_lib):
    """Izhikevich, IF_curr_exp, QIF, Hodgkin-Huxley, PoissonSource and Input
    populations with random firing and current stimulus every cycle."""
    f32 = np.float32
    spec = netgen.mixed_plugins(n_iz=700, n_lif=500, n_qif=300, n_hh=60, m=60, dmax=10, seed=5)
    rng = np.random.default_rng(3)
    npois, ninp = 100, 50
    base = spec.neuron_count
    spec.populations.append(netgen.Population("PoissonSource", np.arange(base, base + npois, dtype=np.uint32),
                                              [rng.random(npois, dtype=f32) * f32(0.05)]))
    spec.populations.append(netgen.Population("Input", np.arange(base + npois, base + npois + ninp, dtype=np.uint32), []))
    n = base + npois + ninp
    extra_src = np.arange(base, n, dtype=np.uint32).repeat(20)
    extra_tgt = rng.integers(0, base, extra_src.size, dtype=np.uint32)
    spec.source = np.concatenate([spec.source, extra_src])
    spec.target = np.concatenate([spec.target, extra_tgt])
    spec.delay = np.concatenate([spec.delay, rng.integers(1, 11, extra_src.size, dtype=np.uint32)])
    spec.weight = np.concatenate([spec.weight, rng.random(extra_src.size, dtype=f32) * f32(2)])
    spec.plastic = np.concatenate([spec.plastic, np.zeros(extra_src.size, np.uint8)])
    (_, g), (_, o) = _pair(spec, oracle_lib)
    for c in range(150):
        fstim = np.nonzero(rng.random(n) < 0.01)[0]
        ii = np.nonzero(rng.random(n) < 0.02)[0]
        istim = [(int(i), float(rng.normal(5, 5))) for i in ii]
        a, b = g.step(fstim=fstim, istim=istim), o.step(fstim=fstim, istim=istim)
        assert np.array_equal(a, b), "cycle %d" % c
    for p in spec.populations:
        if p.type_name in ("PoissonSource", "Input"):
            continue
        for i in p.idx[::13]:
            assert np.float32(g.get_membrane_potential(int(i))).view(np.uint32) == \
                np.float32(o.get_membrane_potential(int(i))).view(np.uint32)


def test_device_resident_run_matches_steps(oracle_lib):
    """nemo_b200_run (one persistent launch of many cycles) gives the same
    trace as stepping the oracle cycle by cycle."""
    spec = netgen.izhikevich_random(1500, 100, dmax=20, seed=6, stdp=True)
    pre, post = netgen.standard_stdp()
    (_, g), (_, o) = _pair(spec, oracle_lib, stdp=(pre, post, (0.0, 1.0, 0.0, -1.0)))
    lib = g.lib
    P = ctypes.POINTER
    lib.dll.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    lib.dll.nemo_b200_fired_at.argtypes = [ctypes.c_void_p, ctypes.c_uint64, P(P(ctypes.c_uint)), P(ctypes.c_size_t)]
    # a few ordinary steps first, then graph runs of two different lengths
    for _ in range(7):
        assert np.array_equal(g.step(), o.step())
    cycle = 7
    for chunk in (100, 250, 100):
        counts = np.zeros(chunk, np.uint32)
        events = np.zeros(chunk, np.uint64)
        lib.call("nemo_b200_run", g.handle, chunk, counts.ctypes.data_as(P(ctypes.c_uint32)),
                 events.ctypes.data_as(P(ctypes.c_uint64)))
        outdeg = spec.out_degree()
        for k in range(chunk):
            ref = o.step()
            ptr = P(ctypes.c_uint)()
            cnt = ctypes.c_size_t()
            lib.call("nemo_b200_fired_at", g.handle, cycle + k, ctypes.byref(ptr), ctypes.byref(cnt))
            got = np.ctypeslib.as_array(ptr, shape=(cnt.value,)).copy() if cnt.value else np.zeros(0, np.uint32)
            assert np.array_equal(got, ref), "cycle %d" % (cycle + k)
            assert counts[k] == ref.size
            assert events[k] == int(outdeg[ref].sum())
        cycle += chunk
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
    assert np.array_equal(g.step(), o.step())


@pytest.mark.parametrize("dmax", [1, 5, 20])
def test_every_event_delivered_once(dmax):
    """The kernel's own counters: over a device-resident run every synaptic
    event (fired neuron x out-degree) is added into a current exactly once,
    through the delay-1 inbox or the gather, for delays including 1."""
    spec = netgen.izhikevich_random(3000, 200, dmax=dmax, seed=12, stdp=True)
    lib = Library()
    net = spec.build(Network(lib))
    conf = Configuration(lib)
    pre, post = netgen.standard_stdp()
    conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
    sim = Simulation(net, conf)
    out = (ctypes.c_double * 4)()
    lib.dll.nemo_b200_timed_steps.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_double * 4]
    lib.call("nemo_b200_timed_steps", sim.handle, 3, 100, 1, ctypes.c_float(1.0), out)
    fired, events, delivered = out[1], out[2], out[3]
    assert fired > 0
    assert delivered == events


def test_steps_runs_and_applies_interleaved(oracle_lib):
    """One-phase nemo_step calls (each leaves its cycle's gathering for the
    next call), with short stimulus carried in the kernel parameters --
    current stimulus on Hodgkin-Huxley neurons included -- interleaved with
    device-resident runs, allocation-free steps and applyStdp, which flush
    the pending gathering first: firing and weights identical to the
    oracle's every cycle."""
    f32 = np.float32
    spec = netgen.mixed_plugins(n_iz=600, n_lif=300, n_qif=200, n_hh=40, m=50, dmax=12, seed=11)
    spec.plastic = (spec.source < 480).astype(np.uint8)   # excitatory Izhikevich sources
    n = spec.neuron_count
    pre, post = netgen.standard_stdp()
    (_, g), (_, o) = _pair(spec, oracle_lib, stdp=(pre, post, (0.0, 1.0, 0.0, -1.0)))
    lib = g.lib
    P = ctypes.POINTER
    lib.dll.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    lib.dll.nemo_b200_fired_at.argtypes = [ctypes.c_void_p, ctypes.c_uint64, P(P(ctypes.c_uint)), P(ctypes.c_size_t)]
    lib.dll.nemo_b200_step_noalloc.argtypes = [ctypes.c_void_p, P(ctypes.c_uint), ctypes.c_size_t, P(ctypes.c_uint),
                                               P(ctypes.c_float), ctypes.c_size_t, P(ctypes.c_uint), ctypes.c_size_t,
                                               P(ctypes.c_size_t)]
    rng = np.random.default_rng(7)
    hh = spec.populations[-1].idx
    cycle = 0

    def stimulus():
        fstim = np.sort(rng.choice(n, size=int(rng.integers(0, 8)), replace=False)).astype(np.uint32)
        ii = np.concatenate([rng.choice(hh, size=4, replace=False), rng.choice(n, size=6, replace=False)])
        return fstim, [(int(i), float(rng.uniform(5, 30))) for i in np.unique(ii)]

    out = np.zeros(n, np.uint32)
    cnt = ctypes.c_size_t()
    for rnd in range(3):
        for _ in range(40):
            fstim, istim = stimulus()
            assert np.array_equal(g.step(fstim=fstim, istim=istim), o.step(fstim=fstim, istim=istim)), cycle
            cycle += 1
        for _ in range(10):
            fstim, istim = stimulus()
            inidx = np.array([p[0] for p in istim], np.uint32)
            icur = np.array([p[1] for p in istim], np.float32)
            lib.call("nemo_b200_step_noalloc", g.handle, fstim.ctypes.data_as(P(ctypes.c_uint)), fstim.size,
                     inidx.ctypes.data_as(P(ctypes.c_uint)), icur.ctypes.data_as(P(ctypes.c_float)), inidx.size,
                     out.ctypes.data_as(P(ctypes.c_uint)), out.size, ctypes.byref(cnt))
            assert np.array_equal(out[:cnt.value], o.step(fstim=fstim, istim=istim)), cycle
            cycle += 1
        chunk = 30
        lib.call("nemo_b200_run", g.handle, chunk, None, None)
        for k in range(chunk):
            ref = o.step()
            ptr = P(ctypes.c_uint)()
            c2 = ctypes.c_size_t()
            lib.call("nemo_b200_fired_at", g.handle, cycle + k, ctypes.byref(ptr), ctypes.byref(c2))
            got = np.ctypeslib.as_array(ptr, shape=(c2.value,)).copy() if c2.value else np.zeros(0, np.uint32)
            assert np.array_equal(got, ref), cycle + k
        cycle += chunk
        g.apply_stdp(1.0)
        o.apply_stdp(1.0)
    for src in range(0, 480, 9):
        for sid in g.get_synapses_from(src):
            assert g.get_synapse_weight(sid) == o.get_synapse_weight(sid), (src, sid)
