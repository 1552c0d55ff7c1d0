"""Batches of independent networks in one simulation (nemo_b200_new_batch),
CUDA-graph runs and the block-size autotuner, against each instance's own
oracle simulation: every instance's firing must equal, cycle by cycle, what
the reference CPU backend gives for that network alone."""

import ctypes

import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, Network, NemoError, Simulation

pytestmark = pytest.mark.gpu

P = ctypes.POINTER


def _bind(lib):
    d = lib.dll
    d.nemo_b200_new_batch.restype = ctypes.c_void_p
    d.nemo_b200_new_batch.argtypes = [P(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_void_p]
    d.nemo_b200_batch_instances.argtypes = [ctypes.c_void_p, P(ctypes.c_size_t)]
    d.nemo_b200_batch_fired_at.argtypes = [ctypes.c_void_p, ctypes.c_uint64, P(P(ctypes.c_uint)),
                                           P(P(ctypes.c_size_t))]
    d.nemo_b200_run_graph.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, P(ctypes.c_int)]
    d.nemo_b200_autotune.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint), ctypes.c_double * 3]
    d.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    d.nemo_delete_simulation.argtypes = [ctypes.c_void_p]


class Batch:
    def __init__(self, lib, specs):
        _bind(lib)
        self.lib = lib
        self.nets = [spec.build(Network(lib)) for spec in specs]
        conf = Configuration(lib)
        handles = (ctypes.c_void_p * len(self.nets))(*[n.handle for n in self.nets])
        self.handle = lib.dll.nemo_b200_new_batch(handles, len(self.nets), conf.handle)
        if not self.handle:
            raise NemoError(-1, lib.dll.nemo_strerror().decode())
        self.cycle = 0

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.dll.nemo_delete_simulation(self.handle)

    def fired(self, cycle):
        f = P(ctypes.c_uint)()
        o = P(ctypes.c_size_t)()
        self.lib.call("nemo_b200_batch_fired_at", self.handle, cycle, ctypes.byref(f), ctypes.byref(o))
        n = len(self.nets)
        offs = np.ctypeslib.as_array(o, shape=(n + 1,)).copy()
        total = int(offs[-1])
        arr = np.ctypeslib.as_array(f, shape=(total,)).copy() if total else np.zeros(0, np.uint32)
        return [arr[offs[j]:offs[j + 1]] for j in range(n)]

    def step(self):
        fptr = P(ctypes.c_uint)()
        cnt = ctypes.c_size_t()
        self.lib.call("nemo_step", self.handle, None, 0, None, None, 0, ctypes.byref(fptr), ctypes.byref(cnt))
        self.cycle += 1
        return self.fired(self.cycle - 1)

    def run_graph(self, cycles, per_launch):
        used = ctypes.c_int(-1)
        self.lib.call("nemo_b200_run_graph", self.handle, cycles, per_launch, ctypes.byref(used))
        self.cycle += cycles
        return used.value

    def autotune(self, trial):
        t = ctypes.c_uint()
        ms = (ctypes.c_double * 3)()
        self.lib.call("nemo_b200_autotune", self.handle, trial, ctypes.byref(t), ms)
        self.cycle += 6 * trial
        return t.value, list(ms)


def _specs(sizes, seed0=100):
    rng = np.random.default_rng(seed0)
    specs = []
    for k, n in enumerate(sizes):
        sig = float(rng.uniform(3, 7))
        specs.append(netgen.izhikevich_random(n, 100, dmax=20, seed=seed0 + k, sigma_exc=sig,
                                              sigma_inh=0.4 * sig))
    return specs


def _oracles(specs, oracle_lib):
    sims = []
    for spec in specs:
        net = spec.build(Network(oracle_lib))
        conf = Configuration(oracle_lib)
        conf.set_cpu_backend()
        sims.append((net, Simulation(net, conf)))
    return [s for _, s in sims], [n for n, _ in sims]


def test_batch_matches_each_instance(oracle_lib):
    sizes = [400, 1500, 700, 2300, 900, 333]
    specs = _specs(sizes)
    batch = Batch(Library(), specs)
    count = ctypes.c_size_t()
    batch.lib.call("nemo_b200_batch_instances", batch.handle, ctypes.byref(count))
    assert count.value == len(sizes)
    oracles, _keep = _oracles(specs, oracle_lib)

    def check(cycle):
        got = batch.fired(cycle)
        for j, o in enumerate(oracles):
            ref = o.step()
            assert np.array_equal(got[j], ref), "instance %d cycle %d" % (j, cycle)
        return sum(g.size for g in got)

    fired = 0
    # per-cycle steps through the reference ABI
    for c in range(40):
        batch.step()
        fired += check(c)
    # graph runs of the device-resident loop
    start = batch.cycle
    used = batch.run_graph(200, 50)
    assert used in (0, 1)
    for c in range(start, batch.cycle):
        fired += check(c)
    # replay of the same graph
    start = batch.cycle
    batch.run_graph(200, 50)
    for c in range(start, batch.cycle):
        fired += check(c)
    # the autotuner's trial cycles are ordinary cycles
    start = batch.cycle
    threads, ms = batch.autotune(10)
    assert threads in (256, 512, 1024) and all(x > 0 for x in ms)
    for c in range(start, batch.cycle):
        fired += check(c)
    start = batch.cycle
    batch.run_graph(100, 0)
    for c in range(start, batch.cycle):
        fired += check(c)
    assert fired > 1000


def test_graph_run_single_network(oracle_lib):
    spec = netgen.izhikevich_random(2000, 100, dmax=20, seed=31)
    batch = Batch(Library(), [spec])
    oracles, _keep = _oracles([spec], oracle_lib)
    for rep in range(3):
        start = batch.cycle
        batch.run_graph(150, 40)
        for c in range(start, batch.cycle):
            assert np.array_equal(batch.fired(c)[0], oracles[0].step()), "cycle %d" % c
