"""nemo_b200_step_noalloc against nemo_step.

Two simulations are built from the same seeded network; one is stepped with
nemo_step, the other with the allocation-free entry point, on identical
stimulus (firing stimulus, current stimulus with repeated indices). Fired
lists must agree on every call, starting with two calls in a row, and so must
the membrane potentials afterwards. Size limits and an invalid index are
checked against their documented errors. This file is collected last so that
it also runs after the rest of the suite has used the device."""

import ctypes

import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, NemoError, Network, Simulation

pytestmark = pytest.mark.gpu

NEMO_INVALID_INPUT = 6
STIM_MAX = 16384

U32P = ctypes.POINTER(ctypes.c_uint)
F32P = ctypes.POINTER(ctypes.c_float)


def _bind(lib):
    fn = lib.dll.nemo_b200_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, U32P, ctypes.c_size_t, U32P, F32P, ctypes.c_size_t,
                   U32P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    return fn


def _sims(n=3000, m=100, seed=5):
    lib = Library()
    spec = netgen.izhikevich_random(n, m, dmax=20, seed=seed, stdp=True)
    pre, post = netgen.standard_stdp()
    sims = []
    for _ in range(2):
        net = spec.build(Network(lib))
        conf = Configuration(lib)
        conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
        sims.append(Simulation(net, conf))
    return lib, spec, sims[0], sims[1]


class NoAlloc:
    def __init__(self, lib, sim, n):
        self.fn = _bind(lib)
        self.lib = lib
        self.sim = sim
        self.out = np.zeros(n, np.uint32)
        self.count = ctypes.c_size_t()

    def status(self, fstim=(), istim=(), capacity=None):
        f = np.ascontiguousarray(np.asarray(fstim, np.uint32))
        idx = np.ascontiguousarray(np.asarray([p[0] for p in istim], np.uint32))
        cur = np.ascontiguousarray(np.asarray([p[1] for p in istim], np.float32))
        cap = self.out.size if capacity is None else capacity
        return self.fn(self.sim.handle, f.ctypes.data_as(U32P), f.size, idx.ctypes.data_as(U32P),
                       cur.ctypes.data_as(F32P), idx.size, self.out.ctypes.data_as(U32P), cap,
                       ctypes.byref(self.count))

    def step(self, fstim=(), istim=()):
        st = self.status(fstim, istim)
        if st != 0:
            raise NemoError(st, self.lib.dll.nemo_strerror().decode())
        return self.out[:self.count.value].copy()


def _stimulus(rng, n):
    fstim = rng.choice(n, size=int(rng.integers(0, 40)), replace=False).astype(np.uint32)
    k = int(rng.integers(0, 60))
    idx = rng.integers(0, n, size=k)
    if k > 4:
        idx[-1] = idx[0]   # repeated neuron: the last entry wins
        idx[-2] = idx[1]
    cur = rng.uniform(0.0, 25.0, size=k).astype(np.float32)
    return fstim, list(zip(idx.tolist(), cur.tolist()))


def _potentials(sim, n):
    return np.array([np.float32(sim.get_membrane_potential(i)).view(np.uint32) for i in range(n)])


def test_noalloc_step_matches_nemo_step():
    lib, spec, ref, sut = _sims()
    n = spec.neuron_count
    na = NoAlloc(lib, sut, n)
    rng = np.random.default_rng(17)
    # two calls in a row with the same stimulus
    fstim, istim = _stimulus(rng, n)
    for _ in range(2):
        a = ref.step(fstim, istim)
        b = na.step(fstim, istim)
        assert np.array_equal(a, b)
    fired = 0
    for cycle in range(150):
        fstim, istim = _stimulus(rng, n)
        if cycle % 3 == 0:
            fstim, istim = (), ()
        a = ref.step(fstim, istim)
        b = na.step(fstim, istim)
        assert np.array_equal(a, b), "cycle %d" % cycle
        fired += a.size
        if cycle % 50 == 49:
            ref.apply_stdp(1.0)
            sut.apply_stdp(1.0)
    assert fired > 0
    assert np.array_equal(_potentials(ref, n), _potentials(sut, n))


def test_noalloc_limits_and_errors():
    lib, spec, ref, sut = _sims(n=1000, m=50, seed=9)
    n = spec.neuron_count
    na = NoAlloc(lib, sut, n)
    # beyond the scratch size: rejected before anything runs
    big = np.arange(STIM_MAX + 1, dtype=np.uint32) % n
    assert na.status(fstim=big) == NEMO_INVALID_INPUT
    assert "16384" in lib.dll.nemo_strerror().decode()
    assert na.status(istim=[(0, 1.0)] * (STIM_MAX + 1)) == NEMO_INVALID_INPUT
    # a fired array smaller than the network: rejected before anything runs
    assert na.status(capacity=n - 1) == NEMO_INVALID_INPUT
    # the limit itself is accepted
    full = np.arange(STIM_MAX, dtype=np.uint32) % n
    a = ref.step(full, [(int(i), 2.0) for i in full[:STIM_MAX]])
    b = na.step(full, [(int(i), 2.0) for i in full[:STIM_MAX]])
    assert np.array_equal(a, b) and a.size == n
    # an invalid index: the entries before it apply, then the error
    bad = [3, 7, n + 100]
    with pytest.raises(NemoError):
        ref.step(bad)
    assert na.status(fstim=bad) == NEMO_INVALID_INPUT
    for _ in range(30):
        assert np.array_equal(ref.step(), na.step())


def test_noalloc_with_plugin_model():
    """A network with a GPU plugin population (tests/plugins/QIFPlugin): the
    allocation-free step runs the plugin's update like nemo_step does."""
    import copy
    import os
    from nemo_b200 import build as nb_build
    plugin_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "plugins")
    nb_build.build_plugin(os.path.join(plugin_dir, "QIFPlugin.cu"))
    lib = Library()
    lib.add_plugin_path(plugin_dir)
    spec = netgen.mixed_plugins(n_iz=400, n_lif=0, n_qif=300, n_hh=0, m=40, dmax=8, seed=3)
    spec = copy.deepcopy(spec)
    for p in spec.populations:
        if p.type_name == "QIF":
            p.type_name = "QIFPlugin"
    a = Simulation(spec.build(Network(lib)), Configuration(lib))
    b = Simulation(spec.build(Network(lib)), Configuration(lib))
    n = spec.neuron_count
    na = NoAlloc(lib, b, n)
    rng = np.random.default_rng(8)
    for c in range(60):
        fstim = np.sort(rng.choice(n, 5, replace=False)).astype(np.uint32)
        istim = [(int(i), float(rng.normal(40, 20))) for i in rng.choice(n, 30, replace=False)]
        assert np.array_equal(a.step(fstim=fstim, istim=istim), na.step(fstim=fstim, istim=istim)), c
    for i in range(400, 700, 7):
        assert np.float32(a.get_membrane_potential(i)).view(np.uint32) == \
            np.float32(b.get_membrane_potential(i)).view(np.uint32), i


def test_noalloc_step_allocates_nothing():
    """The promise itself: once a first call at the size limit has set up
    the scratch, further calls (at the limit, short, empty) leave the
    device's free memory unchanged -- the entry point grows no staging buffer
    and allocates nothing else."""
    import torch
    torch.cuda.mem_get_info()   # torch's own context set-up happens before the count
    lib, spec, ref, sut = _sims(n=2000, m=50, seed=11)
    n = spec.neuron_count
    na = NoAlloc(lib, sut, n)
    full = np.arange(STIM_MAX, dtype=np.uint32) % n
    istim = [(int(i), 1.5) for i in full]
    na.step(full, istim)
    na.step()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(4):
        na.step(full[k:], istim[:STIM_MAX - 3 * k])
        na.step()
        na.step(full[:10], istim[:7])
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
