"""Pins of the oracle restatement.

1. Each restated neuron-model update is run beside the reference's own CPU
   plugin source (src/nemo/cpu/plugins/<Model>.cpp) compiled unmodified into
   oracle/_ref/lib<Model>.so by oracle/Makefile, on the same seeded inputs for
   many cycles; all outputs must agree bit for bit. Both link the same
   urand/nrand restatement (the reference RNG.cpp needs Boost).
2. The fixed-point and RNG-seeding restatements against values derived from
   their published definitions.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import ORACLE_REF_DIR, ensure_oracle

UPDATE_T = ctypes.CFUNCTYPE(None, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                            ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                            ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)

# (model, nParam, nState, parameter sampler, state sampler, current scale)
MODELS = {
    "Izhikevich": (5, 2),
    "IF_curr_exp": (9, 4),
    "QIF": (1, 1),
    "HH": (0, 5),
    "PoissonSource": (1, 0),
    "Input": (0, 0),
}


def _inputs(model, n, rng):
    f32 = np.float32
    if model == "Izhikevich":
        r = rng.random(n, dtype=f32)
        b = (f32(0.2) + f32(0.05) * r).astype(f32)
        param = np.stack([np.full(n, 0.02, f32), b, (f32(-65) + f32(15) * r * r).astype(f32),
                          np.full(n, 8.0, f32), (rng.random(n, dtype=f32) * f32(6)).astype(f32)])
        param[4, ::5] = 0.0
        v = np.full(n, -65.0, f32)
        state = np.stack([(b * v).astype(f32), v])
        scale = 10.0
    elif model == "IF_curr_exp":
        vals = [-65.0, -65.0, 1.0, 20.0, 2.0, 5.0, 5.0, -50.0, 0.5]
        param = np.stack([np.full(n, x, f32) for x in vals])
        state = np.stack([np.full(n, -65.0, f32), np.zeros(n, f32), np.zeros(n, f32), np.full(n, 3.0, f32)])
        scale = 5.0
    elif model == "QIF":
        param = np.full((1, n), 0.04, f32)
        state = rng.random((1, n), dtype=f32)
        scale = 20.0
    elif model == "HH":
        param = np.zeros((0, n), f32)
        vals = [-65.0, 0.3177, 0.0529, 0.5961, 0.0]
        state = np.stack([np.full(n, x, f32) for x in vals])
        state[0] += rng.normal(0, 3, n).astype(f32)
        scale = 0.5
    elif model == "PoissonSource":
        param = (rng.random((1, n), dtype=f32) * f32(0.1)).astype(f32)
        state = np.zeros((0, n), f32)
        scale = 0.0
    else:
        param = np.zeros((0, n), f32)
        state = np.zeros((0, n), f32)
        scale = 0.0
    return np.ascontiguousarray(param), np.ascontiguousarray(state), scale


class _Run:
    def __init__(self, fn, model, n, seed):
        rng = np.random.default_rng(seed)
        self.fn = fn
        self.n = n
        self.param, self.state, self.scale = _inputs(model, n, rng)
        self.rng = np.ascontiguousarray(rng.integers(1, 2**31, size=(n, 4), dtype=np.uint32))
        self.rf = np.zeros(n, np.uint64)
        self.fired = np.zeros(n, np.uint32)
        self.fstim = np.zeros(n, np.uint32)

    def step(self, cycle, E, I, ext, fstim):
        self.fstim[:] = fstim
        ext = ext.copy()
        p = lambda a: a.ctypes.data if a.size else None
        self.fn(0, self.n, cycle, p(self.param), self.n, p(self.state), self.state.size, self.n,
                20, p(self.fstim), p(self.rng), p(E), p(I), p(ext), p(self.rf), p(self.fired), None)
        return self.fired.copy(), ext


@pytest.mark.parametrize("model", list(MODELS))
def test_restated_update_matches_reference_plugin(model):
    lib_path = os.path.join(ORACLE_REF_DIR, "lib%s.so" % model)
    if not os.path.exists(lib_path):
        pytest.skip("reference plugin sources were not available when oracle/_ref was built")
    ref = UPDATE_T(("cpu_update_neurons", ctypes.CDLL(lib_path)))
    oracle = ctypes.CDLL(ensure_oracle())
    oracle.oracle_model_update.restype = ctypes.c_void_p
    mine = UPDATE_T(oracle.oracle_model_update(model.encode()))

    n = 257
    cycles = 40 if model == "HH" else 300
    a, b = _Run(ref, model, n, 7), _Run(mine, model, n, 7)
    drv = np.random.default_rng(11)
    for cycle in range(cycles):
        E = np.ascontiguousarray((drv.random(n, dtype=np.float32) * np.float32(a.scale)).astype(np.float32))
        I = np.ascontiguousarray((-drv.random(n, dtype=np.float32) * np.float32(a.scale) * np.float32(0.5)).astype(np.float32))
        ext = np.ascontiguousarray(np.where(drv.random(n) < 0.1, np.float32(1.5), np.float32(0)).astype(np.float32))
        fstim = (drv.random(n) < 0.02).astype(np.uint32)
        fa, ea = a.step(cycle, E, I, ext, fstim)
        fb, eb = b.step(cycle, E, I, ext, fstim)
        assert np.array_equal(fa, fb), "cycle %d fired" % cycle
        assert np.array_equal(ea, eb)
        assert np.array_equal(a.state.view(np.uint32), b.state.view(np.uint32)), "cycle %d state" % cycle
        assert np.array_equal(a.rf, b.rf)
        assert np.array_equal(a.rng, b.rng)
    if model in ("Izhikevich", "QIF", "PoissonSource"):
        assert a.rf.any(), "the pin should exercise firing"


def test_rng_seeds_follow_mt19937():
    """src/nemo/RNG.cpp:39-62: seeds are consecutive outputs of a default-
    seeded mt19937 reduced to [0, 2^31) (bucket size 2: mt() >> 1). The first
    outputs of mt19937(5489) are a published known answer (C++11 [rand.predef]
    requires the 10000th to be 4123659995)."""
    from nemo_b200.nemo import Library, Network, Simulation
    from conftest import configuration
    # the 10000th output, via numpy's MT19937 legacy seeding with 5489
    mt = np.random.RandomState(5489)
    vals = mt.randint(0, 2**32, size=10000, dtype=np.uint64)
    assert int(vals[-1]) == 4123659995
    # seeds drive the first urand of neuron 0: a Poisson source with rate 1 fires
    # unless (urand & 0xffff) >= 65536 (never) - so check the xorshift stream
    # through the Izhikevich noise instead: two identically built networks agree
    lib = Library(ensure_oracle())
    net = Network(lib)
    t = net.add_neuron_type("PoissonSource")
    net.add_neuron(t, np.arange(4), np.full(4, 0.5, np.float32))
    sim = Simulation(net, configuration(lib))
    seeds = (vals[:16] >> 1).astype(np.uint32).reshape(4, 4)
    # restated xorshift128 on the seeds; fired iff (urand & 0xffff) < 0.5 * 2^16
    def urand(s):
        t_ = np.uint32(s[0] ^ np.uint32((int(s[0]) << 11) & 0xffffffff))
        s[0], s[1], s[2] = s[1], s[2], s[3]
        s[3] = np.uint32((s[3] ^ (s[3] >> np.uint32(19))) ^ (t_ ^ (t_ >> np.uint32(8))))
        return int(s[3])
    state = [list(map(np.uint32, row)) for row in seeds]
    for _ in range(50):
        expected = [n for n in range(4) if (urand(state[n]) & 0xffff) < 32768]
        assert list(sim.step()) == expected
