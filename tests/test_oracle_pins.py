"""Pins of the oracle restatement.

1. Each restated neuron-model update is run beside the reference's own CPU
   plugin source (src/nemo/cpu/plugins/<Model>.cpp) compiled unmodified into
   oracle/_ref/lib<Model>.so by oracle/Makefile, on the same seeded inputs for
   many cycles; all outputs must agree bit for bit. Both link the same
   urand/nrand restatement (the reference RNG.cpp needs Boost).
2. The same runs against tests/golden/plugins.npz, which
   tests/golden/make_golden.py wrote from those compiled reference plugins, so
   the pin holds where the reference sources are absent.
3. The fixed-point conversions (fx_toFix, fx_toFloat, wfx_toFloat, fx_mul)
   and the STDP process (potentiation/depression bits, weightChange,
   updatedWeight) against the reference's own src/nemo/{fixedpoint,
   StdpFunction,StdpProcess}.cpp compiled into oracle/_ref/libnemo_stdp_ref.so,
   and against tests/golden/stdp_fixedpoint.npz written from that build.
4. The RNG-seeding restatement against values derived from its published
   definition.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import ORACLE_REF_DIR, ROOT, ensure_oracle
from plugin_harness import MODELS, PIN_N, UPDATE_T, _Run, drive_inputs, pin_cycles, pin_outputs, run_digest

GOLDEN = os.path.join(ROOT, "tests", "golden", "plugins.npz")


def _oracle_update(model):
    oracle = ctypes.CDLL(ensure_oracle())
    oracle.oracle_model_update.restype = ctypes.c_void_p
    return UPDATE_T(oracle.oracle_model_update(model.encode()))


@pytest.mark.parametrize("model", list(MODELS))
def test_restated_update_matches_reference_plugin(model):
    lib_path = os.path.join(ORACLE_REF_DIR, "lib%s.so" % model)
    if not os.path.exists(lib_path):
        pytest.skip("reference plugin sources were not available when oracle/_ref was built")
    ref = UPDATE_T(("cpu_update_neurons", ctypes.CDLL(lib_path)))
    mine = _oracle_update(model)

    n = PIN_N
    a, b = _Run(ref, model, n, 7), _Run(mine, model, n, 7)
    inputs = drive_inputs(n, a.scale)
    for cycle in range(pin_cycles(model)):
        E, I, ext, fstim = next(inputs)
        fa, ea = a.step(cycle, E, I, ext, fstim)
        fb, eb = b.step(cycle, E, I, ext, fstim)
        assert np.array_equal(fa, fb), "cycle %d fired" % cycle
        assert np.array_equal(ea, eb)
        assert np.array_equal(a.state.view(np.uint32), b.state.view(np.uint32)), "cycle %d state" % cycle
        assert np.array_equal(a.rf, b.rf)
        assert np.array_equal(a.rng, b.rng)
    if model in ("Izhikevich", "QIF", "PoissonSource"):
        assert a.rf.any(), "the pin should exercise firing"


@pytest.mark.parametrize("model", list(MODELS))
def test_restated_update_matches_golden_vectors(model):
    """The oracle against the reference plugins' recorded outputs."""
    g = np.load(GOLDEN)
    fired, crcs, state, rf, rng = run_digest(_oracle_update(model), model)
    assert np.array_equal(fired, g[model + "/fired"])
    bad = np.nonzero(crcs != g[model + "/crc"])[0]
    assert bad.size == 0, "first differing cycle %d" % (bad[0] if bad.size else -1)
    assert np.array_equal(state.view(np.uint32), g[model + "/state"].view(np.uint32))
    assert np.array_equal(rf, g[model + "/rf"])
    assert np.array_equal(rng, g[model + "/rng"])


def _compare_pins(mine, theirs):
    assert set(mine) == set(theirs)
    for key in sorted(mine):
        bad = np.nonzero(np.asarray(mine[key]) != np.asarray(theirs[key]))[0]
        assert bad.size == 0, "%s: %d of %d differ (first at %d)" % (key, bad.size, np.asarray(mine[key]).size, bad[0])


def test_fixed_point_and_stdp_match_reference_sources():
    path = os.path.join(ORACLE_REF_DIR, "libnemo_stdp_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference sources were not available when oracle/_ref was built")
    ours = pin_outputs(ctypes.CDLL(ensure_oracle()))
    _compare_pins(ours, pin_outputs(ctypes.CDLL(path)))
    # the inputs reach every branch: overflow, saturation, both windows
    assert any(ours[k].any() for k in ours if k.startswith("to_fix_threw"))
    assert any(np.any(ours[k] != 0) for k in ours if k.startswith("weight_change"))


def test_fixed_point_and_stdp_match_golden_vectors():
    g = np.load(os.path.join(ROOT, "tests", "golden", "stdp_fixedpoint.npz"))
    _compare_pins(pin_outputs(ctypes.CDLL(ensure_oracle())), {k: g[k] for k in g.files})


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
