"""The network compiler on the device (csrc/compile.cu) against the host
build: the same network built both ways (NEMO_B200_DEVICE_BUILD_MIN forces
the choice) must answer every synapse query alike, fire alike cycle by cycle
and learn the same weights. Both are compared to nothing else: the GPU parity
suite checks the host build against the oracle."""
import numpy as np
import pytest

from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, Network, Simulation

pytestmark = pytest.mark.gpu


def _build(lib, spec, stdp, device, monkeypatch):
    monkeypatch.setenv("NEMO_B200_DEVICE_BUILD_MIN", "0" if device else str(10**15))
    conf = Configuration(lib)
    if stdp:
        pre, post = netgen.standard_stdp()
        conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
    return Simulation(spec.build(Network(lib)), conf)


@pytest.mark.parametrize("stdp", [False, True])
def test_device_build_matches_host_build(monkeypatch, stdp):
    spec = netgen.izhikevich_random(3000, 200, dmax=20, seed=13, stdp=stdp)
    lib = Library()
    dev = _build(lib, spec, stdp, True, monkeypatch)
    host = _build(lib, spec, stdp, False, monkeypatch)
    # queries read the forward matrix through each synapse's position
    for src in range(0, 3000, 37):
        a, b = dev.get_synapses_from(src), host.get_synapses_from(src)
        assert np.array_equal(a, b), src
        for sid in a[::7]:
            assert dev.get_synapse_target(int(sid)) == host.get_synapse_target(int(sid))
            assert dev.get_synapse_delay(int(sid)) == host.get_synapse_delay(int(sid))
            assert dev.get_synapse_weight(int(sid)) == host.get_synapse_weight(int(sid))
    for c in range(300):
        assert np.array_equal(dev.step(), host.step()), c
        if stdp and c % 100 == 99:
            dev.apply_stdp(1.0)
            host.apply_stdp(1.0)
    if stdp:
        # the learned weights, through the reverse matrices the two builds made
        for src in range(0, 2400, 13):
            for sid in dev.get_synapses_from(src):
                assert dev.get_synapse_weight(int(sid)) == host.get_synapse_weight(int(sid)), sid
    for i in range(0, 3000, 29):
        assert np.float32(dev.get_membrane_potential(i)).view(np.uint32) == \
            np.float32(host.get_membrane_potential(i)).view(np.uint32), i


def test_device_build_mixed_delays_and_types(monkeypatch):
    """A mixed-model network with delay-1 synapses and HH neurons (eight
    lanes each, so device indices are not contiguous in user order)."""
    spec = netgen.mixed_plugins(n_iz=800, n_lif=500, n_qif=300, n_hh=40, m=60, dmax=5, seed=17)
    lib = Library()
    dev = _build(lib, spec, False, True, monkeypatch)
    host = _build(lib, spec, False, False, monkeypatch)
    rng = np.random.default_rng(6)
    n = spec.neuron_count
    for c in range(120):
        fstim = np.sort(rng.choice(n, 10, replace=False)).astype(np.uint32)
        assert np.array_equal(dev.step(fstim=fstim), host.step(fstim=fstim)), c
