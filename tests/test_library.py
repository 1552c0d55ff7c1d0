"""CPU checks of the product library boundary: it loads, exports every entry
point declared in include/*.h, and its host-side network construction and
queries agree with the oracle (no GPU needed for these calls)."""

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from nemo_b200 import netgen
from nemo_b200.nemo import PRODUCT_LIBRARY, Library, NemoError, Network


def _declared_functions():
    names = []
    for h in ("nemo.h", "nemo_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(nemo_\w+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(PRODUCT_LIBRARY), "build with __graft_entry__.build()"
    out = subprocess.check_output(["nm", "-D", "--defined-only", PRODUCT_LIBRARY], text=True)
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    declared = _declared_functions()
    assert len(declared) > 60
    missing = [n for n in declared if n not in exported]
    assert not missing, missing


def test_oracle_exports_the_reference_abi():
    from conftest import ensure_oracle
    out = subprocess.check_output(["nm", "-D", "--defined-only", ensure_oracle()], text=True)
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "nemo.h")).read(), flags=re.S)
    declared = set(re.findall(r"\b(nemo_\w+)\s*\(", text))
    assert not [n for n in declared if n not in exported]


def test_network_construction_matches_oracle(oracle_lib):
    gpu = Library()
    spec = netgen.izhikevich_random(200, 30, dmax=15, seed=9, stdp=True)
    a = spec.build(Network(gpu))
    b = spec.build(Network(oracle_lib))
    assert a.neuron_count() == b.neuron_count() == 200
    for src in (0, 17, 199):
        ia, ib = a.get_synapses_from(src), b.get_synapses_from(src)
        assert list(ia) == list(ib)
        for sid in ia:
            assert a.get_synapse_target(sid) == b.get_synapse_target(sid)
            assert a.get_synapse_delay(sid) == b.get_synapse_delay(sid)
            assert a.get_synapse_weight(sid) == b.get_synapse_weight(sid)
            assert a.get_synapse_plastic(sid) == b.get_synapse_plastic(sid)
    assert a.get_neuron_parameter(5, 2) == b.get_neuron_parameter(5, 2)
    assert a.get_neuron_state(150, 0) == b.get_neuron_state(150, 0)


def test_network_file_round_trip(tmp_path, oracle_lib):
    """A generated network written to one file and read back is the same
    network, and both libraries build identical networks from the file."""
    spec = netgen.mixed_plugins(n_iz=120, n_lif=80, n_qif=40, n_hh=9, m=20, dmax=10, seed=3)
    path = tmp_path / "net.npz"
    spec.save(path)
    back = netgen.NetSpec.load(path)
    assert [p.type_name for p in back.populations] == [p.type_name for p in spec.populations]
    for p, q in zip(spec.populations, back.populations):
        assert np.array_equal(p.idx, q.idx)
        assert all(np.array_equal(np.asarray(a, np.float32), b) for a, b in zip(p.args, q.args))
    for k in ("source", "target", "delay", "weight", "plastic"):
        assert np.array_equal(getattr(spec, k), getattr(back, k))
    a, b = back.build(Network(Library())), back.build(Network(oracle_lib))
    assert a.neuron_count() == b.neuron_count() == spec.neuron_count
    for src in (0, 100, 230):
        ids = a.get_synapses_from(src)
        assert list(ids) == list(b.get_synapses_from(src))
        for sid in ids:
            assert a.get_synapse_weight(sid) == b.get_synapse_weight(sid)
    bad = tmp_path / "other.npz"
    np.savez(bad, x=np.zeros(3))
    with pytest.raises(ValueError):
        netgen.NetSpec.load(bad)


@pytest.mark.parametrize("which", ["b200", "oracle"])
def test_network_errors(which, oracle_lib):
    lib = Library() if which == "b200" else oracle_lib
    net = Network(lib)
    with pytest.raises(NemoError) as e:
        net.add_neuron_type("NoSuchModel")
    assert e.value.status == 6
    iz = net.add_neuron_type("Izhikevich")
    assert net.add_neuron_type("Izhikevich") == iz
    with pytest.raises(NemoError):
        net.add_neuron(iz, 0, 1.0, 2.0)
    with pytest.raises(NemoError):
        net.add_synapse(0, 1, 0, 1.0, False)
    with pytest.raises(NemoError):
        net.get_neuron_state(3, 0)
    assert len(net.get_synapses_from(12345)) == 0
    sid = net.add_synapse(7, 8, 3, 0.5, True)
    assert sid == (7 << 32)
    assert net.add_synapse(7, 9, 3, 0.5, True) == (7 << 32) | 1
    with pytest.raises(NemoError) as e:
        net.get_synapse_target((7 << 32) | 5)
    assert e.value.status == 14  # std::out_of_range in the reference


def test_plugin_descriptors_parse():
    gpu = Library()
    net = Network(gpu)
    for name, nargs in [("Izhikevich", 7), ("IF_curr_exp", 13), ("QIF", 2), ("HH", 5),
                        ("PoissonSource", 1), ("Input", 0)]:
        t = net.add_neuron_type(name)
        net.add_neuron(t, 1000 + t, *([0.0] * nargs))


def test_simulation_without_gpu_fails_loudly():
    """On a machine without a GPU the library reports a CUDA error instead of
    falling back to any CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nemo_b200.nemo import Configuration, Simulation
    gpu = Library()
    net = netgen.ring(64).build(Network(gpu))
    with pytest.raises(NemoError, match="CUDA"):
        Simulation(net, Configuration(gpu))


def test_expf_exception_table_is_small():
    """The host-built table of inputs where glibc expf rounds differently from
    the device candidate: about 1e-4 of the 2.2e9 floats in [-104, 89], all
    close to a rounding boundary."""
    import ctypes
    from nemo_b200.nemo import PRODUCT_LIBRARY
    lib = ctypes.CDLL(PRODUCT_LIBRARY)
    count, tau = ctypes.c_size_t(), ctypes.c_double()
    assert lib.nemo_b200_expf_exceptions(ctypes.byref(count), ctypes.byref(tau)) == 0
    assert 0 < count.value < 2_000_000
    assert 0.0 < tau.value < 0.01


def _build_cpp_check(tmp_path):
    import shutil
    import subprocess
    from nemo_b200.nemo import PRODUCT_LIBRARY
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "cpp_api_check")
    cxx = shutil.which("g++") or "g++"
    libdir = os.path.dirname(PRODUCT_LIBRARY)
    subprocess.check_call([cxx, "-std=c++11", "-Wall", "-I", os.path.join(root, "include"),
                           os.path.join(root, "tests", "cpp_api_check.cpp"), "-L", libdir, "-lnemo_b200",
                           "-Wl,-rpath," + libdir, "-o", exe])
    return exe


def test_cpp_api_without_device(tmp_path):
    """include/nemo.hpp, the reference's C++ classes over the C ABI, compiled
    into a C++ caller: construction, queries, configuration checks, and a
    simulation that fails with a status when there is no device."""
    import subprocess
    exe = _build_cpp_check(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split("\n")[:3] == ["ok construction", "ok configuration", "ok no device"]


@pytest.mark.gpu
def test_cpp_api_simulation(tmp_path):
    """The C++ caller simulates a 64-neuron ring through nemo::simulation():
    neuron k fires at cycle k."""
    import subprocess
    exe = _build_cpp_check(tmp_path)
    r = subprocess.run([exe, "simulate"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok ring" in r.stdout
