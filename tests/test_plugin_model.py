"""Neuron models supplied as GPU plugins (include/nemo_b200_plugin.h): a
model whose name is not built in is loaded from <dir>/b200/lib<Name>.so
beside <Name>.ini, as the reference loads lib<Name>.so from <dir>/{cpu,cuda}/
(src/nemo/NeuronType.cpp:48-73). tests/plugins/QIFPlugin.cu restates the
QIF update as a user's plugin; a network using it must fire and evolve
exactly as the oracle's network with the built-in QIF."""
import copy
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from nemo_b200 import build as nb_build
from nemo_b200 import netgen
from nemo_b200.nemo import Configuration, Library, NemoError, Network, Simulation

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN_DIR = os.path.join(ROOT, "tests", "plugins")

NEMO_CUDA_INVOCATION_ERROR = 1
NEMO_CUDA_ERROR = 4
NEMO_API_UNSUPPORTED = 5
NEMO_INVALID_INPUT = 6
NEMO_DL_ERROR = 12


def build_test_plugins():
    src = os.path.join(PLUGIN_DIR, "QIFPlugin.cu")
    nb_build.build_plugin(src)
    nb_build.build_plugin(src, name="QIFPluginInit", extra_flags=["-DQIF_PLUGIN_INIT"])
    nb_build.build_plugin(os.path.join(PLUGIN_DIR, "LIFPlugin.cu"))
    nb_build.build_plugin(os.path.join(PLUGIN_DIR, "IzhikevichRS.cu"))


@pytest.fixture(scope="module")
def plugin_lib():
    build_test_plugins()
    lib = Library()
    lib.add_plugin_path(PLUGIN_DIR)
    return lib


def _spec(n_iz=700, n_qif=300, m=60, seed=4, stdp=False):
    """Izhikevich and QIF populations, m synapses per neuron; with stdp the
    excitatory Izhikevich sources' synapses are plastic."""
    spec = netgen.mixed_plugins(n_iz=n_iz, n_lif=0, n_qif=n_qif, n_hh=0, m=m, dmax=8, seed=seed)
    if stdp:
        n_exc = int(n_iz * 0.8)
        spec.plastic = (spec.source < n_exc).astype(np.uint8)
    return spec


def _as_plugin(spec, name="QIFPlugin"):
    s = copy.deepcopy(spec)
    for p in s.populations:
        if p.type_name == "QIF":
            p.type_name = name
    return s


def test_plugin_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "use.c"
    src.write_text('#include <nemo_b200_plugin.h>\n'
                   'static b200_update_neurons_t* f;\n'
                   'int main(void) { b200_neuron_batch b; b.count = 0; (void) b; (void) f; return 0; }\n')
    for compiler, flags in (("gcc", ["-std=c99"]), ("g++", ["-std=c++11", "-x", "c++"])):
        exe = shutil.which(compiler)
        if exe is None:
            pytest.skip("%s not found" % compiler)
        subprocess.check_call([exe] + flags + ["-Wall", "-Werror", "-fsyntax-only", "-I",
                                               os.path.join(ROOT, "include"), str(src)])


def test_plugin_exports_update(plugin_lib):
    so = ctypes.CDLL(os.path.join(PLUGIN_DIR, "b200", "libQIFPlugin.so"))
    assert hasattr(so, "b200_update_neurons")


def _simulation_status(lib, type_name, plugin_path=None):
    if plugin_path:
        lib.add_plugin_path(plugin_path)
    net = Network(lib)
    t = net.add_neuron_type(type_name)
    net.add_neuron(t, 0, 0.04, 0.0)   # parameter a, state v (QIFPlugin.ini)
    try:
        Simulation(net, Configuration(lib))
    except NemoError as e:
        return e.status, str(e)
    return 0, ""


def test_unknown_model_without_plugin_is_unsupported(tmp_path):
    """A model with a descriptor but neither a built-in kernel nor a plugin
    library: the simulation is refused before any device work."""
    (tmp_path / "NoKernel.ini").write_text(open(os.path.join(PLUGIN_DIR, "QIFPlugin.ini")).read())
    status, msg = _simulation_status(Library(), "NoKernel", str(tmp_path))
    assert status == NEMO_API_UNSUPPORTED, msg
    assert "b200/libNoKernel.so" in msg


def test_plugin_without_update_symbol_is_rejected(tmp_path):
    """A plugin library that does not export b200_update_neurons."""
    (tmp_path / "NoUpdate.ini").write_text(open(os.path.join(PLUGIN_DIR, "QIFPlugin.ini")).read())
    (tmp_path / "b200").mkdir()
    src = tmp_path / "noupdate.c"
    src.write_text("int b200_something_else(void) { return 0; }\n")
    subprocess.check_call(["gcc", "-shared", "-fPIC", "-o", str(tmp_path / "b200" / "libNoUpdate.so"), str(src)])
    status, msg = _simulation_status(Library(), "NoUpdate", str(tmp_path))
    assert status == NEMO_INVALID_INPUT, msg
    assert "b200_update_neurons" in msg


@pytest.mark.parametrize("version", [None, 0, 99])
def test_plugin_of_another_abi_version_is_rejected(tmp_path, version):
    """A plugin library whose b200_plugin_abi_version is missing (built
    against an older header) or differs from the library's: refused with
    NEMO_DL_ERROR before anything runs, so that no kernel reads the batch
    with wrong field offsets."""
    name = "Abi%s" % ("None" if version is None else version)
    (tmp_path / ("%s.ini" % name)).write_text(open(os.path.join(PLUGIN_DIR, "QIFPlugin.ini")).read())
    (tmp_path / "b200").mkdir()
    src = tmp_path / "abi.c"
    body = "int b200_update_neurons(const void* b, void* s) { return 0; }\n"
    if version is not None:
        body += "const unsigned b200_plugin_abi_version = %du;\n" % version
    src.write_text(body)
    subprocess.check_call(["gcc", "-shared", "-fPIC", "-o", str(tmp_path / "b200" / ("lib%s.so" % name)), str(src)])
    status, msg = _simulation_status(Library(), name, str(tmp_path))
    assert status == NEMO_DL_ERROR, msg
    assert "ABI version" in msg


def test_plugin_built_from_the_header_carries_its_abi_version(plugin_lib):
    so = ctypes.CDLL(os.path.join(PLUGIN_DIR, "b200", "libQIFPlugin.so"))
    assert ctypes.c_uint.in_dll(so, "b200_plugin_abi_version").value == 1


def test_plugin_that_cannot_load_is_a_dl_error(tmp_path):
    (tmp_path / "Broken.ini").write_text(open(os.path.join(PLUGIN_DIR, "QIFPlugin.ini")).read())
    (tmp_path / "b200").mkdir()
    (tmp_path / "b200" / "libBroken.so").write_bytes(b"not an ELF file")
    status, msg = _simulation_status(Library(), "Broken", str(tmp_path))
    assert status == NEMO_DL_ERROR, msg


@pytest.mark.gpu
def test_plugin_model_matches_builtin(plugin_lib, oracle_lib):
    """Izhikevich + plugin QIF on the B200 against Izhikevich + built-in QIF
    on the oracle: identical firing every cycle (firing and current stimulus
    on both populations), identical v bits of every QIF neuron, STDP applied
    every 50 cycles."""
    spec = _spec(stdp=True)
    pspec = _as_plugin(spec)
    pre, post = netgen.standard_stdp()
    sims = []
    for lib, s in ((plugin_lib, pspec), (oracle_lib, spec)):
        net = s.build(Network(lib))
        conf = Configuration(lib)
        conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
        if lib is oracle_lib:
            conf.set_cpu_backend()
        sims.append((net, Simulation(net, conf)))
    (_, g), (_, o) = sims
    n = spec.neuron_count
    qif = [p for p in spec.populations if p.type_name == "QIF"][0].idx
    rng = np.random.default_rng(11)
    fired_qif = 0
    for c in range(200):
        fstim = np.sort(rng.choice(n, 8, replace=False)).astype(np.uint32)
        ii = rng.choice(n, 40, replace=False)
        istim = [(int(i), float(rng.normal(40, 20))) for i in ii]
        a, b = g.step(fstim=fstim, istim=istim), o.step(fstim=fstim, istim=istim)
        assert np.array_equal(a, b), "cycle %d" % c
        fired_qif += int(np.isin(a, qif).sum())
        if c % 50 == 49:
            g.apply_stdp(1.0)
            o.apply_stdp(1.0)
    assert fired_qif > 100
    for i in qif:
        assert np.float32(g.get_membrane_potential(int(i))).view(np.uint32) == \
            np.float32(o.get_membrane_potential(int(i))).view(np.uint32), i


@pytest.mark.gpu
def test_plugin_model_refuses_persistent_multi_cycle_calls(plugin_lib):
    """Plugin updates run between the kernel's cycles: the calls that need
    one persistent launch over many cycles (timed steps, graph runs) refuse
    such a network with NEMO_API_UNSUPPORTED, and the simulation goes on."""
    net = _as_plugin(_spec(n_iz=64, n_qif=64, m=8)).build(Network(plugin_lib))
    sim = Simulation(net, Configuration(plugin_lib))
    sim.step()
    plugin_lib.dll.nemo_b200_timed_steps.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                                     ctypes.c_float, ctypes.c_double * 4]
    out = (ctypes.c_double * 4)()
    with pytest.raises(NemoError) as e:
        plugin_lib.call("nemo_b200_timed_steps", sim.handle, 1, 10, 0, ctypes.c_float(0), out)
    assert e.value.status == NEMO_API_UNSUPPORTED
    sim.step()


@pytest.mark.gpu
def test_plugin_model_device_resident_run(plugin_lib):
    """nemo_b200_run on a network with plugin models (the cycles queued
    without host synchronisation) fires exactly as nemo_step cycle by cycle
    on a second copy: per-cycle counts, fired lists and final potentials."""
    spec = _as_plugin(_spec(n_iz=600, n_qif=300, m=50, seed=21))
    iz = [p for p in spec.populations if p.type_name == "Izhikevich"][0]
    iz.args[4] = np.full(iz.idx.size, 5.0, np.float32)   # thalamic noise: firing every cycle
    a = Simulation(spec.build(Network(plugin_lib)), Configuration(plugin_lib))
    b = Simulation(spec.build(Network(plugin_lib)), Configuration(plugin_lib))
    P = ctypes.POINTER
    dll = plugin_lib.dll
    dll.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    dll.nemo_b200_fired_at.argtypes = [ctypes.c_void_p, ctypes.c_uint64, P(P(ctypes.c_uint)), P(ctypes.c_size_t)]
    n = spec.neuron_count
    rng = np.random.default_rng(4)
    cycle = 0
    for chunk in (50, 120):
        # a stimulated cycle before each run, so that there is activity
        fstim = np.sort(rng.choice(n, 200, replace=False)).astype(np.uint32)
        assert np.array_equal(a.step(fstim=fstim), b.step(fstim=fstim))
        cycle += 1
        counts = np.zeros(chunk, np.uint32)
        plugin_lib.call("nemo_b200_run", a.handle, chunk, counts.ctypes.data_as(P(ctypes.c_uint32)), None)
        for k in range(chunk):
            expected = b.step()
            assert counts[k] == expected.size, (chunk, k)
            ptr, cnt = P(ctypes.c_uint)(), ctypes.c_size_t()
            plugin_lib.call("nemo_b200_fired_at", a.handle, cycle + k, ctypes.byref(ptr), ctypes.byref(cnt))
            got = np.ctypeslib.as_array(ptr, (cnt.value,)).copy() if cnt.value else np.zeros(0, np.uint32)
            assert np.array_equal(got, expected), (chunk, k)
        cycle += chunk
        assert counts.sum() > chunk, counts.sum()
    for i in range(0, n, 11):
        assert np.float32(a.get_membrane_potential(i)).view(np.uint32) == \
            np.float32(b.get_membrane_potential(i)).view(np.uint32), i


@pytest.mark.gpu
def test_plugin_init_sets_initial_state(plugin_lib, oracle_lib):
    """b200_init_neurons runs once when the simulation is created: the
    QIFPluginInit population starts from v = 5 a whatever state it was given,
    and then fires like built-in QIF neurons that were given v = 5 a."""
    spec = _spec(n_iz=500, n_qif=200, m=40, seed=9)
    pspec = _as_plugin(spec, "QIFPluginInit")
    q = [p for p in spec.populations if p.type_name == "QIF"][0]
    q.args[1] = (np.asarray(q.args[0], np.float32) * np.float32(5)).astype(np.float32)
    g = Simulation(pspec.build(Network(plugin_lib)), Configuration(plugin_lib))
    conf = Configuration(oracle_lib)
    conf.set_cpu_backend()
    o = Simulation(spec.build(Network(oracle_lib)), conf)
    v0 = np.float32(0.04) * np.float32(5)
    for i in q.idx[::17]:
        assert np.float32(g.get_membrane_potential(int(i))).view(np.uint32) == v0.view(np.uint32), i
    rng = np.random.default_rng(2)
    n = spec.neuron_count
    for c in range(100):
        istim = [(int(i), float(rng.normal(40, 20))) for i in rng.choice(n, 30, replace=False)]
        assert np.array_equal(g.step(istim=istim), o.step(istim=istim)), "cycle %d" % c
    for i in q.idx:
        assert np.float32(g.get_membrane_potential(int(i))).view(np.uint32) == \
            np.float32(o.get_membrane_potential(int(i))).view(np.uint32), i


@pytest.mark.gpu
def test_two_plugin_models_with_strided_state(plugin_lib, oracle_lib):
    """Two plugin populations in one network, LIFPlugin (nine parameters,
    four state variables through the batch's strides) and QIFPlugin, beside
    Izhikevich: identical firing to the oracle's IF_curr_exp and QIF every
    cycle, and identical bits of every state variable afterwards."""
    spec = netgen.mixed_plugins(n_iz=600, n_lif=400, n_qif=200, n_hh=0, m=50, dmax=6, seed=12)
    pspec = copy.deepcopy(spec)
    names = {"IF_curr_exp": "LIFPlugin", "QIF": "QIFPlugin"}
    for p in pspec.populations:
        p.type_name = names.get(p.type_name, p.type_name)
    g = Simulation(pspec.build(Network(plugin_lib)), Configuration(plugin_lib))
    conf = Configuration(oracle_lib)
    conf.set_cpu_backend()
    o = Simulation(spec.build(Network(oracle_lib)), conf)
    n = spec.neuron_count
    rng = np.random.default_rng(5)
    fired = {k: 0 for k in names}
    for c in range(150):
        fstim = np.sort(rng.choice(n, 6, replace=False)).astype(np.uint32)
        istim = [(int(i), float(rng.normal(30, 15))) for i in rng.choice(n, 40, replace=False)]
        a, b = g.step(fstim=fstim, istim=istim), o.step(fstim=fstim, istim=istim)
        assert np.array_equal(a, b), "cycle %d" % c
        for p in spec.populations:
            if p.type_name in fired:
                fired[p.type_name] += int(np.isin(a, p.idx).sum())
    assert min(fired.values()) > 20, fired
    for p in spec.populations:
        if p.type_name not in names:
            continue
        nstate = 4 if p.type_name == "IF_curr_exp" else 1
        for var in range(nstate):
            for i in p.idx:
                assert np.float32(g.get_neuron_state(int(i), var)).view(np.uint32) == \
                    np.float32(o.get_neuron_state(int(i), var)).view(np.uint32), (p.type_name, var, i)


def _failing_plugin(tmp_path, name, body):
    """A plugin library (plain C, no kernels) named `name` with the given
    entry points, and its descriptor."""
    (tmp_path / (name + ".ini")).write_text(open(os.path.join(PLUGIN_DIR, "QIFPlugin.ini")).read())
    (tmp_path / "b200").mkdir(exist_ok=True)
    src = tmp_path / (name + ".c")
    # built against the plugin header, so that it carries its ABI version
    src.write_text("#include <nemo_b200_plugin.h>\n" + body)
    subprocess.check_call(["gcc", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
                           "-o", str(tmp_path / "b200" / ("lib%s.so" % name)), str(src)])


@pytest.mark.gpu
def test_plugin_update_error_is_reported(tmp_path):
    """An update that returns a CUDA error code (here 1, cudaErrorInvalidValue,
    without launching anything): nemo_step fails with
    NEMO_CUDA_INVOCATION_ERROR naming the plugin's entry point."""
    _failing_plugin(tmp_path, "FailingUpdate",
                    "int b200_update_neurons(const b200_neuron_batch* batch, void* stream) { return 1; }\n")
    lib = Library()
    lib.add_plugin_path(str(tmp_path))
    net = Network(lib)
    t = net.add_neuron_type("FailingUpdate")
    net.add_neuron(t, 0, 0.04, 0.0)
    sim = Simulation(net, Configuration(lib))
    with pytest.raises(NemoError) as e:
        sim.step()
    assert e.value.status == NEMO_CUDA_INVOCATION_ERROR
    assert "b200_update_neurons" in str(e.value)


@pytest.mark.gpu
def test_plugin_init_error_is_reported(tmp_path):
    """An initialisation that returns a CUDA error code: the simulation is
    not created, with NEMO_CUDA_INVOCATION_ERROR naming b200_init_neurons."""
    _failing_plugin(tmp_path, "FailingInit",
                    "int b200_update_neurons(const b200_neuron_batch* batch, void* stream) { return 0; }\n"
                    "int b200_init_neurons(const b200_neuron_batch* batch, void* stream) { return 1; }\n")
    lib = Library()
    lib.add_plugin_path(str(tmp_path))
    net = Network(lib)
    t = net.add_neuron_type("FailingInit")
    net.add_neuron(t, 0, 0.04, 0.0)
    with pytest.raises(NemoError) as e:
        Simulation(net, Configuration(lib))
    assert e.value.status == NEMO_CUDA_INVOCATION_ERROR
    assert "b200_init_neurons" in str(e.value)


@pytest.mark.gpu
def test_no_parameter_plugin_model(plugin_lib):
    """src/test/test.cpp:988-1006 (plugins/no_parameters): 1000 neurons of
    IzhikevichRS, a model with no parameters that the reference ships only as
    a CUDA kernel, run here as a B200 plugin; 100 cycles without synapses
    leave u and v finite. Then a current of 100 in one cycle makes the
    stimulated neurons fire and reset (v = -65); the others stay at rest."""
    net = Network(plugin_lib)
    rs = net.add_neuron_type("IzhikevichRS")
    for n in range(1000):
        net.add_neuron(rs, n, -13.0, -65.0)
    sim = Simulation(net, Configuration(plugin_lib))
    for _ in range(100):
        sim.step()
        u, v = sim.get_neuron_state(100, 0), sim.get_neuron_state(100, 1)
        assert np.isfinite(u) and np.isfinite(v)
    fired = sim.step(istim=[(n, 100.0) for n in range(0, 1000, 3)])
    assert np.array_equal(fired, np.arange(0, 1000, 3, dtype=np.uint32))
    assert sim.get_membrane_potential(0) == -65.0 and sim.get_membrane_potential(1) != -65.0


def test_build_plugin_places_and_rebuilds(tmp_path):
    """nemo_b200.build.build_plugin compiles <dir>/<Name>.cu into
    <dir>/b200/lib<Name>.so, exporting the entry point, and rebuilds only when
    the source is newer than the library."""
    src = tmp_path / "Tiny.cu"
    src.write_text('#include <nemo_b200_plugin.h>\n'
                   'extern "C" int b200_update_neurons(const b200_neuron_batch* b, void* s) { return 0; }\n')
    out = nb_build.build_plugin(str(src))
    assert out == str(tmp_path / "b200" / "libTiny.so")
    assert hasattr(ctypes.CDLL(out), "b200_update_neurons")
    t0 = os.path.getmtime(out)
    assert nb_build.build_plugin(str(src)) == out and os.path.getmtime(out) == t0
    os.utime(src, (t0 + 10, t0 + 10))
    nb_build.build_plugin(str(src))
    assert os.path.getmtime(out) > t0
    other = nb_build.build_plugin(str(src), name="Renamed", plugin_dir=str(tmp_path / "elsewhere"))
    assert other == str(tmp_path / "elsewhere" / "b200" / "libRenamed.so") and os.path.exists(other)


def test_plugin_batch_layout(tmp_path):
    """The binary layout of b200_neuron_batch on LP64 (the plugin ABI): field
    offsets and size as compiled plugins see them, from a C compiler."""
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include <nemo_b200_plugin.h>\n'
                   '#define F(x) printf("%s %zu\\n", #x, offsetof(b200_neuron_batch, x));\n'
                   'int main(void) { F(count) F(cycle) F(param) F(param_stride) F(state) F(state_stride)\n'
                   ' F(current_epsp) F(current_ipsp) F(current_external) F(fstim) F(recent_firing) F(fired) F(rng)\n'
                   ' printf("size %zu\\n", sizeof(b200_neuron_batch)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)], text=True).splitlines())
    expected = {"count": 0, "cycle": 8, "param": 16, "param_stride": 24, "state": 32, "state_stride": 40,
                "current_epsp": 48, "current_ipsp": 56, "current_external": 64, "fstim": 72,
                "recent_firing": 80, "fired": 88, "rng": 96, "size": 104}
    assert {k: int(v) for k, v in got.items()} == expected
