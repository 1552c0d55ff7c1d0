"""ctypes binding of the NeMo C ABI (include/nemo.h).

Mirrors the reference Python API (src/api/python/nemo_py.cpp:733-815):
``Network``, ``Configuration`` and ``Simulation`` with the same method names
(``add_neuron_type``, ``add_neuron``, ``add_synapse``, ``step``,
``apply_stdp``, ``get_synapses_from`` ...), including the vector forms of
``add_neuron`` / ``add_synapse``. Errors raise :class:`NemoError` carrying the
C ABI status code and ``nemo_strerror()`` message, like the reference
binding's translation of ``nemo::exception``.

The binding is bound to one shared library; by default the B200 library
``libnemo_b200.so`` built in this package. Loading fails loudly when it is
missing: there is no fallback implementation.
"""

import ctypes
import os
from ctypes import (POINTER, byref, c_char_p, c_float, c_int, c_size_t,
                    c_uint, c_uint64, c_ubyte, c_ulong, c_void_p)

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIBRARY = os.path.join(_HERE, "libnemo_b200.so")

NEMO_OK = 0
NEMO_API_UNSUPPORTED = 5
NEMO_INVALID_INPUT = 6
NEMO_LOGIC_ERROR = 9
NEMO_UNKNOWN_ERROR = 14
NEMO_BACKEND_CUDA = 0
NEMO_BACKEND_CPU = 1


class NemoError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("nemo error %d: %s" % (status, message))
        self.status = status
        self.message = message


_PROTOTYPES = {
    "nemo_version": (c_char_p, []),
    "nemo_strerror": (c_char_p, []),
    "nemo_add_plugin_path": (c_int, [c_char_p]),
    "nemo_cuda_device_count": (c_int, [POINTER(c_uint)]),
    "nemo_cuda_device_description": (c_int, [c_uint, POINTER(c_char_p)]),
    "nemo_new_configuration": (c_void_p, []),
    "nemo_delete_configuration": (None, [c_void_p]),
    "nemo_log_stdout": (c_int, [c_void_p]),
    "nemo_set_stdp_function": (c_int, [c_void_p, POINTER(c_float), c_size_t, POINTER(c_float), c_size_t,
                                       c_float, c_float, c_float, c_float]),
    "nemo_set_cpu_backend": (c_int, [c_void_p]),
    "nemo_set_cuda_backend": (c_int, [c_void_p, c_int]),
    "nemo_cuda_device": (c_int, [c_void_p, POINTER(c_int)]),
    "nemo_backend": (c_int, [c_void_p, POINTER(c_uint)]),
    "nemo_backend_description": (c_int, [c_void_p, POINTER(c_char_p)]),
    "nemo_set_write_only_synapses": (c_int, [c_void_p]),
    "nemo_new_network": (c_void_p, []),
    "nemo_delete_network": (None, [c_void_p]),
    "nemo_add_neuron_type": (c_int, [c_void_p, c_char_p, POINTER(c_uint)]),
    "nemo_add_neuron_iz": (c_int, [c_void_p, c_uint] + [c_float] * 7),
    "nemo_add_neuron": (c_int, [c_void_p, c_uint, c_uint, c_uint, POINTER(c_float)]),
    "nemo_add_neurons": (c_int, [c_void_p, c_uint, c_size_t, POINTER(c_uint), c_uint, POINTER(c_float)]),
    "nemo_add_synapse": (c_int, [c_void_p, c_uint, c_uint, c_uint, c_float, c_ubyte, POINTER(c_uint64)]),
    "nemo_add_synapses": (c_int, [c_void_p, c_size_t, POINTER(c_uint), POINTER(c_uint), POINTER(c_uint),
                                  POINTER(c_float), POINTER(c_ubyte), POINTER(c_uint64)]),
    "nemo_neuron_count": (c_int, [c_void_p, POINTER(c_uint)]),
    "nemo_new_simulation": (c_void_p, [c_void_p, c_void_p]),
    "nemo_delete_simulation": (None, [c_void_p]),
    "nemo_step": (c_int, [c_void_p, POINTER(c_uint), c_size_t, POINTER(c_uint), POINTER(c_float), c_size_t,
                          POINTER(POINTER(c_uint)), POINTER(c_size_t)]),
    "nemo_apply_stdp": (c_int, [c_void_p, c_float]),
    "nemo_get_membrane_potential": (c_int, [c_void_p, c_uint, POINTER(c_float)]),
    "nemo_get_neuron_state_n": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_get_neuron_parameter_n": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_get_neuron_state_s": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_get_neuron_parameter_s": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_get_synapse_source_n": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_source_s": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_target_n": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_target_s": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_delay_n": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_delay_s": (c_int, [c_void_p, c_uint64, POINTER(c_uint)]),
    "nemo_get_synapse_weight_n": (c_int, [c_void_p, c_uint64, POINTER(c_float)]),
    "nemo_get_synapse_weight_s": (c_int, [c_void_p, c_uint64, POINTER(c_float)]),
    "nemo_get_synapse_plastic_n": (c_int, [c_void_p, c_uint64, POINTER(c_ubyte)]),
    "nemo_get_synapse_plastic_s": (c_int, [c_void_p, c_uint64, POINTER(c_ubyte)]),
    "nemo_get_synapses_from_n": (c_int, [c_void_p, c_uint, POINTER(POINTER(c_uint64)), POINTER(c_size_t)]),
    "nemo_get_synapses_from_s": (c_int, [c_void_p, c_uint, POINTER(POINTER(c_uint64)), POINTER(c_size_t)]),
    "nemo_set_neuron_n": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_set_neuron_s": (c_int, [c_void_p, c_uint, c_uint, POINTER(c_float)]),
    "nemo_set_neuron_state_n": (c_int, [c_void_p, c_uint, c_uint, c_float]),
    "nemo_set_neuron_parameter_n": (c_int, [c_void_p, c_uint, c_uint, c_float]),
    "nemo_set_neuron_state_s": (c_int, [c_void_p, c_uint, c_uint, c_float]),
    "nemo_set_neuron_parameter_s": (c_int, [c_void_p, c_uint, c_uint, c_float]),
    "nemo_elapsed_wallclock": (c_int, [c_void_p, POINTER(c_ulong)]),
    "nemo_elapsed_simulation": (c_int, [c_void_p, POINTER(c_ulong)]),
    "nemo_reset_timer": (c_int, [c_void_p]),
}


class Library:
    """One loaded implementation of the C ABI."""

    _cache = {}

    def __new__(cls, path=None):
        path = os.path.abspath(path or PRODUCT_LIBRARY)
        if path in cls._cache:
            return cls._cache[path]
        if not os.path.exists(path):
            raise OSError("NeMo library not found: %s (build it with __graft_entry__.build())" % path)
        self = super().__new__(cls)
        self.path = path
        self.dll = ctypes.CDLL(path)
        for name, (restype, argtypes) in _PROTOTYPES.items():
            fn = getattr(self.dll, name)
            fn.restype = restype
            fn.argtypes = argtypes
        cls._cache[path] = self
        return self

    def call(self, name, *args):
        status = getattr(self.dll, name)(*args)
        if status != NEMO_OK:
            raise NemoError(status, self.dll.nemo_strerror().decode(errors="replace"))

    def version(self):
        return self.dll.nemo_version().decode()

    def add_plugin_path(self, path):
        """Search `path` for neuron-model descriptors <Name>.ini (and GPU plugins
        b200/lib<Name>.so beside them) before the default directories
        (nemo_add_plugin_path, src/nemo.h)."""
        self.call("nemo_add_plugin_path", os.fsencode(os.path.abspath(path)))


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1))


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))


def _ptr(a, ctype):
    return a.ctypes.data_as(POINTER(ctype))


class Configuration:
    def __init__(self, lib=None):
        self.lib = lib if isinstance(lib, Library) else Library(lib)
        self.handle = self.lib.dll.nemo_new_configuration()
        if not self.handle:
            raise NemoError(NEMO_UNKNOWN_ERROR, self.lib.dll.nemo_strerror().decode())

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.dll.nemo_delete_configuration(self.handle)
            self.handle = None

    def enable_logging(self):
        self.lib.call("nemo_log_stdout", self.handle)

    def set_stdp_function(self, prefire, postfire, *limits):
        """6-limit form (minE, maxE, minI, maxI) or the 2-limit form
        (minWeight, maxWeight), which maps to (0, maxWeight, 0, minWeight)
        (src/nemo/Configuration.cpp:148-151)."""
        if len(limits) == 2:
            limits = (0.0, limits[1], 0.0, limits[0])
        pre, post = _f32(prefire), _f32(postfire)
        self.lib.call("nemo_set_stdp_function", self.handle, _ptr(pre, c_float), pre.size,
                      _ptr(post, c_float), post.size, *[float(x) for x in limits])

    def set_cuda_backend(self, device=-1):
        self.lib.call("nemo_set_cuda_backend", self.handle, device)

    def set_cpu_backend(self):
        self.lib.call("nemo_set_cpu_backend", self.handle)

    def set_write_only_synapses(self):
        self.lib.call("nemo_set_write_only_synapses", self.handle)

    def backend(self):
        b = c_uint()
        self.lib.call("nemo_backend", self.handle, byref(b))
        return b.value

    def backend_description(self):
        d = c_char_p()
        self.lib.call("nemo_backend_description", self.handle, byref(d))
        return d.value.decode()


class Network:
    def __init__(self, lib=None):
        self.lib = lib if isinstance(lib, Library) else Library(lib)
        self.handle = self.lib.dll.nemo_new_network()

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.dll.nemo_delete_network(self.handle)
            self.handle = None

    def add_neuron_type(self, name):
        t = c_uint()
        self.lib.call("nemo_add_neuron_type", self.handle, name.encode(), byref(t))
        return t.value

    def add_neuron(self, type, idx, *args):
        """Scalar form add_neuron(type, idx, p0, p1, ..., s0, ...) or vector
        form with equal-length arrays for idx and every argument."""
        if np.ndim(idx) == 0:
            a = _f32(args)
            self.lib.call("nemo_add_neuron", self.handle, type, int(idx), a.size, _ptr(a, c_float))
            return
        idx = _u32(idx)
        cols = [np.broadcast_to(np.asarray(x, dtype=np.float32), idx.shape) for x in args]
        a = np.ascontiguousarray(np.stack(cols, axis=1) if cols else np.zeros((idx.size, 0), np.float32))
        self.lib.call("nemo_add_neurons", self.handle, type, idx.size, _ptr(idx, c_uint), len(cols),
                      _ptr(a, c_float))

    def add_neuron_iz(self, idx, a, b, c, d, u, v, sigma):
        self.lib.call("nemo_add_neuron_iz", self.handle, idx, a, b, c, d, u, v, sigma)

    def add_synapse(self, source, target, delay, weight, plastic):
        if all(np.ndim(x) == 0 for x in (source, target, delay, weight, plastic)):
            sid = c_uint64()
            self.lib.call("nemo_add_synapse", self.handle, int(source), int(target), int(delay),
                          float(weight), int(bool(plastic)), byref(sid))
            return sid.value
        n = max(np.size(x) for x in (source, target, delay, weight, plastic))
        src = _u32(np.broadcast_to(source, (n,)))
        tgt = _u32(np.broadcast_to(target, (n,)))
        dly = _u32(np.broadcast_to(delay, (n,)))
        w = _f32(np.broadcast_to(weight, (n,)))
        pl = np.ascontiguousarray(np.broadcast_to(np.asarray(plastic).astype(np.uint8), (n,)))
        ids = np.empty(n, dtype=np.uint64)
        self.lib.call("nemo_add_synapses", self.handle, n, _ptr(src, c_uint), _ptr(tgt, c_uint),
                      _ptr(dly, c_uint), _ptr(w, c_float), _ptr(pl, c_ubyte), _ptr(ids, c_uint64))
        return ids

    def neuron_count(self):
        n = c_uint()
        self.lib.call("nemo_neuron_count", self.handle, byref(n))
        return n.value

    def set_neuron(self, idx, *args):
        a = _f32(args)
        self.lib.call("nemo_set_neuron_n", self.handle, idx, a.size, _ptr(a, c_float))

    def get_neuron_state(self, idx, var):
        v = c_float()
        self.lib.call("nemo_get_neuron_state_n", self.handle, idx, var, byref(v))
        return v.value

    def get_neuron_parameter(self, idx, p):
        v = c_float()
        self.lib.call("nemo_get_neuron_parameter_n", self.handle, idx, p, byref(v))
        return v.value

    def set_neuron_state(self, idx, var, val):
        self.lib.call("nemo_set_neuron_state_n", self.handle, idx, var, val)

    def set_neuron_parameter(self, idx, p, val):
        self.lib.call("nemo_set_neuron_parameter_n", self.handle, idx, p, val)

    def get_synapses_from(self, source):
        return _synapses_from(self.lib, "nemo_get_synapses_from_n", self.handle, source)

    def get_synapse_source(self, sid):
        return _query(self.lib, "nemo_get_synapse_source_n", self.handle, sid, c_uint)

    def get_synapse_target(self, sid):
        return _query(self.lib, "nemo_get_synapse_target_n", self.handle, sid, c_uint)

    def get_synapse_delay(self, sid):
        return _query(self.lib, "nemo_get_synapse_delay_n", self.handle, sid, c_uint)

    def get_synapse_weight(self, sid):
        return _query(self.lib, "nemo_get_synapse_weight_n", self.handle, sid, c_float)

    def get_synapse_plastic(self, sid):
        return _query(self.lib, "nemo_get_synapse_plastic_n", self.handle, sid, c_ubyte)


def _query(lib, fn, handle, sid, ctype):
    out = ctype()
    lib.call(fn, handle, c_uint64(int(sid)), byref(out))
    return out.value


def _synapses_from(lib, fn, handle, source):
    ids = POINTER(c_uint64)()
    n = c_size_t()
    lib.call(fn, handle, source, byref(ids), byref(n))
    if n.value == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.ctypeslib.as_array(ids, shape=(n.value,)).copy()


class Simulation:
    def __init__(self, net, conf):
        self.lib = net.lib
        if conf.lib is not net.lib:
            raise ValueError("network and configuration are bound to different libraries")
        self.handle = self.lib.dll.nemo_new_simulation(net.handle, conf.handle)
        if not self.handle:
            # the constructor returns NULL; the status of the failure, where
            # the library reports it
            status = self.lib.dll.nemo_b200_last_status() if hasattr(self.lib.dll, "nemo_b200_last_status") else -1
            raise NemoError(status, self.lib.dll.nemo_strerror().decode(errors="replace"))
        self._fired = POINTER(c_uint)()
        self._nfired = c_size_t()

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.dll.nemo_delete_simulation(self.handle)
            self.handle = None

    def step(self, fstim=(), istim=()):
        """One 1 ms cycle. fstim: neuron indices forced to fire; istim: sequence
        of (neuron, current) pairs. Returns the fired neurons (uint32 array)."""
        f = _u32(fstim) if len(fstim) else None
        if len(istim):
            inidx = _u32([p[0] for p in istim])
            icur = _f32([p[1] for p in istim])
        else:
            inidx = icur = None
        self.lib.call("nemo_step", self.handle,
                      _ptr(f, c_uint) if f is not None else None, 0 if f is None else f.size,
                      _ptr(inidx, c_uint) if inidx is not None else None,
                      _ptr(icur, c_float) if icur is not None else None,
                      0 if inidx is None else inidx.size,
                      byref(self._fired), byref(self._nfired))
        n = self._nfired.value
        if n == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(self._fired, shape=(n,)).copy()

    def apply_stdp(self, reward):
        self.lib.call("nemo_apply_stdp", self.handle, float(reward))

    def get_membrane_potential(self, idx):
        v = c_float()
        self.lib.call("nemo_get_membrane_potential", self.handle, idx, byref(v))
        return v.value

    def get_neuron_state(self, idx, var):
        v = c_float()
        self.lib.call("nemo_get_neuron_state_s", self.handle, idx, var, byref(v))
        return v.value

    def get_neuron_parameter(self, idx, p):
        v = c_float()
        self.lib.call("nemo_get_neuron_parameter_s", self.handle, idx, p, byref(v))
        return v.value

    def set_neuron(self, idx, *args):
        a = _f32(args)
        self.lib.call("nemo_set_neuron_s", self.handle, idx, a.size, _ptr(a, c_float))

    def set_neuron_state(self, idx, var, val):
        self.lib.call("nemo_set_neuron_state_s", self.handle, idx, var, val)

    def set_neuron_parameter(self, idx, p, val):
        self.lib.call("nemo_set_neuron_parameter_s", self.handle, idx, p, val)

    def get_synapses_from(self, source):
        return _synapses_from(self.lib, "nemo_get_synapses_from_s", self.handle, source)

    def get_synapse_source(self, sid):
        return _query(self.lib, "nemo_get_synapse_source_s", self.handle, sid, c_uint)

    def get_synapse_target(self, sid):
        return _query(self.lib, "nemo_get_synapse_target_s", self.handle, sid, c_uint)

    def get_synapse_delay(self, sid):
        return _query(self.lib, "nemo_get_synapse_delay_s", self.handle, sid, c_uint)

    def get_synapse_weight(self, sid):
        return _query(self.lib, "nemo_get_synapse_weight_s", self.handle, sid, c_float)

    def get_synapse_plastic(self, sid):
        return _query(self.lib, "nemo_get_synapse_plastic_s", self.handle, sid, c_ubyte)

    def run(self, cycles):
        """Device-resident run of `cycles` cycles without stimulus
        (nemo_b200_run); returns the fired count of each cycle."""
        counts = np.zeros(cycles, dtype=np.uint32)
        fn = self.lib.dll.nemo_b200_run
        fn.argtypes = [c_void_p, c_uint, POINTER(ctypes.c_uint32), POINTER(c_uint64)]
        self.lib.call("nemo_b200_run", self.handle, cycles, counts.ctypes.data_as(POINTER(ctypes.c_uint32)), None)
        return counts

    def fired_at(self, cycle):
        """Fired neurons of one of the last 1024 cycles (nemo_b200_fired_at),
        in nemo_step's order."""
        ptr = POINTER(c_uint)()
        n = c_size_t()
        fn = self.lib.dll.nemo_b200_fired_at
        fn.argtypes = [c_void_p, c_uint64, POINTER(POINTER(c_uint)), POINTER(c_size_t)]
        self.lib.call("nemo_b200_fired_at", self.handle, cycle, byref(ptr), byref(n))
        if n.value == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).astype(np.uint32)

    def autotune(self, trial_cycles=100):
        """Choose the step kernel's work shape by timing (nemo_b200_autotune_shape):
        returns (threads per block, synapses of a full STDP entry, {(threads,
        run): ms per cycle}). The trial cycles are simulated like any others."""
        threads, run = c_uint(), c_uint()
        ms = (ctypes.c_double * 6)()
        fn = self.lib.dll.nemo_b200_autotune_shape
        fn.argtypes = [c_void_p, c_uint, POINTER(c_uint), POINTER(c_uint), ctypes.c_double * 6]
        self.lib.call("nemo_b200_autotune_shape", self.handle, trial_cycles, byref(threads), byref(run), ms)
        table = {(t, r): ms[3 * i + k] for i, r in enumerate((128, 64)) for k, t in enumerate((1024, 512, 256))
                 if ms[3 * i + k] > 0}
        return threads.value, run.value, table

    def host_bytes(self):
        """Bytes that nemo_step calls moved to and from the device since the
        simulation was made (nemo_b200_host_bytes): (to device, to host)."""
        out = (ctypes.c_ulonglong * 2)()
        fn = self.lib.dll.nemo_b200_host_bytes
        fn.argtypes = [c_void_p, ctypes.c_ulonglong * 2]
        self.lib.call("nemo_b200_host_bytes", self.handle, out)
        return int(out[0]), int(out[1])

    def get_weights(self, ids):
        """Weights of many synapses at once (nemo_b200_get_weights)."""
        ids = np.ascontiguousarray(np.asarray(ids, dtype=np.uint64))
        out = np.empty(ids.size, dtype=np.float32)
        fn = self.lib.dll.nemo_b200_get_weights
        fn.argtypes = [c_void_p, POINTER(c_uint64), c_size_t, POINTER(c_float)]
        self.lib.call("nemo_b200_get_weights", self.handle, ids.ctypes.data_as(POINTER(c_uint64)), ids.size,
                      out.ctypes.data_as(POINTER(c_float)))
        return out

    def elapsed_wallclock(self):
        e = c_ulong()
        self.lib.call("nemo_elapsed_wallclock", self.handle, byref(e))
        return e.value

    def elapsed_simulation(self):
        e = c_ulong()
        self.lib.call("nemo_elapsed_simulation", self.handle, byref(e))
        return e.value

    def reset_timer(self):
        self.lib.call("nemo_reset_timer", self.handle)
def _bind_shard(lib):
    d = lib.dll
    if getattr(d, "_shard_bound", False):
        return d
    d.nemo_b200_new_shard.restype = ctypes.c_void_p
    d.nemo_b200_new_shard.argtypes = [ctypes.c_void_p, ctypes.c_void_p, c_uint, c_uint]
    d.nemo_b200_shard_warps.argtypes = [c_uint, c_uint, c_uint, POINTER(c_uint), POINTER(c_uint)]
    d.nemo_b200_shard_range.argtypes = [ctypes.c_void_p, POINTER(c_uint), POINTER(c_uint), POINTER(c_uint)]
    d.nemo_b200_shard_step.argtypes = [ctypes.c_void_p, POINTER(c_uint), c_size_t, POINTER(c_uint), POINTER(c_float),
                                       c_size_t, POINTER(ctypes.c_uint32)]
    d.nemo_b200_shard_deliver.argtypes = [ctypes.c_void_p, POINTER(ctypes.c_uint32), POINTER(POINTER(c_uint)),
                                          POINTER(c_size_t)]
    d.nemo_b200_shard_step_async.argtypes = [ctypes.c_void_p, POINTER(c_uint), c_size_t, POINTER(c_uint),
                                             POINTER(c_float), c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    d.nemo_b200_shard_deliver_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    d.nemo_b200_stream_wait.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    d._shard_bound = True
    return d


class ShardedSimulation(Simulation):
    """Shard `rank` of `world` of one network simulated over several GPUs,
    one process each (nemo_b200_new_shard): the shard updates the neurons of
    its own warp range and holds the synapses to them. Every cycle the
    shards' fired words are all-gathered -- ``exchange(local_words)`` returns
    the cycle's words of all warps; by default
    ``nemo_b200.dist.exchange_fired_words`` over torch.distributed -- and
    delivered. Firing and weights equal the unsharded simulation's."""

    def __init__(self, net, conf, rank, world, exchange=None):
        self.lib = net.lib
        d = _bind_shard(self.lib)
        self.handle = d.nemo_b200_new_shard(net.handle, conf.handle, int(rank), int(world))
        if not self.handle:
            raise NemoError(-1, d.nemo_strerror().decode(errors="replace"))
        first, words, total = c_uint(), c_uint(), c_uint()
        self.lib.call("nemo_b200_shard_range", self.handle, byref(first), byref(words), byref(total))
        self.rank, self.world = int(rank), int(world)
        self.first_word, self.words, self.total_words = first.value, words.value, total.value
        self._exchange = exchange
        self._fired = POINTER(c_uint)()
        self._nfired = c_size_t()

    def step_local(self, fstim=(), istim=()):
        """Stimulus (entries for other shards' neurons are skipped) and the
        update of this shard's neurons; returns its fired words."""
        f = _u32(fstim) if len(fstim) else None
        if len(istim):
            inidx = _u32([p[0] for p in istim])
            icur = _f32([p[1] for p in istim])
        else:
            inidx = icur = None
        out = np.zeros(self.words, dtype=np.uint32)
        self.lib.call("nemo_b200_shard_step", self.handle,
                      _ptr(f, c_uint) if f is not None else None, 0 if f is None else f.size,
                      _ptr(inidx, c_uint) if inidx is not None else None,
                      _ptr(icur, c_float) if icur is not None else None,
                      0 if inidx is None else inidx.size,
                      out.ctypes.data_as(POINTER(ctypes.c_uint32)))
        return out

    def deliver(self, all_words):
        """The cycle's fired words of every warp; returns all fired neurons."""
        a = np.ascontiguousarray(all_words, dtype=np.uint32)
        if a.size != self.total_words:
            raise ValueError("expected %d fired words, got %d" % (self.total_words, a.size))
        self.lib.call("nemo_b200_shard_deliver", self.handle, a.ctypes.data_as(POINTER(ctypes.c_uint32)),
                      byref(self._fired), byref(self._nfired))
        n = self._nfired.value
        if n == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(self._fired, shape=(n,)).copy()

    def step(self, fstim=(), istim=()):
        local = self.step_local(fstim, istim)
        if self._exchange is not None:
            all_words = self._exchange(local)
        else:
            from .dist import exchange_fired_words
            all_words = exchange_fired_words(local, self.first_word, self.total_words)
        return self.deliver(all_words)

    def step_device(self, fstim=(), istim=(), exchange=None):
        """One cycle with the fired words exchanged as CUDA tensors on the
        current stream (nemo_b200_shard_step_async / _deliver_async):
        nothing waits on the host and no word crosses to host memory.
        ``exchange(local)`` maps this shard's words (int32 CUDA tensor) to
        every warp's; by default nemo_b200.dist.exchange_fired_words_device
        (NCCL). The cycle's fired neurons: fired_at(cycle)."""
        import torch
        from .dist import exchange_fired_words_device
        f = _u32(fstim) if len(fstim) else None
        if len(istim):
            inidx = _u32([p[0] for p in istim])
            icur = _f32([p[1] for p in istim])
        else:
            inidx = icur = None
        stream = torch.cuda.current_stream().cuda_stream
        local = torch.empty(self.words, dtype=torch.int32, device="cuda")
        self.lib.call("nemo_b200_shard_step_async", self.handle,
                      _ptr(f, c_uint) if f is not None else None, 0 if f is None else f.size,
                      _ptr(inidx, c_uint) if inidx is not None else None,
                      _ptr(icur, c_float) if icur is not None else None,
                      0 if inidx is None else inidx.size, local.data_ptr(), stream)
        if exchange is None:
            all_words = exchange_fired_words_device(local, self.first_word, self.total_words)
        else:
            all_words = exchange(local)
        self.lib.call("nemo_b200_shard_deliver_async", self.handle, all_words.data_ptr(), stream)
        # the simulation reads both buffers later on its own stream: keep
        # them until the next cycle's step, which that stream runs after
        self._in_flight = (local, all_words)

    def stream_wait(self):
        """Order the current stream after the simulation's queued work."""
        import torch
        self.lib.call("nemo_b200_stream_wait", self.handle, torch.cuda.current_stream().cuda_stream)



