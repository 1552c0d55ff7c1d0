"""Seeded single-type drive of a neuron-model update function with the CPU
plugin signature (src/nemo/cpu/plugins/neuron_model.h:25-38), shared by the
oracle pins and by tests/golden/make_golden.py.

Inputs per model follow the parameter/state order of the reference's .ini
descriptors (src/nemo/plugins/*.ini); the currents, external currents and
firing stimulus of each cycle come from a second seeded generator."""

import ctypes
import zlib

import numpy as np

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


def drive_inputs(n, scale, seed=11):
    """Per-cycle (E, I, ext, fstim) of the pins, as an endless generator."""
    drv = np.random.default_rng(seed)
    while True:
        E = np.ascontiguousarray((drv.random(n, dtype=np.float32) * np.float32(scale)).astype(np.float32))
        I = np.ascontiguousarray((-drv.random(n, dtype=np.float32) * np.float32(scale) * np.float32(0.5)).astype(np.float32))
        ext = np.ascontiguousarray(np.where(drv.random(n) < 0.1, np.float32(1.5), np.float32(0)).astype(np.float32))
        fstim = (drv.random(n) < 0.02).astype(np.uint32)
        yield E, I, ext, fstim


PIN_N = 257


def pin_cycles(model):
    return 40 if model == "HH" else 300


def run_digest(fn, model):
    """Run `fn` over the pin's cycles; returns (fired bitmaps [cycles, n/8]
    packed, per-cycle CRC32 of state|history|rng|ext, final state, history,
    rng)."""
    n = PIN_N
    run = _Run(fn, model, n, 7)
    inputs = drive_inputs(n, run.scale)
    fired, crcs = [], []
    for cycle in range(pin_cycles(model)):
        E, I, ext, fstim = next(inputs)
        f, e = run.step(cycle, E, I, ext, fstim)
        fired.append(np.packbits(f.astype(np.uint8)))
        crc = zlib.crc32(run.state.tobytes())
        crc = zlib.crc32(run.rf.tobytes(), crc)
        crc = zlib.crc32(run.rng.tobytes(), crc)
        crc = zlib.crc32(e.tobytes(), crc)
        crcs.append(crc)
    return (np.array(fired, np.uint8), np.array(crcs, np.uint32), run.state.copy(), run.rf.copy(),
            run.rng.copy())
