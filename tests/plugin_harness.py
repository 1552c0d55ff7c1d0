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


# ---- fixed-point conversions and the STDP process (oracle/pin_shim.cpp) ----

FBITS = (0, 10, 20, 24, 30)


def stdp_functions():
    """STDP functions the pins exercise: (prefire, postfire, limits)."""
    f32 = np.float32
    dt = np.arange(1, 21, dtype=f32)
    std_pre = (f32(0.1) * np.exp(-dt / f32(20.0))).astype(f32)
    std_post = (f32(-0.12) * np.exp(-dt / f32(20.0))).astype(f32)
    mixed_pre = np.array([0.1, -0.05, 0.0, 0.2, 0.03, -0.3, 0.0], f32)
    mixed_post = np.array([-0.08, 0.04, 0.0, -0.2, 0.5], f32)
    long_pre = np.linspace(0.3, 0.01, 30).astype(f32)
    long_post = -np.linspace(0.25, 0.02, 30).astype(f32)
    return [(std_pre, std_post, (0.0, 1.0, 0.0, -1.0)),
            (mixed_pre, mixed_post, (0.1, 0.9, -0.2, -1.5)),
            (long_pre, long_post, (0.0, 4.0, 0.0, -4.0)),
            (np.array([0.5], f32), np.array([-0.5], f32), (0.2, 0.6, -0.1, -0.7))]


def pin_inputs(seed=11):
    """Seeded inputs of every pinned function."""
    rng = np.random.default_rng(seed)
    f32 = np.float32
    floats = np.concatenate([
        rng.normal(0, 3, 4000).astype(f32), rng.uniform(-2100, 2100, 2000).astype(f32),
        rng.uniform(-1.5, 1.5, 2000).astype(f32),
        np.array([0.0, -0.0, 1e-30, -1e-30, 2047.999, -2047.999, 2048.0, -2048.0, 1023.5, -1024.0, 0.5, -0.5,
                  1.0 / 3.0, 2.0 ** -20, -(2.0 ** -21), 1e-45], f32)])
    ints = np.concatenate([rng.integers(-2**31, 2**31, 4000, dtype=np.int64),
                           np.array([0, 1, -1, 2**31 - 1, -2**31, 2**20, -2**20], np.int64)]).astype(np.int32)
    wides = np.concatenate([rng.integers(-2**40, 2**40, 3000, dtype=np.int64),
                            rng.integers(-2**33, 2**33, 3000, dtype=np.int64),
                            np.array([0, 2**31 - 1, 2**31, -2**31, -2**31 - 1, 2**62, -2**62], np.int64)])
    ma = rng.integers(-2**31, 2**31, 3000, dtype=np.int64).astype(np.int32)
    mb = rng.integers(-2**24, 2**24, 3000, dtype=np.int64).astype(np.int32)
    spikes = []
    for p in (0.02, 0.1, 0.5):
        bits = rng.random((3000, 64)) < p
        spikes.append((bits.astype(np.uint64) << np.arange(64, dtype=np.uint64)).sum(1, dtype=np.uint64))
    spikes.append(np.uint64(1) << np.arange(64, dtype=np.uint64))
    spikes.append(np.array([0, 2**64 - 1], np.uint64))
    spikes = np.concatenate(spikes).astype(np.uint64)
    w_old = np.concatenate([rng.integers(-2**21, 2**21, 3000, dtype=np.int64),
                            np.array([0, 1, -1, 2**20, -2**20, 2**22, -2**22], np.int64)]).astype(np.int32)
    w_diff = rng.integers(-2**21, 2**21, w_old.size, dtype=np.int64).astype(np.int32)
    return dict(floats=floats, ints=ints, wides=wides, ma=ma, mb=mb, spikes=spikes, w_old=w_old, w_diff=w_diff)


def pin_outputs(lib):
    """Every pinned function of one library (ctypes.CDLL exporting the
    pin_shim.cpp surface) on pin_inputs(): a dict of arrays."""
    import ctypes
    P = ctypes.POINTER
    x = pin_inputs()
    ptr = lambda a, t: a.ctypes.data_as(P(t))   # noqa: E731
    out = {}
    for b in FBITS:
        fix = np.zeros(x["floats"].size, np.int32)
        threw = np.zeros(x["floats"].size, np.uint8)
        lib.pin_fx_to_fix(ptr(x["floats"], ctypes.c_float), ctypes.c_size_t(x["floats"].size), b,
                          ptr(fix, ctypes.c_int32), ptr(threw, ctypes.c_uint8))
        out["to_fix/%d" % b], out["to_fix_threw/%d" % b] = fix, threw
        fl = np.zeros(x["ints"].size, np.float32)
        lib.pin_fx_to_float(ptr(x["ints"], ctypes.c_int32), ctypes.c_size_t(x["ints"].size), b, ptr(fl, ctypes.c_float))
        out["to_float/%d" % b] = fl.view(np.uint32)
        wf = np.zeros(x["wides"].size, np.float32)
        lib.pin_wfx_to_float(ptr(x["wides"], ctypes.c_int64), ctypes.c_size_t(x["wides"].size), b,
                             ptr(wf, ctypes.c_float))
        out["wide_to_float/%d" % b] = wf.view(np.uint32)
        m = np.zeros(x["ma"].size, np.int32)
        lib.pin_fx_mul(ptr(x["ma"], ctypes.c_int32), ptr(x["mb"], ctypes.c_int32), ctypes.c_size_t(x["ma"].size), b,
                       ptr(m, ctypes.c_int32))
        out["mul/%d" % b] = m
    lib.pin_stdp_new.restype = ctypes.c_void_p
    lib.pin_stdp_new.argtypes = [P(ctypes.c_float), ctypes.c_size_t, P(ctypes.c_float), ctypes.c_size_t,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint]
    lib.pin_stdp_delete.argtypes = [ctypes.c_void_p]
    lib.pin_stdp_weight_change.argtypes = [ctypes.c_void_p, P(ctypes.c_uint64), ctypes.c_size_t, P(ctypes.c_int32)]
    lib.pin_stdp_updated_weight.argtypes = [ctypes.c_void_p, P(ctypes.c_int32), P(ctypes.c_int32), ctypes.c_size_t,
                                            P(ctypes.c_int32)]
    for k, (pre, post, lim) in enumerate(stdp_functions()):
        bits = np.zeros(2, np.uint64)
        assert lib.pin_stdp_bits(ptr(pre, ctypes.c_float), ctypes.c_size_t(pre.size), ptr(post, ctypes.c_float),
                                 ctypes.c_size_t(post.size), ptr(bits, ctypes.c_uint64)) == 0
        out["stdp_bits/%d" % k] = bits
        for b in (16, 20):
            h = lib.pin_stdp_new(ptr(pre, ctypes.c_float), pre.size, ptr(post, ctypes.c_float), post.size, *lim, b)
            assert h, "STDP function %d rejected" % k
            wc = np.zeros(x["spikes"].size, np.int32)
            lib.pin_stdp_weight_change(h, ptr(x["spikes"], ctypes.c_uint64), x["spikes"].size, ptr(wc, ctypes.c_int32))
            uw = np.zeros(x["w_old"].size, np.int32)
            lib.pin_stdp_updated_weight(h, ptr(x["w_old"], ctypes.c_int32), ptr(x["w_diff"], ctypes.c_int32),
                                        x["w_old"].size, ptr(uw, ctypes.c_int32))
            lib.pin_stdp_delete(h)
            out["weight_change/%d/%d" % (k, b)] = wc
            out["updated_weight/%d/%d" % (k, b)] = uw
    return out
