"""Write tests/golden/plugins.npz from the reference's own CPU neuron-model
plugins, and tests/golden/stdp_fixedpoint.npz from its fixed-point
conversions and STDP process.

oracle/Makefile (`make -C oracle ref`) compiles the unmodified plugin sources
src/nemo/cpu/plugins/{Izhikevich,IF_curr_exp,QIF,HH,PoissonSource,Input}.cpp
of the reference tree into oracle/_ref/lib<Model>.so. This script drives each
one through the seeded single-type run of tests/plugin_harness.py and stores,
per model: the packed firing bitmap of every cycle, a CRC32 per cycle of the
state, firing history, RNG state and external-current array, and the final
state, history and RNG state. The oracle is then checked against these vectors
in the CPU test suite, on machines without the reference sources.

The same recipe compiles src/nemo/{fixedpoint,StdpFunction,StdpProcess}.cpp
into oracle/_ref/libnemo_stdp_ref.so behind oracle/pin_shim.cpp's C surface;
tests/plugin_harness.py pin_outputs() runs every function of it on seeded
inputs (fx_toFix, fx_toFloat, wfx_toFloat, fx_mul over several fractional
widths; potentiation/depression bits, weightChange and updatedWeight of four
STDP functions) and the outputs are stored.

Usage: python tests/golden/make_golden.py   (after `make -C oracle ref`)
"""

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from plugin_harness import MODELS, UPDATE_T, pin_outputs, run_digest  # noqa: E402


def main():
    out = {}
    for model in MODELS:
        path = os.path.join(ROOT, "oracle", "_ref", "lib%s.so" % model)
        if not os.path.exists(path):
            sys.exit("missing %s: run `make -C oracle ref` with the reference sources present" % path)
        fn = UPDATE_T(("cpu_update_neurons", ctypes.CDLL(path)))
        fired, crcs, state, rf, rng = run_digest(fn, model)
        out[model + "/fired"] = fired
        out[model + "/crc"] = crcs
        out[model + "/state"] = state
        out[model + "/rf"] = rf
        out[model + "/rng"] = rng
        print("%-14s cycles %3d  fired %6d" % (model, len(crcs), int(np.unpackbits(fired).sum())))
    np.savez_compressed(os.path.join(HERE, "plugins.npz"), **out)
    path = os.path.join(ROOT, "oracle", "_ref", "libnemo_stdp_ref.so")
    if not os.path.exists(path):
        sys.exit("missing %s: run `make -C oracle ref` with the reference sources present" % path)
    pins = pin_outputs(ctypes.CDLL(path))
    np.savez_compressed(os.path.join(HERE, "stdp_fixedpoint.npz"), **pins)
    print("stdp_fixedpoint: %d arrays" % len(pins))


if __name__ == "__main__":
    main()
