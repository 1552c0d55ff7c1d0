"""nemo_b200 — a B200-native backend for the NeMo spiking-network simulator.

The product is the shared library ``libnemo_b200.so`` (C ABI in
``include/nemo.h``), whose per-cycle step path runs as hand-written sm_100a
CUDA kernels. This package holds its sources (``csrc/``), the neuron-model
descriptors (``plugins/``), a ctypes binding mirroring the reference Python
API (:mod:`nemo_b200.nemo`, with :class:`ShardedSimulation` for one network
over several GPUs), the differentiable LIF form (:mod:`nemo_b200.lif`), the
multi-process helpers (:mod:`nemo_b200.dist`) and seeded network generators
(:mod:`nemo_b200.netgen`).
"""

from .nemo import (Configuration, Library, NemoError, Network, Simulation,  # noqa: F401
                   ShardedSimulation, PRODUCT_LIBRARY)
