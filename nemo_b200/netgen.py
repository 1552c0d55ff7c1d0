"""Seeded synthetic networks.

Every generator returns plain numpy arrays (a :class:`NetSpec`) that are added
to a network through the vector forms of ``add_neuron`` / ``add_synapse``, so
that two implementations of the C ABI receive identical networks by
construction.

* :func:`izhikevich_random` — the random excitatory/inhibitory Izhikevich
  network of the reference's examples (src/examples/randomNetUtils.cpp:6-55):
  excitatory a=0.02, b=0.2, c=-65+15r^2, d=8-6r^2, sigma 5; inhibitory
  a=0.02+0.08r, b=0.25-0.05r, c=-65, d=2, sigma 2; v=-65, u=b*v; M outgoing
  synapses per neuron to uniform targets with uniform delays 1..dmax, weights
  0.5*U(0,1) (excitatory) and -U(0,1) (inhibitory), excitatory synapses plastic
  when STDP is used. With n=1000, m=100, dmax=20 this is the 1000-neuron
  benchmark network; with n=100000, m=1000 the 1e8-synapse STDP network.
* :func:`ring` — the reference's ring network (src/test/utils.cpp:132-155).
* :func:`mixed_plugins` — Izhikevich / IF_curr_exp / QIF / HH populations.
* :func:`batched_sizes` — instance sizes log-uniform in [lo, hi].

A :class:`NetSpec` saves to one file and loads from it (:meth:`NetSpec.save`,
:meth:`NetSpec.load`), so that a network is generated once and the same file
is built by the B200 library and by the oracle.
"""

from dataclasses import dataclass, field
from typing import List

import numpy as np


@dataclass
class Population:
    type_name: str
    idx: np.ndarray            # uint32 user indices
    args: List[np.ndarray]     # per-argument float32 arrays (parameters, then state)


@dataclass
class NetSpec:
    populations: List[Population] = field(default_factory=list)
    source: np.ndarray = None
    target: np.ndarray = None
    delay: np.ndarray = None
    weight: np.ndarray = None
    plastic: np.ndarray = None

    @property
    def neuron_count(self):
        return int(sum(p.idx.size for p in self.populations))

    @property
    def synapse_count(self):
        return 0 if self.source is None else int(self.source.size)

    def out_degree(self):
        n = self.neuron_count
        return np.bincount(self.source, minlength=n) if self.source is not None else np.zeros(n, np.int64)

    FORMAT = "nemo-b200-network-v1"

    def save(self, path):
        """Write the network to one file (numpy .npz: the neuron types in
        registration order with their indices and per-argument arrays, then
        the synapses in insertion order), so that every implementation of the
        C ABI -- the B200 library and the oracle -- builds it from the same
        file."""
        arrays = {"format": np.array(self.FORMAT), "types": np.array([p.type_name for p in self.populations])}
        for k, p in enumerate(self.populations):
            arrays["idx_%d" % k] = np.asarray(p.idx, np.uint32)
            arrays["args_%d" % k] = (np.stack([np.asarray(a, np.float32) for a in p.args])
                                     if p.args else np.zeros((0, p.idx.size), np.float32))
        if self.synapse_count:
            arrays.update(source=np.asarray(self.source, np.uint32), target=np.asarray(self.target, np.uint32),
                          delay=np.asarray(self.delay, np.uint32), weight=np.asarray(self.weight, np.float32),
                          plastic=np.asarray(self.plastic, np.uint8))
        with open(path, "wb") as f:
            np.savez(f, **arrays)

    @classmethod
    def load(cls, path):
        """The network a :meth:`save` wrote."""
        with np.load(path, allow_pickle=False) as z:
            if "format" not in z.files or str(z["format"]) != cls.FORMAT:
                raise ValueError("%s is not a %s file" % (path, cls.FORMAT))
            pops = []
            for k, name in enumerate(z["types"]):
                args = z["args_%d" % k]
                pops.append(Population(str(name), z["idx_%d" % k].copy(), [a.copy() for a in args]))
            spec = cls(pops)
            if "source" in z.files:
                spec.source, spec.target = z["source"].copy(), z["target"].copy()
                spec.delay, spec.weight, spec.plastic = z["delay"].copy(), z["weight"].copy(), z["plastic"].copy()
            return spec

    def build(self, net):
        """Add the neurons and synapses to a nemo.Network (any library)."""
        for p in self.populations:
            t = net.add_neuron_type(p.type_name)
            net.add_neuron(t, p.idx, *p.args)
        if self.synapse_count:
            net.add_synapse(self.source, self.target, self.delay, self.weight, self.plastic)
        return net


def izhikevich_random(n, m, dmax=20, seed=0, stdp=False, sigma_exc=5.0, sigma_inh=2.0,
                      exc_fraction=0.8):
    rng = np.random.default_rng(seed)
    f32 = np.float32
    nexc = int(n * exc_fraction)
    ninh = n - nexc
    # excitatory (regular spiking)
    r1 = rng.random(nexc, dtype=f32)
    r2 = rng.random(nexc, dtype=f32)
    a_e = np.full(nexc, 0.02, f32)
    b_e = np.full(nexc, 0.2, f32)
    c_e = (f32(-65.0) + f32(15.0) * r1 * r1).astype(f32)
    d_e = (f32(8.0) - f32(6.0) * r2 * r2).astype(f32)
    # inhibitory (fast spiking)
    r3 = rng.random(ninh, dtype=f32)
    r4 = rng.random(ninh, dtype=f32)
    a_i = (f32(0.02) + f32(0.08) * r3).astype(f32)
    b_i = (f32(0.25) - f32(0.05) * r4).astype(f32)
    c_i = np.full(ninh, -65.0, f32)
    d_i = np.full(ninh, 2.0, f32)
    a = np.concatenate([a_e, a_i])
    b = np.concatenate([b_e, b_i])
    c = np.concatenate([c_e, c_i])
    d = np.concatenate([d_e, d_i])
    sigma = np.concatenate([np.full(nexc, sigma_exc, f32), np.full(ninh, sigma_inh, f32)])
    v = np.full(n, -65.0, f32)
    u = (b * v).astype(f32)
    pop = Population("Izhikevich", np.arange(n, dtype=np.uint32), [a, b, c, d, sigma, u, v])

    s = NetSpec([pop])
    if m > 0:
        total = n * m
        s.source = np.repeat(np.arange(n, dtype=np.uint32), m)
        s.target = rng.integers(0, n, size=total, dtype=np.uint32)
        s.delay = rng.integers(1, dmax + 1, size=total, dtype=np.uint32)
        w = rng.random(total, dtype=f32)
        exc = s.source < nexc
        s.weight = np.where(exc, f32(0.5) * w, -w).astype(f32)
        s.plastic = (exc & bool(stdp)).astype(np.uint8)
    return s


def ring(ncount, n0=0, plastic=False, nstep=1, delay=1, weight=1000.0):
    """src/test/utils.cpp:124-145: RS neurons (r=0.5, sigma 0) in a ring."""
    idx = (n0 + np.arange(ncount, dtype=np.uint64) * nstep).astype(np.uint32)
    f32 = np.float32
    v = f32(-65.0)
    b = f32(0.2)
    r2 = f32(0.5) * f32(0.5)
    args = [np.full(ncount, 0.02, f32), np.full(ncount, b, f32), np.full(ncount, v + f32(15.0) * r2, f32),
            np.full(ncount, f32(8.0) - f32(6.0) * r2, f32), np.zeros(ncount, f32),
            np.full(ncount, b * v, f32), np.full(ncount, v, f32)]
    s = NetSpec([Population("Izhikevich", idx, args)])
    s.source = idx
    s.target = np.roll(idx, -1)
    s.delay = np.full(ncount, delay, np.uint32)
    s.weight = np.full(ncount, weight, f32)
    s.plastic = np.full(ncount, bool(plastic), np.uint8)
    return s


def standard_stdp(prefire_len=20, postfire_len=20, a_plus=0.1, a_minus=-0.12, tau=20.0):
    """Exponential STDP windows sampled at dt = 1..len: prefire[i] =
    a_plus*exp(-(i+1)/tau), postfire[i] = a_minus*exp(-(i+1)/tau)
    (src/examples/common.cpp:153-164)."""
    i = np.arange(1, prefire_len + 1, dtype=np.float32)
    j = np.arange(1, postfire_len + 1, dtype=np.float32)
    pre = (np.float32(a_plus) * np.exp(-i / np.float32(tau))).astype(np.float32)
    post = (np.float32(a_minus) * np.exp(-j / np.float32(tau))).astype(np.float32)
    return pre, post


def batched_sizes(count, lo=500, hi=20000, seed=0):
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def mixed_plugins(n_iz=20000, n_lif=15000, n_qif=10000, n_hh=5000, m=500, dmax=10, seed=0):
    """Mixed-model network: Izhikevich (80% RS / 20% FS, sigma 0), IF_curr_exp,
    QIF and HH populations, m synapses per neuron to uniform targets across
    all populations, delays U{1..dmax}, weights 0.3*U (excitatory sources) and
    -0.6*U (inhibitory Izhikevich sources)."""
    rng = np.random.default_rng(seed)
    f32 = np.float32
    pops = []
    base = 0
    iz = izhikevich_random(n_iz, 0, seed=seed, sigma_exc=0.0, sigma_inh=0.0)
    pops.append(iz.populations[0])
    base += n_iz
    n_exc_iz = int(n_iz * 0.8)
    if n_lif:
        idx = np.arange(base, base + n_lif, dtype=np.uint32)
        # parameters in IF_curr_exp.h order: v_rest, v_reset, c_m, tau_m,
        # tau_refrac, tau_syn_E, tau_syn_I, v_thresh, i_offset; state v, ie, ii, lastfire
        vals = [-65.0, -65.0, 1.0, 20.0, 2.0, 5.0, 5.0, -50.0, 0.0, -65.0, 0.0, 0.0, 3.0]
        pops.append(Population("IF_curr_exp", idx, [np.full(n_lif, x, f32) for x in vals]))
        base += n_lif
    if n_qif:
        idx = np.arange(base, base + n_qif, dtype=np.uint32)
        pops.append(Population("QIF", idx, [np.full(n_qif, 0.04, f32), np.zeros(n_qif, f32)]))
        base += n_qif
    if n_hh:
        idx = np.arange(base, base + n_hh, dtype=np.uint32)
        # resting state of the squid axon model at v = -65 mV
        vals = [-65.0, 0.3177, 0.0529, 0.5961, 0.0]
        pops.append(Population("HH", idx, [np.full(n_hh, x, f32) for x in vals]))
        base += n_hh
    n = base
    s = NetSpec(pops)
    total = n * m
    s.source = np.repeat(np.arange(n, dtype=np.uint32), m)
    s.target = rng.integers(0, n, size=total, dtype=np.uint32)
    s.delay = rng.integers(1, dmax + 1, size=total, dtype=np.uint32)
    w = rng.random(total, dtype=f32)
    inh = (s.source >= n_exc_iz) & (s.source < n_iz)
    s.weight = np.where(inh, f32(-0.6) * w, f32(0.3) * w).astype(f32)
    s.plastic = np.zeros(total, np.uint8)
    return s
