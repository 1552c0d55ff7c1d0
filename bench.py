#!/usr/bin/env python
"""Synaptic events/s of the NeMo step path on B200.

Workload: the 1e8-synapse STDP network — 100,000 Izhikevich neurons (80%
excitatory, thalamic noise sigma 5 / 2), 1000 outgoing synapses per neuron
to uniform targets, delays U{1..20} ms, excitatory weights 0.5*U(0,1)
(plastic), inhibitory -U(0,1); STDP windows 0.1*exp(-dt/20) /
-0.12*exp(-dt/20) over 20+20 ms, excitatory weights clipped to [0, 1];
applyStdp(1.0) every 100 cycles. Seeded synthetic network (numpy PCG64).

One bench step = 100 simulated 1 ms cycles followed by applyStdp(1.0).

  value : synaptic events/s (fired neurons x out-degree, the reference
          benchmark's unit, src/examples/common.cpp:93-98) of the
          device-resident step loop (nemo_b200_timed_steps: one persistent
          launch of 100 cycles + the applyStdp kernel per step), timed with
          CUDA events on the simulation's stream; the 800 MB forward matrix
          exceeds L2. The default 100 steps are the workload's 10,000 cycles.
  e2e   : the same metric through the reference-facing C ABI: nemo_step per
          cycle with a one-neuron firing stimulus copied host->device and the
          fired list copied device->host every cycle, nemo_apply_stdp every
          100 cycles; host wall clock.
  --impl reference : the reference CPU backend (the oracle restatement of
          src/nemo/cpu/, OpenMP on all host cores) on the same network and
          the same e2e protocol, rank 0 only.

Multi-GPU (--gpus N under torchrun): N independent replicas of the workload,
one per GPU (weak scaling); value = all replicas' events / max device time.
--sharded: one network over the N GPUs as shards, the fired words
all-gathered every cycle (strong scaling).
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from nemo_b200 import netgen  # noqa: E402
from nemo_b200.nemo import Configuration, Library, Network, Simulation  # noqa: E402

METRIC = "synaptic events/s"
UNIT = "events/s"
CYCLES_PER_STEP = 100
REWARD = 1.0


def workload(small=False):
    if small:
        return dict(name="izhikevich-20k-m1000-stdp", n=20000, m=1000, dmax=20, seed=1)
    return dict(name="izhikevich-100k-m1000-stdp", n=100000, m=1000, dmax=20, seed=1)


def bench_config(wl, world):
    """The workload description both arms (B200 and reference) report."""
    n, m = wl["n"], wl["m"]
    return {"workload": wl["name"], "neurons": n, "synapses_per_neuron": m, "synapses": n * m,
            "delays": "U{1..%d}" % wl["dmax"], "stdp": "exc plastic, applyStdp(1.0) every 100 cycles",
            "cycles_per_step": CYCLES_PER_STEP, "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (%d MB forward matrix)" % (n * m * 8 // 10**6)}


def build_sim(lib, wl, oracle=False):
    spec = netgen.izhikevich_random(wl["n"], wl["m"], dmax=wl["dmax"], seed=wl["seed"], stdp=True)
    net = spec.build(Network(lib))
    conf = Configuration(lib)
    pre, post = netgen.standard_stdp()
    conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
    conf.set_write_only_synapses()
    if oracle:
        conf.set_cpu_backend()
    t = time.perf_counter()
    sim = Simulation(net, conf)
    build_s = time.perf_counter() - t
    del net
    return sim, spec, build_s


def stim_stream(n, cycles, seed=7):
    """One random neuron forced to fire per cycle (the reference benchmark's
    --fstim option, src/examples/common.cpp:64-67)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, size=cycles, dtype=np.uint32)


def e2e_steps(sim, n, steps, seed):
    """K steps through nemo_step / nemo_apply_stdp; returns (seconds, events)."""
    lib = sim.lib
    stim = stim_stream(n, steps * CYCLES_PER_STEP, seed)
    fptr = ctypes.POINTER(ctypes.c_uint)()
    nfired = ctypes.c_size_t()
    fired_total = 0
    step = lib.dll.nemo_step
    # host buffers and call arguments prepared before the timed region
    base = stim.ctypes.data
    ptrs = [ctypes.cast(base + 4 * k, ctypes.POINTER(ctypes.c_uint)) for k in range(stim.size)]
    fref, nref = ctypes.byref(fptr), ctypes.byref(nfired)
    t0 = time.perf_counter()
    for s in range(steps):
        for c in range(CYCLES_PER_STEP):
            status = step(sim.handle, ptrs[s * CYCLES_PER_STEP + c], 1, None, None, 0, fref, nref)
            if status != 0:
                raise RuntimeError(lib.dll.nemo_strerror().decode())
            fired_total += nfired.value
        if lib.dll.nemo_apply_stdp(sim.handle, ctypes.c_float(REWARD)) != 0:
            raise RuntimeError(lib.dll.nemo_strerror().decode())
    t1 = time.perf_counter()
    return t1 - t0, fired_total


def run_oracle_steps(wl, warmup, steps, budget_s=None):
    """The oracle (reference CPU backend restatement, OpenMP on all host
    cores) on the workload: `warmup` untimed steps, then up to `steps` timed
    steps of 100 cycles + applyStdp, stopping early after budget_s seconds."""
    lib = Library(oracle_library())
    sim, spec, build_s = build_sim(lib, wl, oracle=True)
    m = wl["m"]
    for s in range(warmup):
        e2e_steps(sim, wl["n"], 1, seed=100 + s)
    times, events = [], 0
    t_start = time.perf_counter()
    done = 0
    while done < steps:
        dt, fired = e2e_steps(sim, wl["n"], 1, seed=1000 + done)
        times.append(dt)
        events += fired * m
        done += 1
        if budget_s is not None and time.perf_counter() - t_start > budget_s:
            break
    total = sum(times)
    return events / total, done, total, build_s


def cpu_model():
    """The host CPU's model name (stated beside every CPU figure)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def oracle_library():
    path = os.path.join(ROOT, "oracle", "_build", "libnemo_oracle.so")
    if not os.path.exists(path):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return path


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region,
    into a temporary file (or the file NEMO_B200_CLOCKS_CSV names, which is
    kept)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.keep = bool(os.environ.get("NEMO_B200_CLOCKS_CSV"))
        if self.keep:
            self.path = os.path.abspath(os.environ["NEMO_B200_CLOCKS_CSV"])
        else:
            fd, self.path = tempfile.mkstemp(prefix="nemo_b200_clocks_", suffix=".csv")
            os.close(fd)

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: wait for its first sample so
        # that the samples cover the region that follows
        deadline = time.time() + 5.0
        while time.time() < deadline and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            if self.proc is None or not os.path.exists(self.path):
                return None
            return self._summary()
        finally:
            if not self.keep and os.path.exists(self.path):
                os.unlink(self.path)

    def _summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        p = json.load(open(path))
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def load_traffic(kernel, workload_name):
    """DRAM bytes per launch of `kernel` on the workload, from the committed
    ncu summary (a 1-pass dram__bytes_read.sum + dram__bytes_write.sum
    capture of a full-size launch); None when there is none."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_%s.md" % workload_name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) == 4 and f[0] == "traffic" and f[1] == kernel and f[2] == workload_name:
            return float(f[3])
    return None


def parity_check(wl, cycles_before=100, cycles_after=50):
    """The headline workload on a fresh B200 simulation and a fresh oracle
    simulation: `cycles_before` cycles in one device-resident launch (the
    timed path), applyStdp(1.0), `cycles_after` more; the fired list of every
    cycle compared. The firing after the apply depends on every weight the
    apply changed."""
    lib = Library()
    sim, _, _ = build_sim(lib, wl)
    osim, _, _ = build_sim(Library(oracle_library()), wl, oracle=True)
    bad = firings = 0
    cycle = 0
    for block in (cycles_before, cycles_after):
        lib.dll.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p]
        lib.call("nemo_b200_run", sim.handle, block, None, None)
        for k in range(block):
            want = osim.step()
            got = sim.fired_at(cycle + k)
            bad += 0 if np.array_equal(got, want) else 1
            firings += want.size
        cycle += block
        if block == cycles_before:
            sim.apply_stdp(REWARD)
            osim.apply_stdp(REWARD)
    return {"cycles_checked": cycle, "applies": 1, "mismatched_cycles": bad, "firings": firings,
            "against": "oracle (reference CPU backend restated), fired list of every cycle",
            "path": "device-resident launches, as timed"}


def roofline(sim, lib, wl):
    """Device times of one step's two kernels — the persistent step kernel
    (100 cycles of update, spike push and STDP accumulation) and applyStdp —
    and the dominant one's algorithmic bytes / time against the measured HBM
    copy bandwidth. Algorithmic bytes (per unit of work of the reference
    algorithm): spike delivery 8 B per delivered synapse (packed
    target/delay + i32 weight); Izhikevich update 92 B per neuron per cycle;
    STDP accumulation 20 B per (post-spike x plastic in-synapse) visit (4 B
    reverse synapse, 8 B source history, 4+4 B accumulator); applyStdp 20 B
    per plastic synapse."""
    out = (ctypes.c_double * 10)()
    lib.dll.nemo_b200_profile.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_float, ctypes.c_double * 10]
    lib.call("nemo_b200_profile", sim.handle, CYCLES_PER_STEP, ctypes.c_float(REWARD), out)
    tcyc, blocks, _, pushed, fired, visits, updates, tapply, nplastic, generated = list(out)
    kernels = {
        "k_cycles": (8.0 * pushed + 92.0 * updates + 20.0 * visits, tcyc, 1),
        "k_apply_stdp": (20.0 * nplastic, tapply, 1),
    }
    peak, peak_kind = measured_peaks()
    table = {}
    for k, (bytes_, ms, launches) in kernels.items():
        gbs = bytes_ / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        table[k] = {"ms_per_launch": ms / launches, "bytes_per_launch": bytes_ / launches, "gbs": gbs,
                    "share": 0.0}
    tot = tcyc + tapply
    for k, (bytes_, ms, launches) in kernels.items():
        table[k]["share"] = ms / tot if tot else 0.0
    dom = max(table, key=lambda k: table[k]["share"])
    d = table[dom]
    roof = {"kernel": dom, "bound": "hbm", "achieved": round(d["gbs"], 1), "peak": peak, "unit": "GB/s",
            "frac": round(d["gbs"] / peak, 4), "peak_source": peak_kind, "traffic": load_traffic(dom, wl["name"]),
            "bytes_per_launch": d["bytes_per_launch"], "ms_per_launch": d["ms_per_launch"],
            "per_kernel": {k: {kk: (round(vv, 5) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                           for k, v in table.items()},
            "work_per_step": {"cycles": CYCLES_PER_STEP, "pushed_synapses": int(pushed), "fired": int(fired),
                              "stdp_visits": int(visits), "neuron_updates": int(updates),
                              "plastic_synapses": int(nplastic), "grid_blocks": int(blocks)}}
    return roof


def apply_launches(sim, lib):
    """Kernel launches of one applyStdp (one per group of owner regions)."""
    lib.dll.nemo_b200_apply_launches.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint)]
    n = ctypes.c_uint()
    lib.call("nemo_b200_apply_launches", sim.handle, ctypes.byref(n))
    return n.value


def run_b200(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    wl = workload(args.small)
    lib = Library()
    torch.cuda.set_device(local)
    conf_dev = local

    spec = netgen.izhikevich_random(wl["n"], wl["m"], dmax=wl["dmax"], seed=wl["seed"], stdp=True)
    net = spec.build(Network(lib))
    conf = Configuration(lib)
    pre, post = netgen.standard_stdp()
    conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
    conf.set_write_only_synapses()
    conf.set_cuda_backend(conf_dev)
    t_build = time.perf_counter()
    sim = Simulation(net, conf)
    t_build = time.perf_counter() - t_build
    del net
    m = wl["m"]
    n = wl["n"]

    lib.dll.nemo_b200_timed_steps.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_double * 4]
    out = (ctypes.c_double * 4)()
    # the step kernel's work shape (threads per partition, synapses of an
    # STDP work entry), chosen by timing 100-cycle trials (simulated like any
    # other cycles) after a first warm-up step
    lib.dll.nemo_b200_autotune_shape.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.POINTER(ctypes.c_uint),
                                                 ctypes.POINTER(ctypes.c_uint), ctypes.c_double * 6]
    lib.call("nemo_b200_timed_steps", sim.handle, 1, CYCLES_PER_STEP, 1, ctypes.c_float(REWARD), out)
    tuned, tuned_run = ctypes.c_uint(), ctypes.c_uint()
    tune_ms = (ctypes.c_double * 6)()
    lib.call("nemo_b200_autotune_shape", sim.handle, CYCLES_PER_STEP, ctypes.byref(tuned), ctypes.byref(tuned_run),
             tune_ms)
    # the clock sampler runs through warm-up and the timed region, so that the
    # GPU is under the same load for every sample
    with ClockSampler(local) as clocks:
        # warm-up: W steps
        lib.call("nemo_b200_timed_steps", sim.handle, max(args.warmup, 1), CYCLES_PER_STEP, 1,
                 ctypes.c_float(REWARD), out)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        lib.call("nemo_b200_timed_steps", sim.handle, args.steps, CYCLES_PER_STEP, 1, ctypes.c_float(REWARD), out)
        torch.cuda.synchronize()
    ms, fired, events, delivered = out[0], out[1], out[2], out[3]
    if world > 1:
        t = torch.tensor([ms, events], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms_max, events_all = float(mx[0]), float(t[1])
    else:
        ms_max, events_all = ms, events
    value = events_all / (ms_max * 1e-3)

    # end to end through the C ABI (host buffers, per-cycle copies), the
    # same number of steps as the device-timed loop
    e2e_steps_n = max(1, args.steps)
    lib.dll.nemo_b200_host_bytes.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong * 2]
    bytes0 = (ctypes.c_ulonglong * 2)()
    bytes1 = (ctypes.c_ulonglong * 2)()
    lib.call("nemo_b200_host_bytes", sim.handle, bytes0)
    e2e_s, e2e_fired = e2e_steps(sim, n, e2e_steps_n, seed=11)
    lib.call("nemo_b200_host_bytes", sim.handle, bytes1)
    e2e_value = e2e_fired * m / e2e_s

    roof = roofline(sim, lib, wl)
    clk = clocks.summary()
    tr = (ctypes.c_double * 24)()
    lib.dll.nemo_b200_trace.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_double * 24]
    lib.call("nemo_b200_trace", sim.handle, CYCLES_PER_STEP, tr)
    phase_ns = dict(zip(["phase", "update_max", "update_mean", "work_max", "work_mean",
                         "to_last_arrival", "barrier_release", "arrival_spread", "after_update_max",
                         "after_update_mean", "gather_unit", "stdp_unit", "gather_units_per_block",
                         "stdp_units_per_block", "update_warp_to_model", "update_warp",
                         "fired_warp_after_lists", "fired_warps_per_block", "noise_unit",
                         "noise_units_per_block", "last_unit_taken", "warp_leaves_units",
                         "last_unit_to_end", "last_unit_end"], [round(x, 1) for x in tr]))

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64 fixed point + f32/f64 state",
        "data": "synthetic (seeded generator, numpy PCG64 seed %d)" % wl["seed"],
        "config": bench_config(wl, world),
        "sim_ms_per_wall_s": round(CYCLES_PER_STEP * args.steps / (ms_max * 1e-3), 1),
        "fired_per_cycle": round(fired / (CYCLES_PER_STEP * args.steps), 1),
        "delivered_synapses": int(delivered), "build_s": round(t_build, 2),
        "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                # counted by the library: the stimulus commands in, the
                # fired lists (pairs of fired word and warp) out
                "h2d_bytes_per_step": round((bytes1[0] - bytes0[0]) / e2e_steps_n),
                "d2h_bytes_per_step": round((bytes1[1] - bytes0[1]) / e2e_steps_n),
                "steps": e2e_steps_n, "s_per_step": round(e2e_s / e2e_steps_n, 4)},
        "roofline": roof,
        "phase_ns": phase_ns,
        "gpu_launches": args.steps * (1 + apply_launches(sim, lib)),
        "autotune": {"threads": tuned.value, "stdp_run": tuned_run.value,
                     "ms_per_cycle": {"%d/%d" % (t, r): round(tune_ms[3 * i + k], 5)
                                      for i, r in enumerate((128, 64)) for k, t in enumerate((1024, 512, 256))}},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        del sim
        v, nsteps, secs, o_build = run_oracle_steps(wl, 0, args.cpu_steps, budget_s=args.cpu_seconds)
        line["cpu_baseline"] = {"value": round(v, 1), "unit": UNIT, "cores": os.cpu_count(), "cpu_model": cpu_model(), "kind": "port",
                                "sample": "%d step(s) of 100 cycles + applyStdp from a fresh network, %.1f s, "
                                          "e2e protocol" % (nsteps, secs),
                                "build_s": round(o_build, 2)}
    if rank == 0 and world == 1 and not args.no_parity:
        line["parity"] = parity_check(wl)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = workload(args.small)
    v, nsteps, secs, build_s = run_oracle_steps(wl, args.warmup, args.steps, budget_s=args.cpu_seconds * 6)
    n = wl["n"]
    line = {
        "metric": METRIC, "value": round(v, 1), "unit": UNIT, "impl": "reference", "n_gpus": 0,
        "steps": nsteps, "warmup": args.warmup, "ms_per_step": round(secs * 1000 / nsteps, 2),
        "build_s": round(build_s, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/int64 fixed point + f32/f64 state", "data": "synthetic (seeded generator)",
        "config": bench_config(wl, 1),
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": os.cpu_count(), "cpu_model": cpu_model(), "kind": "port",
                         "sample": "%d step(s) of 100 cycles + applyStdp after %d warm-up step(s)"
                                   % (nsteps, args.warmup)},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batched(args):
    """The batched form: 256 independent Izhikevich networks (sizes
    log-uniform in [500, 20000], 100 synapses per neuron, delays U{1..20},
    per-instance seed and thalamic sigma U(3, 7) / 0.4x for inhibitory
    neurons) advanced together for 1000 cycles by one persistent kernel
    replayed from a CUDA graph, block size chosen by the autotuner; against
    the same networks run one after another with the plain step loop
    (nemo_step per cycle) and with the device-resident loop."""
    lib = Library()
    P = ctypes.POINTER
    d = lib.dll
    d.nemo_b200_new_batch.restype = ctypes.c_void_p
    d.nemo_b200_new_batch.argtypes = [P(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_void_p]
    d.nemo_b200_run_graph.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, P(ctypes.c_int)]
    d.nemo_b200_autotune.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint), ctypes.c_double * 3]
    d.nemo_b200_counters.argtypes = [ctypes.c_void_p, ctypes.c_uint64 * 4]
    d.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    d.nemo_delete_simulation.argtypes = [ctypes.c_void_p]
    import torch
    import torch.distributed as dist
    from nemo_b200.dist import shard_instances
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    count, cycles = args.batch_count, 1000
    sizes_all = netgen.batched_sizes(count, 500, 20000, seed=3)
    rng = np.random.default_rng(4)
    sig = rng.uniform(3.0, 7.0, size=count)
    # several GPUs: the networks are split over the ranks (strong scaling)
    mine = shard_instances(sizes_all, world)[rank]
    sizes = sizes_all[mine]
    specs = [netgen.izhikevich_random(int(sizes_all[j]), 100, dmax=20, seed=1000 + j, sigma_exc=float(sig[j]),
                                      sigma_inh=float(0.4 * sig[j])) for j in mine]
    count = len(mine)

    def counters(handle):
        c = (ctypes.c_uint64 * 4)()
        lib.call("nemo_b200_counters", handle, c)
        return list(c)

    nets = [spec.build(Network(lib)) for spec in specs]
    conf = Configuration(lib)
    handles = (ctypes.c_void_p * count)(*[n.handle for n in nets])
    t0 = time.perf_counter()
    batch = d.nemo_b200_new_batch(handles, count, conf.handle)
    if not batch:
        raise RuntimeError(d.nemo_strerror().decode())
    build_s = time.perf_counter() - t0
    del nets
    threads = ctypes.c_uint()
    ms = (ctypes.c_double * 3)()
    lib.call("nemo_b200_run_graph", batch, 100, 100, None)
    lib.call("nemo_b200_autotune", batch, 100, ctypes.byref(threads), ms)
    used = ctypes.c_int()
    lib.call("nemo_b200_run_graph", batch, 100, 100, ctypes.byref(used))   # warm-up, graph capture
    before = counters(batch)
    t0 = time.perf_counter()
    lib.call("nemo_b200_run_graph", batch, cycles, 100, ctypes.byref(used))
    batched_s = time.perf_counter() - t0
    events = counters(batch)[3] - before[3]
    d.nemo_delete_simulation(batch)
    if world > 1:
        t = torch.tensor([batched_s, float(events)], dtype=torch.float64, device="cuda")
        mx = t[:1].clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        batched_s, events = float(mx[0]), int(t[1])
        line = {"metric": "synaptic events/s (batched form)", "value": round(events / batched_s, 1), "unit": UNIT,
                "n_gpus": world, "scaling": "strong", "higher_is_better": True, "data": "synthetic (seeded generator)",
                "config": {"workload": "izhikevich-batch-%d-m100" % args.batch_count, "cycles": cycles,
                           "instances_per_rank": "largest first to the least loaded rank"},
                "batched": {"seconds": round(batched_s, 4), "events": events, "graph_used": bool(used.value)}}
        if rank == 0:
            print(json.dumps(line), flush=True)
        dist.destroy_process_group()
        return
    batched = events / batched_s

    # the same networks one after another
    plain_s = resident_s = 0.0
    plain_events = resident_events = 0
    fptr = P(ctypes.c_uint)()
    nf = ctypes.c_size_t()
    for spec in specs:
        for mode in ("plain", "resident"):
            net = spec.build(Network(lib))
            sim = Simulation(net, Configuration(lib))
            del net
            b0 = counters(sim.handle)
            t0 = time.perf_counter()
            if mode == "plain":
                for _ in range(cycles):
                    if d.nemo_step(sim.handle, None, 0, None, None, 0, ctypes.byref(fptr), ctypes.byref(nf)) != 0:
                        raise RuntimeError(d.nemo_strerror().decode())
            else:
                lib.call("nemo_b200_run", sim.handle, cycles, None, None)
            dt = time.perf_counter() - t0
            ev = counters(sim.handle)[3] - b0[3]
            if mode == "plain":
                plain_s += dt
                plain_events += ev
            else:
                resident_s += dt
                resident_events += ev
            del sim
    line = {
        "metric": "synaptic events/s (batched form)", "value": round(batched, 1), "unit": UNIT,
        "n_gpus": 1, "higher_is_better": True, "data": "synthetic (seeded generator)",
        "config": {"workload": "izhikevich-batch-%d-m100" % count, "instances": count,
                   "neurons": int(sizes.sum()), "synapses": int(sizes.sum()) * 100, "cycles": cycles,
                   "sizes": "log-uniform [500, 20000]", "sigma": "U(3,7) exc, 0.4x inh per instance"},
        "batched": {"seconds": round(batched_s, 4), "events": events, "graph_used": bool(used.value),
                    "threads_chosen": threads.value, "autotune_ms_per_cycle": [round(x, 5) for x in ms],
                    "build_s": round(build_s, 2)},
        "sequential_plain_step_loop": {"events_per_s": round(plain_events / plain_s, 1), "seconds": round(plain_s, 3),
                                       "events": plain_events},
        "sequential_device_resident": {"events_per_s": round(resident_events / resident_s, 1),
                                       "seconds": round(resident_s, 3), "events": resident_events},
        "speedup_vs_plain_step_loop": round(batched / (plain_events / plain_s), 2),
        "speedup_vs_device_resident": round(batched / (resident_events / resident_s), 2),
    }
    print(json.dumps(line), flush=True)


def run_bptt(args):
    """The differentiable form: BPTT gradient steps/s of a recurrent LIF
    network of 10,000 neurons (tau_m 20 ms, threshold 1, reset by
    subtraction, 1 ms Euler step), 200 recurrent synapses per neuron
    (float32 weights ~N(0, 1/sqrt(200))) and 50 synapses per neuron from 500
    Poisson input channels at 10 Hz; 32 trials of 500 steps; loss: mean
    squared error between the 10 ms-binned population rate and 20 + 10
    sin(2 pi 4 t) Hz; gradient w.r.t. all weights through the adjoint kernel
    (fast-sigmoid surrogate, slope 10, checkpoints every 50 steps)."""
    import torch
    import torch.distributed as dist
    from nemo_b200.dist import dp_grad
    from nemo_b200.lif import LIFNetwork, lif_bptt, poisson_bits, rate_loss, sinusoid_target
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    n, fan, chans, infan, steps, trials, binsteps = 10000, 200, 500, 50, 500, 32, 10
    t0 = time.perf_counter()
    net = LIFNetwork.random(n, fan, chans, infan, seed=7, checkpoint=50, bin_steps=binsteps, kappa=10.0)
    w = net.initial_weights(seed=7, scale_in=0.35).requires_grad_(True)
    # data parallel over trials: every rank runs 32 trials of its own
    bits, in_spikes = poisson_bits(steps, chans, trials, rate_hz=10.0, seed=8 + 1000 * rank)
    target = sinusoid_target(steps // binsteps, binsteps)
    build_s = time.perf_counter() - t0

    def grad_step():
        w.grad = None
        counts = lif_bptt(w, bits, net, trials)
        loss = rate_loss(counts, n, binsteps, target)
        loss.backward()
        dp_grad(w.grad, trials, trials * world)   # one all-reduce of the weight gradient
        return loss, counts

    for _ in range(max(args.warmup, 1)):
        grad_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = max(args.steps if args.steps < 100 else 10, 1)
    e0.record()
    for _ in range(k):
        loss, counts = grad_step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
    rate = counts.sum().item() / (trials * n * steps / 1000.0)
    # the forward and the adjoint alone
    from nemo_b200.lif import lif_backward, lif_forward
    wd = w.detach()
    f0, f1, b1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    f0.record()
    c2, saved = lif_forward(net, wd, bits, trials)
    f1.record()
    lif_backward(net, wd, bits, trials, saved, torch.ones_like(c2))
    b1.record()
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = f0.elapsed_time(f1), f1.elapsed_time(b1)
    line = {
        "metric": "BPTT grad steps/s", "value": round(1000.0 / ms, 3), "unit": "grad steps/s", "n_gpus": world,
        "scaling": "weak", "global_trials": trials * world,
        "steps": k, "warmup": max(args.warmup, 1), "ms_per_step": round(ms, 3), "higher_is_better": True,
        "dtype": "f32", "data": "synthetic (seeded Poisson inputs)",
        "config": {"workload": "lif-bptt-10k-200", "neurons": n, "recurrent_synapses_per_neuron": fan,
                   "input_channels": chans, "input_synapses_per_neuron": infan, "trials": trials,
                   "steps": steps, "checkpoint_every": 50, "surrogate": "1/(1+10|u-theta|)^2"},
        "loss": round(loss.item(), 3), "mean_rate_hz": round(rate, 3), "build_s": round(build_s, 2),
        "forward_ms": round(fwd_ms, 3), "backward_ms": round(bwd_ms, 3),
        "synapse_steps_per_s": round(net.synapses * trials * world * steps / (ms * 1e-3), 1),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the float64 PyTorch reference of the model (the differentiable
        # form's oracle) on the host cores: a bounded sample of the grad step
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import lif_reference as ref
        cnet = LIFNetwork.random(n, fan, chans, infan, seed=7, checkpoint=50, bin_steps=binsteps, kappa=10.0,
                                 device="cpu")
        t_s, b_s = 10, 4
        w64 = torch.tensor(w.detach().cpu().numpy().astype(np.float64), requires_grad=True)
        c0 = time.perf_counter()
        c = ref.counts(cnet, w64, in_spikes[:t_s], b_s)
        rate_loss(c, n, binsteps, target.cpu().double()[:t_s // binsteps]).backward()
        secs = time.perf_counter() - c0
        scale = (steps / t_s) * (trials / b_s)
        line["cpu_baseline"] = {"value": round(1.0 / (secs * scale), 8), "unit": "grad steps/s",
                                "cores": torch.get_num_threads(), "cpu_model": cpu_model(), "kind": "port",
                                "sample": "float64 PyTorch reference (autograd, surrogate gradient), %d of %d trials x "
                                          "%d of %d steps in %.2f s, scaled linearly to the full grad step"
                                          % (b_s, trials, t_s, steps, secs)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_random1k(args):
    """The 1000-neuron benchmark network (800 excitatory / 200 inhibitory
    Izhikevich neurons with thalamic noise sigma 5 / 2, 100 synapses per
    neuron, delays U{1..20}, no STDP), 1000 cycles: device-resident (one
    persistent launch per 1000 cycles, CUDA events) and through nemo_step
    per cycle; the oracle on the host cores runs the same 1000 cycles, and
    the per-cycle firing counts must agree."""
    lib = Library()
    spec = netgen.izhikevich_random(1000, 100, dmax=20, seed=1)
    cycles = 1000
    P = ctypes.POINTER
    outdeg = spec.out_degree()

    def step_run(sim_lib, sim):
        """nemo_step per cycle; each cycle's fired list is copied out of the
        call's array (memmove) in the timed loop, its events counted after"""
        fptr = P(ctypes.c_uint)()
        nf = ctypes.c_size_t()
        counts = []
        buf = np.zeros(cycles * spec.neuron_count, np.uint32)
        base = buf.ctypes.data
        fref, nref = ctypes.byref(fptr), ctypes.byref(nf)
        step = sim_lib.dll.nemo_step
        h = sim.handle
        pos = 0
        t0 = time.perf_counter()
        for _ in range(cycles):
            if step(h, None, 0, None, None, 0, fref, nref) != 0:
                raise RuntimeError(sim_lib.dll.nemo_strerror().decode())
            n = nf.value
            if n:
                ctypes.memmove(base + 4 * pos, fptr, 4 * n)
            pos += n
            counts.append(n)
        secs = time.perf_counter() - t0
        return secs, counts, int(outdeg[buf[:pos]].sum())

    net = spec.build(Network(lib))
    sim = Simulation(net, Configuration(lib))
    lib.dll.nemo_b200_host_bytes.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong * 2]
    bus = (ctypes.c_ulonglong * 2)()
    e2e_s, e2e_counts, e2e_events = step_run(lib, sim)
    lib.call("nemo_b200_host_bytes", sim.handle, bus)
    # device-resident: fresh simulations, K timed launches of 1000 cycles after W
    lib.dll.nemo_b200_timed_steps.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_double * 4]
    out = (ctypes.c_double * 4)()
    sim2 = Simulation(spec.build(Network(lib)), Configuration(lib))
    lib.call("nemo_b200_timed_steps", sim2.handle, max(args.warmup, 1), cycles, 0, ctypes.c_float(0), out)
    lib.call("nemo_b200_timed_steps", sim2.handle, max(args.steps, 1), cycles, 0, ctypes.c_float(0), out)
    ms, events = out[0], out[2]
    k = max(args.steps, 1)
    line = {"metric": "synaptic events/s (1000-neuron network)", "value": round(events / (ms * 1e-3), 1),
            "unit": UNIT, "n_gpus": 1, "steps": k, "warmup": max(args.warmup, 1),
            "ms_per_step": round(ms / k, 4), "higher_is_better": True,
            "dtype": "int32/int64 fixed point + f32/f64 state", "data": "synthetic (seeded generator)",
            "config": {"workload": "izhikevich-1k-m100", "neurons": 1000, "synapses": 100000,
                       "cycles_per_step": cycles, "noise": "sigma 5 / 2"},
            "sim_ms_per_wall_s": round(cycles * k / (ms * 1e-3), 1),
            "e2e": {"value": round(e2e_events / e2e_s, 1), "unit": UNIT, "sim_ms_per_wall_s": round(cycles / e2e_s, 1),
                    # counted by the library over the 1000 calls (the step)
                    "h2d_bytes_per_step": int(bus[0]), "d2h_bytes_per_step": int(bus[1])}}
    if not args.no_cpu_baseline:
        ol = Library(oracle_library())
        oconf = Configuration(ol)
        oconf.set_cpu_backend()
        osim = Simulation(spec.build(Network(ol)), oconf)
        o_s, o_counts, o_events = step_run(ol, osim)
        line["cpu_baseline"] = {"value": round(o_events / o_s, 1), "unit": UNIT, "cores": os.cpu_count(),
                                "kind": "port", "sample": "the same 1000 cycles, %.2f s" % o_s,
                                "sim_ms_per_wall_s": round(cycles / o_s, 1),
                                "firing_counts_equal": o_counts == e2e_counts}
    print(json.dumps(line), flush=True)


def run_mixed(args):
    """The mixed-plugin network: 50,000 neurons (20k Izhikevich RS/FS with no
    noise, 15k IF_curr_exp, 10k QIF, 5k Hodgkin-Huxley), 500 synapses per
    neuron across all populations, delays U{1..10}, weights 0.3 U (excitatory)
    / -0.6 U (inhibitory Izhikevich sources); Poisson input at 5 Hz per neuron
    as firing stimulus through nemo_step, one Bernoulli(0.005) draw per neuron
    per cycle, seeded. Timed through the C ABI (stimulus copied in, fired list
    copied out every cycle). The reference CPU restatement runs the first
    cycles of the same run within a time budget; its per-cycle event counts
    must equal the GPU's (bit-exact firing at full size), and the GPU's time
    over those same cycles is reported beside it."""
    lib = Library()
    spec = netgen.mixed_plugins(seed=2)
    n = spec.neuron_count
    cycles = args.mixed_cycles
    rng = np.random.default_rng(5)
    stim = [np.nonzero(rng.random(n) < 0.005)[0].astype(np.uint32) for _ in range(cycles)]
    outdeg = spec.out_degree()
    P = ctypes.POINTER

    def run(sim_lib, sim, count, budget_s=None):
        """per-cycle (seconds, events), stopping early past budget_s; the
        fired lists are copied out in the timed loop and counted after"""
        fptr = P(ctypes.c_uint)()
        nf = ctypes.c_size_t()
        fref, nref = ctypes.byref(fptr), ctypes.byref(nf)
        step = sim_lib.dll.nemo_step
        h = sim.handle
        args = [(f.ctypes.data_as(P(ctypes.c_uint)), f.size) for f in stim[:count]]
        times, lists = [], []
        t_start = time.perf_counter()
        for c in range(count):
            fp, fn = args[c]
            t0 = time.perf_counter()
            if step(h, fp, fn, None, None, 0, fref, nref) != 0:
                raise RuntimeError(sim_lib.dll.nemo_strerror().decode())
            out = np.empty(nf.value, np.uint32)
            if nf.value:
                ctypes.memmove(out.ctypes.data, fptr, 4 * nf.value)
            t1 = time.perf_counter()
            times.append(t1 - t0)
            lists.append(out)
            if budget_s is not None and t1 - t_start > budget_s:
                break
        return [(dt, int(outdeg[f].sum())) for dt, f in zip(times, lists)]

    net = spec.build(Network(lib))
    sim = Simulation(net, Configuration(lib))
    del net
    run(lib, sim, min(50, cycles))            # warm-up run on its own copy of the network
    net = spec.build(Network(lib))
    sim2 = Simulation(net, Configuration(lib))
    del net, sim
    per = run(lib, sim2, cycles)
    secs = sum(p[0] for p in per)
    events = sum(p[1] for p in per)
    line = {"metric": "synaptic events/s (mixed plugins)", "value": round(events / secs, 1), "unit": UNIT,
            "n_gpus": 1, "higher_is_better": True, "data": "synthetic (seeded generator, seeded Poisson stimulus)",
            "dtype": "int32/int64 fixed point + f32/f64 state",
            "config": {"workload": "mixed-50k-m500", "neurons": n, "synapses": spec.synapse_count,
                       "populations": "20k Izhikevich, 15k IF_curr_exp, 10k QIF, 5k HH", "cycles": cycles,
                       "stimulus": "Bernoulli(0.005) firing stimulus per neuron per cycle"},
            "sim_ms_per_wall_s": round(cycles / secs, 2), "seconds": round(secs, 3), "events": events,
            "fired_per_cycle": round(events / cycles / (spec.synapse_count / n), 1)}
    if not args.no_cpu_baseline:
        ol = Library(oracle_library())
        net = spec.build(Network(ol))
        conf = Configuration(ol)
        conf.set_cpu_backend()
        osim = Simulation(net, conf)
        del net
        oper = run(ol, osim, cycles, budget_s=args.cpu_seconds)
        k = len(oper)
        osecs = sum(p[0] for p in oper)
        oev = sum(p[1] for p in oper)
        gsecs = sum(p[0] for p in per[:k])
        line["cpu_baseline"] = {"value": round(oev / osecs, 1), "unit": UNIT, "cores": os.cpu_count(), "cpu_model": cpu_model(), "kind": "port",
                                "sample": "first %d cycles of the same run, %.1f s" % (k, osecs),
                                "sim_ms_per_wall_s": round(k / osecs, 3),
                                "gpu_same_cycles": round(oev / gsecs, 1),
                                "events_equal": [p[1] for p in oper] == [p[1] for p in per[:k]]}
    print(json.dumps(line), flush=True)


def run_sharded(args):
    """One network over all ranks (--sharded under torchrun): the
    1e8-synapse STDP network as N shards (ShardedSimulation), one per GPU,
    each owning a contiguous range of the neuron warps and the synapses to
    them; every cycle the shards' fired words are all-gathered (NCCL) and
    delivered, and applyStdp runs every 100 cycles (strong scaling). The
    words stay in device memory (step_device: the step, the all-gather of
    CUDA tensors and the delivery are queued on the GPU without waiting on
    the host); --host-exchange takes them through host memory instead,
    every cycle host-synchronous. Time: CUDA events on the current stream,
    which waits for the shard's work at the end, max over ranks; events are
    the shards' device counters summed over ranks."""
    import torch
    import torch.distributed as dist
    from nemo_b200.nemo import ShardedSimulation

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    wl = workload(args.small)
    lib = Library()
    spec = netgen.izhikevich_random(wl["n"], wl["m"], dmax=wl["dmax"], seed=wl["seed"], stdp=True)
    net = spec.build(Network(lib))
    conf = Configuration(lib)
    pre, post = netgen.standard_stdp()
    conf.set_stdp_function(pre, post, 0.0, 1.0, 0.0, -1.0)
    conf.set_write_only_synapses()
    conf.set_cuda_backend(local)
    sim = ShardedSimulation(net, conf, rank, world)
    del net
    lib.dll.nemo_b200_counters.argtypes = [ctypes.c_void_p, ctypes.c_uint64 * 4]
    counters = (ctypes.c_uint64 * 4)()

    def steps(k):
        for _ in range(k):
            for _ in range(CYCLES_PER_STEP):
                if args.host_exchange:
                    sim.step()
                else:
                    sim.step_device()
            sim.apply_stdp(REWARD)

    steps(max(args.warmup, 1))
    sim.stream_wait()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lib.call("nemo_b200_counters", sim.handle, counters)
    ev0 = counters[3]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    steps(args.steps)
    sim.stream_wait()
    e1.record()
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) * 1e-3
    lib.call("nemo_b200_counters", sim.handle, counters)
    events = float(counters[3] - ev0)
    if world > 1:
        t = torch.tensor([secs, events], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        secs, events = float(mx[0]), float(t[1])
    launches = args.steps * (CYCLES_PER_STEP * (1 + (1 if world > 1 else 0)) + 1 + apply_launches(sim, lib))
    line = {"metric": METRIC, "value": round(events / secs, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs * 1e3 / args.steps, 4),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "int32/int64 fixed point + f32/f64 state",
            "data": "synthetic (seeded generator, numpy PCG64 seed %d)" % wl["seed"],
            "config": {"workload": wl["name"], "neurons": wl["n"], "synapses": wl["n"] * wl["m"],
                       "parallelism": "shards%d" % world, "cycles_per_step": CYCLES_PER_STEP,
                       "exchange": "all-gather of the fired words every cycle, "
                                   + ("through host memory" if args.host_exchange else "in device memory")},
            "timing": "CUDA events on the current stream, which waits for the shard's work, max over ranks",
            "sim_ms_per_wall_s": round(CYCLES_PER_STEP * args.steps / secs, 1),
            "gpu_launches": launches}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_ncu_case(args):
    """A bounded case for ncu: the workload (--small: the 20k-neuron one)
    built, --warmup steps of 100 cycles + applyStdp, then --steps more, all
    through nemo_b200_timed_steps; k_cycles launches: warmup + steps, each
    followed by the applyStdp launches. Prints the device time of the last
    steps. With --batched: the 256 networks of the batched form, warmup +
    steps launches of 100 cycles. With --bptt: the differentiable form's
    configuration, warmup + steps forward and adjoint passes."""
    if args.batched:
        return _ncu_case_batched(args)
    if args.bptt:
        return _ncu_case_bptt(args)
    wl = workload(args.small)
    lib = Library()
    sim, _, build_s = build_sim(lib, wl)
    lib.dll.nemo_b200_timed_steps.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_double * 4]
    out = (ctypes.c_double * 4)()
    lib.call("nemo_b200_timed_steps", sim.handle, max(args.warmup, 1), CYCLES_PER_STEP, 1, ctypes.c_float(REWARD), out)
    lib.call("nemo_b200_timed_steps", sim.handle, max(args.steps, 1), CYCLES_PER_STEP, 1, ctypes.c_float(REWARD), out)
    print(json.dumps({"case": wl["name"], "steps": max(args.steps, 1), "warmup": max(args.warmup, 1),
                      "ms_per_step": round(out[0] / max(args.steps, 1), 4), "build_s": round(build_s, 2),
                      "apply_launches_per_step": apply_launches(sim, lib)}), flush=True)


def _ncu_case_batched(args):
    from nemo_b200.netgen import batched_sizes
    lib = Library()
    d = lib.dll
    d.nemo_b200_new_batch.restype = ctypes.c_void_p
    d.nemo_b200_new_batch.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_void_p]
    d.nemo_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p]
    count = args.batch_count
    sizes = batched_sizes(count, 500, 20000, seed=3)
    sig = np.random.default_rng(4).uniform(3.0, 7.0, size=count)
    nets = [netgen.izhikevich_random(int(sizes[j]), 100, dmax=20, seed=1000 + j, sigma_exc=float(sig[j]),
                                     sigma_inh=float(0.4 * sig[j])).build(Network(lib)) for j in range(count)]
    handles = (ctypes.c_void_p * count)(*[n.handle for n in nets])
    conf = Configuration(lib)
    batch = d.nemo_b200_new_batch(handles, count, conf.handle)
    if not batch:
        raise RuntimeError(d.nemo_strerror().decode())
    del nets
    t0 = time.perf_counter()
    for _ in range(max(args.warmup, 1) + max(args.steps, 1)):
        lib.call("nemo_b200_run", batch, CYCLES_PER_STEP, None, None)
    print(json.dumps({"case": "izhikevich-batch-%d-m100" % count, "launches": max(args.warmup, 1) + max(args.steps, 1),
                      "seconds": round(time.perf_counter() - t0, 3)}), flush=True)
    d.nemo_delete_simulation.argtypes = [ctypes.c_void_p]
    d.nemo_delete_simulation(batch)


def _ncu_case_bptt(args):
    import torch
    from nemo_b200.lif import LIFNetwork, lif_backward, lif_forward, poisson_bits
    n, fan, chans, infan, steps, trials = (2000, 200, 500, 50, 100, 32) if args.small else (10000, 200, 500, 50, 500, 32)
    net = LIFNetwork.random(n, fan, chans, infan, seed=7, checkpoint=50, bin_steps=10, kappa=10.0)
    w = net.initial_weights(seed=7, scale_in=0.35)
    bits, _ = poisson_bits(steps, chans, trials, rate_hz=10.0, seed=8)
    for _ in range(max(args.warmup, 1) + max(args.steps, 1)):
        counts, saved = lif_forward(net, w, bits, trials)
        lif_backward(net, w, bits, trials, saved, torch.ones_like(counts))
    torch.cuda.synchronize()
    print(json.dumps({"case": "lif-bptt-%dk-200" % (n // 1000), "passes": max(args.warmup, 1) + max(args.steps, 1)}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--small", action="store_true", help="20k-neuron variant (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison of the headline workload")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--batched", action="store_true",
                    help="measure the batched form (256 networks) instead of the headline workload")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--bptt", action="store_true",
                    help="measure the differentiable form (BPTT grad steps/s) instead of the headline workload")
    ap.add_argument("--random1k", action="store_true",
                    help="measure the 1000-neuron benchmark network (no STDP)")
    ap.add_argument("--sharded", action="store_true",
                    help="one network over all ranks as shards (fired words all-gathered every cycle)")
    ap.add_argument("--host-exchange", action="store_true",
                    help="--sharded: exchange the fired words through host memory")
    ap.add_argument("--mixed", action="store_true",
                    help="measure the mixed-plugin network (nemo_step with Poisson stimulus)")
    ap.add_argument("--mixed-cycles", type=int, default=5000)
    ap.add_argument("--ncu-case", action="store_true",
                    help="a bounded run of the headline (or --small) workload for ncu captures")
    args = ap.parse_args()
    if args.ncu_case:
        run_ncu_case(args)
    elif args.random1k:
        run_random1k(args)
    elif args.sharded:
        run_sharded(args)
    elif args.mixed:
        run_mixed(args)
    elif args.bptt:
        run_bptt(args)
    elif args.batched:
        run_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
