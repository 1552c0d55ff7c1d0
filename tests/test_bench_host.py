"""Host-side logic of bench.py: the clock record's summary, the reference
arm's JSON line and its behaviour on ranks other than 0 (no GPU needed)."""
import importlib.util
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_summary_median_and_reasons(tmp_path, monkeypatch):
    """nvidia-smi csv rows (index, sm, max sm, power, active mask, then the
    four reasons): the median SM clock, the maximum, and every reason seen
    Active at least once; malformed rows are skipped."""
    path = tmp_path / "clocks.csv"
    rows = [
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1900, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "short row",
    ]
    path.write_text("\n".join(rows) + "\n")
    monkeypatch.setenv("NEMO_B200_CLOCKS_CSV", str(path))
    b = _bench()
    c = b.ClockSampler(0)
    c.proc = object()   # as if nvidia-smi had run
    s = c.summary()
    assert s == {"sm_mhz": 1900.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert path.exists()   # a named record is kept


def test_clock_sampler_without_nvidia_smi(monkeypatch):
    """Without nvidia-smi the sampler reports nothing and leaves no file."""
    monkeypatch.delenv("NEMO_B200_CLOCKS_CSV", raising=False)
    monkeypatch.setenv("PATH", "/nonexistent")
    b = _bench()
    with b.ClockSampler(0) as c:
        pass
    assert c.summary() is None
    assert not os.path.exists(c.path)


def _run(args, env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_other_ranks_exit_silently():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0
    without output."""
    r = _run(["--impl", "reference", "--gpus", "2"], {"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line():
    """One bounded oracle step of the 20k-neuron workload: one JSON line with
    the contract's keys, its cpu_baseline and e2e equal to its value."""
    r = _run(["--impl", "reference", "--small", "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"],
             {"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["build_s"] > 0
    assert line["config"]["workload"] == "izhikevich-20k-m1000-stdp"
    assert line["config"]["synapses"] == 20000 * 1000
    assert "160 MB" in line["config"]["l2"]
