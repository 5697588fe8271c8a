"""bench.py's one JSON line: the reference arm on the CPU (one rank, and two ranks under
torchrun, where rank 0 alone prints), and this library's arm on the GPU, on the 1K workload."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BASE_KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
             "vs_baseline", "dtype", "data", "config")


def _json_lines(cmd, env=None, timeout=600):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=ROOT,
                       env={**os.environ, **(env or {})})
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _check_reference_line(d, n_gpus):
    for k in BASE_KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["n_gpus"] == n_gpus and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_line():
    lines = _json_lines([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                         "--workload", "0"])
    assert len(lines) == 1
    _check_reference_line(lines[0], 1)


def test_reference_arm_line_2d():
    lines = _json_lines([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                         "--workload", "5", "--n", "2048"])
    assert len(lines) == 1
    _check_reference_line(lines[0], 1)
    assert "2d" in lines[0]["config"]["workload"]


def test_reference_arm_two_ranks_print_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "2", "--warmup", "1", "--workload", "0"]
    lines = _json_lines(cmd)
    assert len(lines) == 1
    _check_reference_line(lines[0], 2)


def test_gpu_local_cpus_without_a_device():
    """The e2e placement helper reads NVML only; without a device (or NVML) it returns no CPUs, so
    the measurement keeps the process's own affinity instead of failing."""
    sys.path.insert(0, ROOT)
    import bench
    cpus = bench.gpu_local_cpus(0)
    assert isinstance(cpus, set)
    assert cpus <= os.sched_getaffinity(0)


@pytest.mark.gpu
def test_bench_line_on_gpu():
    lines = _json_lines([sys.executable, "bench.py", "--steps", "3", "--warmup", "3", "--workload", "0"])
    assert len(lines) == 1
    d = lines[0]
    for k in BASE_KEYS:
        assert k in d, k
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] >= 3
    assert "workload" in d["config"] and "l2" in d["config"]
    rf = d["roofline"]
    assert rf["bound"] and rf["achieved"] > 0 and rf["peak"] > 0 and rf["unit"]
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) <= 1e-9 * rf["frac"]
    assert "traffic" in rf
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["unit"] == d["unit"] and e2e["h2d_bytes_per_step"] > 0
    assert e2e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    assert set(d["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] > 0
    acc = d["accuracy"]
    assert acc["E_rel_err"] <= acc["tolerance"]["E"] and acc["grad_rel_err"] <= acc["tolerance"]["grad"]
    assert d["plain_fd"]["adjoint_speedup"] > 1


@pytest.mark.gpu
def test_configs_entry_on_gpu(tmp_path):
    """One entry of the default run's `configs` key (the 1K sphere): device timing, roofline,
    error against the FP64 oracle within the contract, and a clock record."""
    sys.path.insert(0, ROOT)
    import bench
    from dugma_b200 import _lib, synth
    ent = bench.config_single(_lib.load(), "cfg0", synth.workload0(), 0, 36.0e12, steps=3, clock_dir=str(tmp_path))
    assert ent["ms_per_step"] > 0 and ent["pair_terms_per_s"] > 0 and ent["steps"] == 3 and ent["warmup"] >= 3
    assert 0 < ent["roofline"]["frac"] and ent["roofline"]["kernel_ms"] > 0
    acc = ent["accuracy"]
    assert acc["rows"] == 1000
    assert acc["E_rel_err"] <= acc["tolerance"]["E"] and acc["grad_rel_err"] <= acc["tolerance"]["grad"]
    assert set(ent["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
