"""The JSON line bench.py prints, for both arms, at tiny scale: every key the
measurement contract names, with the right types and relations."""
import json
import os
import subprocess
import sys

import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args, timeout=600):
    out = subprocess.run([sys.executable, os.path.join(HERE, "bench.py"), *args],
                         capture_output=True, text=True, timeout=timeout, cwd=HERE)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


BASE_KEYS = {"metric": str, "value": float, "unit": str, "n_gpus": int, "steps": int,
             "warmup": int, "ms_per_step": float, "higher_is_better": bool, "scaling": str,
             "dtype": str, "data": str, "config": dict, "e2e": dict}


def _check_base(d):
    for k, t in BASE_KEYS.items():
        assert isinstance(d[k], t), (k, d.get(k))
    assert "vs_baseline" in d and d["vs_baseline"] is None  # no published number
    assert d["higher_is_better"] is True and d["scaling"] in ("weak", "strong")
    assert isinstance(d["config"]["workload"], str)
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in d["e2e"], k


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_line():
    d = _run("--impl", "reference", "--scale", "0.01", "--steps", "1", "--warmup", "0",
             "--cpu-queries", "200")
    _check_base(d)
    assert d["impl"] == "reference"
    cb = d["cpu_baseline"]
    assert set(cb) >= {"value", "unit", "cores", "kind", "sample"}
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    # e2e: exhaustive-equivalent pairs per second of a full result, the unit
    # of the GPU arm's e2e
    assert d["e2e"]["unit"] == "all-pairs-equivalent pairs/s" and d["e2e"]["value"] > 0
    assert d["e2e"]["s_per_full_result"] == d["s_per_full_result"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the same config object the GPU arm prints for this workload and rank count
    import bench
    assert d["config"] == bench._config(bench.WORKLOADS["clustered3d"](0.01), 1)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_under_torchrun_prints_once(tmp_path):
    """Launched like the multi-GPU runs (torchrun, 2 ranks): rank 0 alone
    runs the CPU reference and prints one line; the other rank exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = subprocess.run(
        [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
         "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
         "reference", "--gpus", "2", "--scale", "0.01", "--steps", "1", "--warmup", "0",
         "--cpu-queries", "200"],
        capture_output=True, text=True, timeout=600, cwd=HERE,
        env={**os.environ, "TMPDIR": str(tmp_path)})  # torchrun's scratch stays here
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    _check_base(d)
    assert d["impl"] == "reference" and d["n_gpus"] == 2


@pytest.mark.gpu
def test_gpu_arm_line():
    d = _run("--scale", "0.01", "--steps", "1", "--warmup", "3", "--cpu-queries", "200")
    _check_base(d)
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3
    assert d["counts_exact_mixed_vs_fp64"] is True
    r = d["roofline"]
    assert r["bound"] == "fp32" and r["unit"] == "TFLOP/s" and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9 and r["traffic"] > 0
    e = d["e2e"]
    assert e["unit"] == "all-pairs-equivalent pairs/s" and e["value"] > 0
    assert e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert e["s_per_full_result"] > 0 and d["s_per_full_result"] > 0
    assert d["fp64_form"]["roofline"]["peak"] > 0
    c = d["clocks"]
    assert set(c) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert isinstance(d["gpu_launches"], int) and d["gpu_launches"] >= 3
    cb = d["cpu_baseline"]
    assert set(cb) >= {"value", "unit", "cores", "kind", "sample"}
    assert cb["gpu_counts_equal_reference_on_sample"] is True
