"""bench.py's reference arm (the CPU explicit DFT, no GPU needed) prints the one
JSON line of the measurement contract: metric, value and unit, the step
bookkeeping, a cpu_baseline record and an e2e record with no host<->device
bytes."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--npix", "256", "--nrow", "2000", "--nchan", "1", "--cpu-seconds", "2"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "vis/s" and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_both_arms_describe_the_same_config():
    """The reference arm's config is the one the GPU arm prints for the same
    arguments (a function of the arguments only), and its ms_per_step is the
    measured sample, not the extrapolation."""
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--npix", "256", "--nrow", "2000", "--nchan", "4", "--cpu-seconds", "2"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    a = argparse.Namespace(nrow=2000, nchan=4, npix=256, fov=3.0, eps=1e-5, window="auto", precision="fp32",
                           accumulate=0)
    assert d["config"] == bench.bench_config(a, 1)
    assert d["ms_per_step"] < 60_000 and d["extrapolated_ms_per_step"] > 0
