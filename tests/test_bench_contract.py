"""The bench's JSON line contract, checked on the reference arm (the CPU
oracle of the shader passes, which needs no GPU), and the product arm failing
loudly where there is no GPU rather than falling back to the CPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                          text=True, timeout=timeout)


def test_reference_arm_line():
    r = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["metric"] == "cell-updates/s" and line["unit"] == "cell-updates/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert "workload" in line["config"]


def _gpu_present():
    import torch
    return torch.cuda.is_available()


@pytest.mark.skipif(_gpu_present(), reason="a GPU is present")
def test_product_arm_fails_without_gpu():
    r = run_bench("--steps", "1", "--warmup", "1", "--no-cpu", timeout=300)
    assert r.returncode != 0
    assert not r.stdout.strip() or "value" not in r.stdout
