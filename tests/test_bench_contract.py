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


def test_clock_summary_keeps_the_timed_window():
    """Clock samples are summarised over the marked timed region; a region
    shorter than the sampling interval takes the next sample after it; a
    throttle reason seen in the window is reported (idle is not a reason)."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0)
    c.samples = [(0.0, 1200.0, 1965.0, 0x1), (1.0, 1965.0, 1965.0, 0x0), (1.5, 1965.0, 1965.0, 0x4),
                 (3.0, 1500.0, 1965.0, 0x20)]
    c.mark(0.9, 2.0)
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1965.0 and s["reasons"] == ["sw_power_cap"]
    c.mark(2.1, 2.2)
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1500.0 and s["reasons"] == ["sw_thermal_slowdown"]
    c.samples = []
    assert c.summary()["reasons"] == ["unsampled"]
