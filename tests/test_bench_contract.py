"""The bench's JSON-line contract, on the CPU.

- The reference arm (`--impl reference`) times the reference's own CPU PDHG,
  one step being every case of the stack solved once, and prints one JSON
  line with the keys the contract names: impl, metric,
  value, unit, n_gpus, steps, warmup, ms_per_step, higher_is_better,
  scaling, vs_baseline, dtype, data, config (with the workload),
  cpu_baseline (value, unit, cores, kind, sample) and e2e (value, unit and
  zero transfer bytes).
- The engine arm has no CPU path: without a device it exits non-zero and
  prints no result line.
"""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                          capture_output=True, text=True, timeout=timeout, cwd=ROOT)


@pytest.mark.skipif(not oracle.have_reference(), reason="oracle/_ref not built")
def test_reference_arm_line():
    p = _bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--no-gpu-reference")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "refinery_case_stack"
    # A step solves the whole stack once; ms_per_step is its measured time.
    assert d["ms_per_step"] == pytest.approx(1e3 * d["cases_optimal"] / d["value"], rel=1e-9)
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "reference" and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_engine_arm_fails_loudly_without_device():
    from anukulan_b200 import pdhg
    if pdhg.device_count() > 0:
        pytest.skip("a device is present")
    p = _bench("--steps", "1", "--warmup", "0", "--no-side", "--no-cpu-baseline")
    assert p.returncode != 0
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
