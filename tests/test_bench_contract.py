"""The benchmark's JSON line: both arms print one line with the keys and types
that their readers rely on.  The reference arm (the CPU oracle port on the host
cores) runs anywhere; the CUDA arm needs a B200."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COMMON = {"metric": str, "value": float, "unit": str, "n_gpus": int, "steps": int, "warmup": int,
          "ms_per_step": float, "higher_is_better": bool, "scaling": str, "dtype": str, "data": str,
          "config": dict, "cpu_baseline": dict, "e2e": dict}


def _line(args, timeout):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=timeout, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def _check_common(d):
    for k, t in COMMON.items():
        assert k in d, k
        assert isinstance(d[k], t) or (t is float and isinstance(d[k], int)), (k, d[k])
    assert d["value"] > 0 and d["cpu_baseline"]["value"] > 0
    assert set(d["cpu_baseline"]) >= {"value", "unit", "cores", "kind", "sample"}
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert set(d["e2e"]) >= {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert "workload" in d["config"] and "vs_baseline" in d


def test_reference_arm_line():
    d = _line(["--impl", "reference", "--steps", "1", "--warmup", "3"], timeout=600)
    _check_common(d)
    assert d["impl"] == "reference"
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1


@pytest.mark.gpu
def test_cuda_arm_line():
    d = _line(["--steps", "3", "--warmup", "3"], timeout=900)
    _check_common(d)
    assert "impl" not in d and d["n_gpus"] == 1 and d["steps"] == 3 and d["device_status"] == 0
    rf = d["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and 0 < rf["frac"] < 1.5
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-9
    assert d["gpu_launches"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    assert set(d["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert d["closure"].get("status") == 0, d["closure"]
