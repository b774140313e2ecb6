"""bench.py's reference arm (the reference's own CPU reply on the host cores, or the oracle
port where the reference is not built) prints one JSON line in the bench contract: the
metric and unit of the GPU arm, a cpu_baseline block and an e2e block without host-device
traffic. Runs on a small sample so that it needs no GPU and a few seconds."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def run_reference_arm(*extra: str) -> dict:
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", *extra], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_reference_arm_line_follows_the_contract():
    d = run_reference_arm("--elements", "2000")
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["unit"] == "GB/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].startswith("memory-bound") and d["config"]["elements_timed"] == 2000
    assert d["config"]["same_config"] is True  # every element of the (here reduced) workload is timed
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["cpu_model"] and len(d["reply_s"]) == d["steps"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_query_generation_reference_arm():
    from oracle import pyoracle as po

    d = run_reference_arm("--workload", "querygen", "--elements", "3000")
    if not po.ref_available():
        assert "unavailable" in d
        return
    assert d["impl"] == "reference" and d["unit"] == "ciphertexts/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert "3000 ciphertexts" in d["config"]["workload"]


def test_extraction_reference_arm():
    from oracle import pyoracle as po

    d = run_reference_arm("--workload", "extract", "--elements", "2000000")
    if not po.ref_available():
        assert "unavailable" in d
        return
    assert d["impl"] == "reference" and d["unit"] == "ciphertexts/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["config"]["reply_ciphertexts"] > 0
