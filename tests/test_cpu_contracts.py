"""CPU-side checks of the two things a caller builds on without a GPU:

* the drop-in shim (reference signatures over the C ABI) compiles and links
  against the library for a reference params configuration;
* `bench.py --impl reference` (the reference's own CPU join, timed on the host)
  prints one JSON line with the keys the benchmark contract names.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_compat_shim_builds():
    p = subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "compat"), "CFG=cpu_d6", "D=6", "K=6", "T=float"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert os.path.exists(os.path.join(ROOT, "_build", "compat", "cpu_d6", "compat_main"))


def test_reference_arm_line():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ref-seconds", "1"], capture_output=True, text=True, timeout=900,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "steps", "warmup", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["unit"] == "pairs/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "c2_18d"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
