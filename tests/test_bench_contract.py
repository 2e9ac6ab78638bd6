"""bench.py's reference arm keeps the JSON contract the measurement relies on:
one line with the headline metric, its unit and direction, the run's shape,
the CPU baseline block and an end-to-end block with no host-device bytes.
The arm times the reference's own CPU twin (oracle/_ref), so it runs here
without a GPU; skipped when that build is absent.  CPU only."""
import json
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    if not (ROOT / "oracle" / "_ref" / "libref_probe.so").exists():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--cpu-budget", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "lp_adam_batched_steps_per_s" and d["unit"] == "steps/s"
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 1, 3)
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["n"] == 8400 and d["config"]["global_batch"] == 256
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
