"""The reference arm of bench.py on the host: the reference's own CPU FFT
(oracle/_ref, built from the reference's sources) timed on the box's cores,
printed as the same one-line JSON contract as the GPU arm."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
import oracle as O  # noqa: E402

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_cpu_reference_sample_describes_itself():
    cb = bench.C2Sweep().cpu_reference(budget_s=1.5)
    assert cb["kind"] == "reference" and cb["unit"] == "GB/s"
    assert cb["value"] > 0 and cb["cores"] >= 1
    assert "oracle/_ref" in cb["sample"]


@needs_ref
def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "c1", "--steps",
                        "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GB/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("C1")
