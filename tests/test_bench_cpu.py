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


def test_correlation_fft_size_model():
    """The ragged batch's FFT size per correlation: a power of two with room
    for the kernel, minimising 2 N log2 N / (N - k + 1), at most 8192 unless
    the kernel has more than 4096 taps."""
    from packed_b200 import correlation_fft_size as f
    for k in (1, 64, 100, 700, 3000, 4096, 4097, 8192, 16377):
        n = f(k)
        assert n & (n - 1) == 0 and n >= k + 7 and 128 <= n <= 16384
        assert n <= 8192 or k > 4096
        cost = 2 * n * (n.bit_length() - 1) / (n - k + 1)
        for m in (128 << i for i in range(8)):
            if m >= k + 7 and (m <= 8192 or k > 4096):
                assert cost <= 2 * m * (m.bit_length() - 1) / (m - k + 1) + 1e-12
    import pytest
    with pytest.raises(ValueError):
        f(16378)
