"""The C++ drop-in headers (include/pcxo/*.hpp): a program written against
the reference's API (fft_unit, ifft, fft_raw, fxcorr_unit, pcxo::vector,
std::vector<std::complex>) is compiled with g++ against libpcx_cuda.so and run
on the GPU.  The compile step alone runs on CPU."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "test_dropin.cpp"
CUDA = Path("/usr/local/cuda")


def _compile(out: Path) -> None:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    lib = ROOT / "packed_b200"
    cmd = [gxx, "-std=c++20", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(SRC),
           "-o", str(out), f"-L{lib}", "-lpcx_cuda", f"-L{CUDA / 'lib64'}", "-lcudart", f"-Wl,-rpath,{lib}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_dropin_headers_compile(tmp_path):
    _compile(tmp_path / "test_dropin")


@pytest.mark.gpu
def test_dropin_program_runs_on_gpu(tmp_path):
    exe = tmp_path / "test_dropin"
    _compile(exe)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
