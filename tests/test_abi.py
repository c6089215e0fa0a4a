"""The C-ABI library: it loads, exports every symbol include/*.h declares, and
rejects invalid plans exactly as the reference's constructor does (checks that
run before any device work).  CPU only."""
import ctypes
import re
from pathlib import Path

import pytest

from packed_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms |= set(re.findall(r"\b(pcx_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    syms = declared_symbols()
    assert {"pcx_plan_create", "pcx_fft_exec", "pcx_fxcorr_create", "pcx_fxcorr_exec"} <= syms
    for s in sorted(syms):
        assert hasattr(lib, s), f"{s} declared but not exported"
    assert syms <= set(_lib.SIGNATURES), "ctypes signatures missing for some entry points"


def test_version_string():
    assert b"sm_100a" in _lib.lib().pcx_version()


@pytest.mark.parametrize("n", [0, 1, 3, 1000, 4097])
def test_plan_rejects_non_power_of_two(n):
    plan = ctypes.c_void_p()
    rc = _lib.lib().pcx_plan_create(ctypes.byref(plan), n, 0, 0, 2048)
    assert rc == _lib.PCX_ERR_INVALID
    assert b"is not a power of two" in _lib.lib().pcx_last_error()
    assert not plan.value


@pytest.mark.parametrize("sub", [0, 4, 100])
def test_plan_rejects_bad_sub_size(sub):
    plan = ctypes.c_void_p()
    rc = _lib.lib().pcx_plan_create(ctypes.byref(plan), 1024, 0, 0, sub)
    assert rc == _lib.PCX_ERR_INVALID
    assert b"sub_size" in _lib.lib().pcx_last_error()


def test_plan_rejects_oversize_and_bad_enums():
    plan = ctypes.c_void_p()
    L = _lib.lib()
    assert L.pcx_plan_create(ctypes.byref(plan), 1 << 21, 0, 0, 2048) == _lib.PCX_ERR_UNSUPPORTED
    assert L.pcx_plan_create(ctypes.byref(plan), 1024, 7, 0, 2048) == _lib.PCX_ERR_INVALID
    assert L.pcx_plan_create(ctypes.byref(plan), 1024, 0, 5, 2048) == _lib.PCX_ERR_INVALID
    assert L.pcx_plan_create(None, 1024, 0, 0, 2048) == _lib.PCX_ERR_INVALID


def test_check_maps_status_to_reference_exceptions():
    L = _lib.lib()
    plan = ctypes.c_void_p()
    L.pcx_plan_create(ctypes.byref(plan), 3, 0, 0, 2048)
    with pytest.raises(ValueError, match="power of two"):
        _lib.check(_lib.PCX_ERR_INVALID)


def test_null_plan_calls_fail_cleanly():
    L = _lib.lib()
    assert L.pcx_plan_destroy(None) == 0
    assert L.pcx_plan_size(None) == 0
    rc = L.pcx_fft_exec(None, None, None, 0, 8, 8, 0, 1, 1, 0, 0, None)
    assert rc == _lib.PCX_ERR_INVALID
