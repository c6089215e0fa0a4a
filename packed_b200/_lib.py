"""ctypes binding of libpcx_cuda.so (the C ABI declared in include/pcx_cuda.h).

The library is built in-tree by ``python -m packed_b200.build``.  There is no
fallback: if the shared library is missing every call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

_PATH = Path(__file__).resolve().parent / "libpcx_cuda.so"

PCX_OK = 0
PCX_ERR_INVALID = 1
PCX_ERR_CUDA = 2
PCX_ERR_UNSUPPORTED = 3
PCX_ERR_TIMEOUT = 4

PCX_F32 = 0
PCX_F64 = 1

_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_i = ctypes.c_int

# name -> (restype, argtypes); keep in sync with include/pcx_cuda.h
SIGNATURES: dict[str, tuple] = {
    "pcx_last_error": (ctypes.c_char_p, []),
    "pcx_version": (ctypes.c_char_p, []),
    "pcx_plan_create": (_i, [ctypes.POINTER(_vp), _sz, _i, _i, _sz]),
    "pcx_plan_destroy": (_i, [_vp]),
    "pcx_plan_size": (_sz, [_vp]),
    "pcx_plan_status": (_i, [_vp]),
    "pcx_selftest_waits": (_i, [ctypes.c_ulonglong, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "pcx_selftest_plan_wait": (_i, [_vp, ctypes.c_ulonglong, _vp]),
    "pcx_plan_workspace_size": (_sz, [_vp, _sz]),
    "pcx_plan_tune": (_i, [_vp, _sz, _vp, ctypes.POINTER(_i)]),
    "pcx_plan_form": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_sz)]),
    "pcx_plan_tuning": (_i, [_vp, _vp]),
    "pcx_plan_set_tuning": (_i, [_vp, _vp]),
    "pcx_tune_cache_load": (_i, [ctypes.c_char_p]),
    "pcx_tune_cache_save": (_i, [ctypes.c_char_p]),
    "pcx_tune_cache_put": (_i, [ctypes.c_char_p, _sz, _i, _sz, _vp]),
    "pcx_tune_cache_get": (_i, [ctypes.c_char_p, _sz, _i, _sz, _vp]),
    "pcx_tune_cache_clear": (_i, []),
    "pcx_tune_cache_size": (_sz, []),
    "pcx_fft_par_exec": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _sz, _sz, _i, _i, _i, _i, _vp]),
    "pcx_vec_eval": (_i, [_i, _vp, _i, _sz, _vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_i), _i, _vp]),
    "pcx_fft_exec": (_i, [_vp, _vp, _vp, _sz, _i, _i, _i, _i, _sz, _sz, _sz, _vp]),
    "pcx_fft_exec_ws": (_i, [_vp, _vp, _vp, _sz, _i, _i, _i, _i, _sz, _sz, _sz, _vp, _sz, _vp]),
    "pcx_fft_vjp": (_i, [_vp, _vp, _vp, _i, _i, _i, _sz, _sz, _vp]),
    "pcx_fft_exec_noalloc": (_i, [_vp, _vp, _vp, _sz, _i, _i, _i, _i, _sz, _sz, _sz, _vp]),
    "pcx_fxcorr_create": (_i, [ctypes.POINTER(_vp), _vp, _sz, _i, _sz, _i]),
    "pcx_fxcorr_destroy": (_i, [_vp]),
    "pcx_fxcorr_exec": (_i, [_vp, _vp, _vp, _sz, _i, _sz, _sz, _sz, _vp]),
    "pcx_fxcorr_vjp": (_i, [_vp, _vp, _vp, _vp, _vp, _sz, _i, _sz, _sz, _vp]),
    "pcx_fxcorr_status": (_i, [_vp]),
    "pcx_tc_fft_exec": (_i, [_vp, _vp, _vp, _i, _i, _sz, _i, _vp]),
    "pcx_ragged_create": (_i, [ctypes.POINTER(_vp), _i, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_vp),
                               ctypes.POINTER(_vp), _i, _i, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_sz),
                               ctypes.POINTER(_vp), ctypes.POINTER(_sz), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "pcx_ragged_create_tc": (_i, [ctypes.POINTER(_vp), _i, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_vp),
                                  ctypes.POINTER(_vp), _i, _i, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_sz),
                                  ctypes.POINTER(_vp), ctypes.POINTER(_sz), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                  _i]),
    "pcx_ragged_exec": (_i, [_vp, _vp]),
    "pcx_ragged_status": (_i, [_vp]),
    "pcx_ragged_items": (_sz, [_vp]),
    "pcx_ragged_destroy": (_i, [_vp]),
}

class TuneResult(ctypes.Structure):
    """pcx_tune_result (include/pcx_cuda.h)."""
    _fields_ = [("form", _i), ("rounds", _i), ("chunk_bytes", _sz), ("log_n1", _i), ("log_n2", _i),
                ("blocks_per_sm", _i), ("stages", _i), ("ms", ctypes.c_double)]


_lib: ctypes.CDLL | None = None


class PcxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def path() -> Path:
    return _PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _PATH.exists():
            raise ImportError(f"{_PATH} is not built; run `python -m packed_b200.build` (no CPU fallback exists)")
        l = ctypes.CDLL(str(_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(rc: int) -> None:
    """Raise the exception type the reference raises for this status."""
    if rc == PCX_OK:
        return
    msg = lib().pcx_last_error().decode()
    if rc == PCX_ERR_INVALID:
        raise ValueError(msg)    # std::invalid_argument in the reference
    if rc == PCX_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == PCX_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise PcxError(rc, msg)
