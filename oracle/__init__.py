"""TEST INFRASTRUCTURE ONLY: the CPU oracle and the reference shim.

Loaded only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg, always as the checker or the timed reference — never by the product
(``packed_b200`` does not import this package).

* ``liboracle.so`` — plain-C restatement of the reference's FFT / overlap-save
  path in double precision (``pcx_oracle.c``; each function cites the
  reference file:line it follows).
* ``_ref/libpcx_ref.so`` — the reference library's own headers compiled from
  their sources (``ref_shim.cpp``, ``Makefile``); present when the reference
  sources were available at build time.

Arrays: complex data is handled as numpy ``complex128`` here and converted to
and from the packed split-complex layout (pack width P: P reals then P
imaginaries per pack, reference vector.hpp:26-382).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = HERE / "liboracle.so"
_REF = HERE / "_ref" / "libpcx_ref.so"

_c_size = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)

_lib = None
_ref = None


# Reference checkout the shim is compiled from: PCX_REFERENCE, else
# /root/reference.  Where neither exists the prebuilt _ref library is used.
REFERENCE_DIR = os.environ.get("PCX_REFERENCE", "/root/reference")


def build() -> None:
    """Compile liboracle.so (and the reference shim when the sources exist)."""
    ref = Path(REFERENCE_DIR)
    args = [f"REF={ref}"] if ref.is_dir() else []
    subprocess.run(["make", "-s", "-C", str(HERE), *args], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB))
        _lib.orc_fft_c128.argtypes = [_dp, _c_size, ctypes.c_int]
        _lib.orc_dft_c128.argtypes = [_dp, _dp, _c_size, ctypes.c_int]
        _lib.orc_order_pos.argtypes = [_c_size, ctypes.c_int, _c_size]
        _lib.orc_order_pos.restype = _c_size
        for suf, ptr in (("f32", _fp), ("f64", _dp)):
            f = getattr(_lib, f"orc_fft_packed_{suf}")
            f.argtypes = [ptr, ptr, _c_size, _c_size, _c_size, _c_size, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            f.restype = ctypes.c_int
        _lib.orc_xcorr_direct.argtypes = [_dp, _c_size, _dp, _c_size, _dp]
        _lib.orc_xcorr_ols.argtypes = [_dp, _c_size, _dp, _c_size, _c_size, _c_size, _dp]
        _lib.orc_xcorr_ols.restype = ctypes.c_int
        _lib.orc_xcorr_vjp_direct.argtypes = [_dp, _c_size, _dp, _c_size, _dp, _dp, _dp]
    return _lib


def ref_available() -> bool:
    return _REF.exists()


def ref() -> ctypes.CDLL:
    """The reference library's own code (compiled from its headers)."""
    global _ref
    if _ref is None:
        if not _REF.exists():
            raise FileNotFoundError(f"{_REF} not built (reference sources absent at build time)")
        _ref = ctypes.CDLL(str(_REF))
        _ref.ref_fft_f32.argtypes = [ctypes.c_int, _c_size, _c_size, _fp, ctypes.c_int, ctypes.c_int]
        _ref.ref_fft_oop_f32.argtypes = [ctypes.c_int, _c_size, _c_size, _fp, _fp, _c_size, ctypes.c_int,
                                         ctypes.c_int]
        _ref.ref_fxcorr_f32.argtypes = [_fp, _c_size, _c_size, _fp, _c_size]
        _ref.ref_fxcorr_fixed_f32.argtypes = [_fp, _c_size, _c_size, _fp, _c_size]
        _ref.ref_fft_batch_f32.argtypes = [ctypes.c_int, _c_size, _c_size, _fp, ctypes.c_int, ctypes.c_int]
        _ref.ref_fxcorr_fixed_batch_f32.argtypes = [_fp, _c_size, _c_size, _fp, _c_size, _c_size, ctypes.c_int]
        _ref.ref_fft_raw_packs_f32.argtypes = [ctypes.c_int, _c_size, _c_size, _fp, _fp, ctypes.c_int,
                                               ctypes.c_int]
        _ref.ref_last_error.restype = ctypes.c_char_p
        for name in ("ref_fft_f32", "ref_fft_oop_f32", "ref_fxcorr_f32", "ref_fxcorr_fixed_f32",
                     "ref_fft_batch_f32", "ref_fxcorr_fixed_batch_f32", "ref_fft_raw_packs_f32"):
            getattr(_ref, name).restype = ctypes.c_int
    return _ref


# ------------------------------------------------------------------ layout
def real_size(n: int, p: int) -> int:
    return (n + p - 1) // p * 2 * p


def pack(z: np.ndarray, p: int, dtype=np.float32) -> np.ndarray:
    """complex array [..., n] -> packed reals [..., real_size(n, p)]."""
    z = np.asarray(z)
    n = z.shape[-1]
    npk = (n + p - 1) // p
    out = np.zeros(z.shape[:-1] + (npk, 2, p), dtype=dtype)
    zz = np.zeros(z.shape[:-1] + (npk * p,), dtype=np.complex128)
    zz[..., :n] = z
    zz = zz.reshape(z.shape[:-1] + (npk, p))
    out[..., 0, :] = zz.real
    out[..., 1, :] = zz.imag
    return out.reshape(z.shape[:-1] + (npk * 2 * p,))


def unpack(a: np.ndarray, n: int, p: int) -> np.ndarray:
    """packed reals [..., >= real_size(n,p)] -> complex128 [..., n]."""
    a = np.asarray(a)
    npk = (n + p - 1) // p
    b = a[..., : npk * 2 * p].reshape(a.shape[:-1] + (npk, 2, p)).astype(np.float64)
    z = b[..., 0, :] + 1j * b[..., 1, :]
    return z.reshape(a.shape[:-1] + (npk * p,))[..., :n]


def order_pos(n: int, order: int) -> np.ndarray:
    """pos[k] = position holding frequency k."""
    L = lib()
    return np.array([L.orc_order_pos(k, order, n) for k in range(n)], dtype=np.int64)


# ------------------------------------------------------------------ oracle
def _c128(z: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(z, dtype=np.complex128)


def fft(z: np.ndarray, inverse: bool = False) -> np.ndarray:
    """Unnormalised natural-order DFT of each row (radix-2 restatement)."""
    z = _c128(z).copy()
    n = z.shape[-1]
    rows = z.reshape(-1, n)
    L = lib()
    for r in rows:
        L.orc_fft_c128(r.ctypes.data_as(_dp), n, int(inverse))
    return rows.reshape(z.shape)


def dft(z: np.ndarray, inverse: bool = False) -> np.ndarray:
    """Direct O(n^2) DFT, long-double accumulation (small n)."""
    z = _c128(z)
    n = z.shape[-1]
    out = np.empty_like(z.reshape(-1, n))
    L = lib()
    for i, r in enumerate(z.reshape(-1, n)):
        r = np.ascontiguousarray(r)
        L.orc_dft_c128(r.ctypes.data_as(_dp), out[i].ctypes.data_as(_dp), n, int(inverse))
    return out.reshape(z.shape)


def fft_packed(src: np.ndarray, n: int, *, order: int = 0, direction: int = 0, normalize: bool = True,
               pack_src: int = 8, pack_dst: int = 8, src_len: int = 0, dtype=np.float32) -> np.ndarray:
    """Reference-semantics transform of packed rows (see pcx_oracle.c)."""
    L = lib()
    src = np.ascontiguousarray(src, dtype=dtype)
    rows = src.reshape(-1, src.shape[-1])
    rd = real_size(n, pack_dst)
    out = np.zeros((rows.shape[0], rd), dtype=dtype)
    f, ptr = (L.orc_fft_packed_f32, _fp) if dtype == np.float32 else (L.orc_fft_packed_f64, _dp)
    for i in range(rows.shape[0]):
        s = np.ascontiguousarray(rows[i])
        rc = f(out[i].ctypes.data_as(ptr), s.ctypes.data_as(ptr), n, src_len, pack_dst, pack_src, order,
               direction, int(normalize))
        assert rc == 0
    return out.reshape(src.shape[:-1] + (rd,))


def xcorr_direct(x: np.ndarray, g: np.ndarray) -> np.ndarray:
    x, g = _c128(x), _c128(g)
    y = np.empty_like(x)
    lib().orc_xcorr_direct(x.ctypes.data_as(_dp), x.shape[-1], g.ctypes.data_as(_dp), g.shape[-1],
                           y.ctypes.data_as(_dp))
    return y


def xcorr_ols(x: np.ndarray, g: np.ndarray, n_fft: int, pack: int = 8) -> np.ndarray:
    x, g = _c128(x), _c128(g)
    y = np.empty_like(x)
    rc = lib().orc_xcorr_ols(x.ctypes.data_as(_dp), x.shape[-1], g.ctypes.data_as(_dp), g.shape[-1], n_fft, pack,
                             y.ctypes.data_as(_dp))
    assert rc == 0
    return y


def xcorr_vjp_direct(x: np.ndarray, g: np.ndarray, gy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    x, g, gy = _c128(x), _c128(g), _c128(gy)
    gx = np.empty_like(x)
    gg = np.empty_like(g)
    lib().orc_xcorr_vjp_direct(x.ctypes.data_as(_dp), x.shape[-1], g.ctypes.data_as(_dp), g.shape[-1],
                               gy.ctypes.data_as(_dp), gx.ctypes.data_as(_dp), gg.ctypes.data_as(_dp))
    return gx, gg


# --------------------------------------------------------------- reference
def ref_fft(packed: np.ndarray, n: int, order: int, direction: int, normalize: bool = True,
            sub_size: int = 2048) -> np.ndarray:
    """In-place transform of one pack-8 row through the reference fft_unit<float>."""
    a = np.ascontiguousarray(packed, dtype=np.float32).copy()
    rc = ref().ref_fft_f32(order, n, sub_size, a.ctypes.data_as(_fp), direction, int(normalize))
    if rc:
        raise ValueError(ref().ref_last_error().decode())
    return a


def ref_fft_oop(src: np.ndarray, n: int, src_len: int, order: int, direction: int, normalize: bool = True,
                sub_size: int = 2048) -> np.ndarray:
    dst = np.zeros(2 * n, dtype=np.float32)
    s = np.ascontiguousarray(src, dtype=np.float32)
    rc = ref().ref_fft_oop_f32(order, n, sub_size, dst.ctypes.data_as(_fp), s.ctypes.data_as(_fp), src_len,
                               direction, int(normalize))
    if rc:
        raise ValueError(ref().ref_last_error().decode())
    return dst


def ref_fft_raw_packs(src: np.ndarray, n: int, pack_dst: int, pack_src: int, order: int = 0,
                      sub_size: int = 2048) -> np.ndarray:
    """Forward transform of one row through the reference's fft_raw<PD, PS>(dest, source)."""
    s = np.ascontiguousarray(src, dtype=np.float32)
    dst = np.zeros(real_size(n, pack_dst), dtype=np.float32)
    rc = ref().ref_fft_raw_packs_f32(order, n, sub_size, dst.ctypes.data_as(_fp), s.ctypes.data_as(_fp), pack_dst,
                                     pack_src)
    if rc:
        raise ValueError(ref().ref_last_error().decode())
    return dst


def ref_fxcorr(g_packed: np.ndarray, k: int, n_fft: int, x_packed: np.ndarray, s: int, fixed: bool) -> np.ndarray:
    a = np.ascontiguousarray(x_packed, dtype=np.float32).copy()
    g = np.ascontiguousarray(g_packed, dtype=np.float32)
    fn = ref().ref_fxcorr_fixed_f32 if fixed else ref().ref_fxcorr_f32
    rc = fn(g.ctypes.data_as(_fp), k, n_fft, a.ctypes.data_as(_fp), s)
    if rc:
        raise ValueError(ref().ref_last_error().decode())
    return a


def host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
