"""Host-side mirror of the reference's FFT API over the CUDA library.

Mirrors ``pcxo::fft_unit`` (reference fft.hpp:565-2166), ``pcxo::vector``
(vector.hpp:26-382) and ``pcxo::fxcorr_unit`` (fxcorr.hpp:44-147): the same
constructor arguments, method names, argument meanings and error behaviour
(``ValueError`` where the reference throws ``std::invalid_argument``, with the
same messages).  Data live in device memory as torch tensors holding the
packed split-complex reals; every transform runs in libpcx_cuda.so.
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np
import torch

from . import _lib

__all__ = ["fft_order", "default_pack_size", "vector", "fft_unit", "fxcorr_unit", "real_size"]


class fft_order(enum.IntEnum):
    """reference fft.hpp:540-544"""
    normal = 0
    bit_reversed = 1
    unordered = 2


def default_pack_size(dtype: torch.dtype) -> int:
    """32 bytes of reals per pack (reference types.hpp:70-72)."""
    return 32 // torch.empty((), dtype=dtype).element_size()


def real_size(n: int, pack: int) -> int:
    """reals needed for n elements at pack width `pack` (vector.hpp:373-381)."""
    return (n + pack - 1) // pack * 2 * pack


def _dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return _lib.PCX_F32
    if dtype == torch.float64:
        return _lib.PCX_F64
    raise TypeError(f"unsupported real type {dtype}")


def _stream_ptr(stream) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class vector:
    """Packed split-complex vector in device memory (pcxo::vector<T, P>).

    ``data`` is a 1-D torch tensor of ``real_size(size, pack)`` reals; element i
    has its real part at ``i + (i // P) * P`` and imaginary part ``P`` further.
    """

    def __init__(self, size: int, dtype: torch.dtype = torch.float32, pack: int | None = None,
                 device: str | torch.device = "cuda", data: torch.Tensor | None = None):
        self.pack_size = pack or default_pack_size(dtype)
        if self.pack_size <= 0 or self.pack_size & (self.pack_size - 1):
            raise ValueError("pack size must be a power of two")
        self._size = int(size)
        if data is None:
            data = torch.zeros(real_size(self._size, self.pack_size), dtype=dtype, device=device)
        self.data = data

    @classmethod
    def from_complex(cls, z, dtype: torch.dtype = torch.float32, pack: int | None = None, device="cuda"):
        z = np.asarray(z)
        p = pack or default_pack_size(dtype)
        n = z.shape[-1]
        npk = (n + p - 1) // p
        zz = np.zeros(npk * p, dtype=np.complex128)
        zz[:n] = z
        zz = zz.reshape(npk, p)
        host = np.stack([zz.real, zz.imag], axis=1).reshape(-1)
        t = torch.as_tensor(host, dtype=dtype).to(device)
        return cls(n, dtype, p, device, t)

    # element-wise arithmetic (lazy expressions, evaluated by assign)
    def __add__(self, o): return _Expr("add", self, _Expr.wrap(o))
    def __radd__(self, o): return _Expr("add", _Expr.wrap(o), self)
    def __sub__(self, o): return _Expr("sub", self, _Expr.wrap(o))
    def __rsub__(self, o): return _Expr("sub", _Expr.wrap(o), self)
    def __mul__(self, o): return _Expr("mul", self, _Expr.wrap(o))
    def __rmul__(self, o): return _Expr("mul", _Expr.wrap(o), self)
    def __truediv__(self, o): return _Expr("div", self, _Expr.wrap(o))
    def __rtruediv__(self, o): return _Expr("div", _Expr.wrap(o), self)

    def assign(self, expr, stream=None) -> "vector":
        """vector = expression (reference vector.hpp:177-182), on the device."""
        evaluate(self, expr, stream)
        return self

    def to_complex(self) -> np.ndarray:
        p = self.pack_size
        a = self.data.detach().cpu().numpy().astype(np.float64).reshape(-1, 2, p)
        return (a[:, 0, :] + 1j * a[:, 1, :]).reshape(-1)[: self._size]

    def size(self) -> int:
        return self._size

    def __len__(self) -> int:
        return self._size

    @property
    def dtype(self) -> torch.dtype:
        return self.data.dtype

    def __getitem__(self, i: int) -> complex:
        if not 0 <= i < self._size:
            raise IndexError("pcxo::vector index out of range")
        p = self.pack_size
        o = i + (i // p) * p
        return complex(float(self.data[o]), float(self.data[o + p]))


# ---------------------------------------------------------------- expressions
class _Expr:
    """Element-wise expression over vectors (reference vector_arithm.hpp:405-1140),
    evaluated on the device by ``vector.assign(expr)`` / ``evaluate``."""

    def __init__(self, kind, *args):
        self.kind, self.args = kind, args

    @staticmethod
    def wrap(x):
        if isinstance(x, (_Expr, vector)):
            return x
        return _Expr("scalar", complex(x))

    def __add__(self, o): return _Expr("add", self, _Expr.wrap(o))
    def __radd__(self, o): return _Expr("add", _Expr.wrap(o), self)
    def __sub__(self, o): return _Expr("sub", self, _Expr.wrap(o))
    def __rsub__(self, o): return _Expr("sub", _Expr.wrap(o), self)
    def __mul__(self, o): return _Expr("mul", self, _Expr.wrap(o))
    def __rmul__(self, o): return _Expr("mul", _Expr.wrap(o), self)
    def __truediv__(self, o): return _Expr("div", self, _Expr.wrap(o))
    def __rtruediv__(self, o): return _Expr("div", _Expr.wrap(o), self)


_OPS = {"vec": 0, "scalar": 1, "add": 2, "sub": 3, "mul": 4, "div": 5, "conj": 6}


class _ExprOp(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("arg", ctypes.c_int), ("re", ctypes.c_double), ("im", ctypes.c_double)]


def conj(x):
    """Complex conjugate of a vector or expression (lazy)."""
    return _Expr("conj", _Expr.wrap(x))


def evaluate(dest: "vector", expr, stream=None) -> None:
    """dest = expr, element-wise on the device (pcx_vec_eval)."""
    ops, vecs = [], []

    def emit(x):
        if isinstance(x, vector):
            if x.size() != dest.size():
                raise ValueError(f"source size (which is {x.size()} is not equal to subrange size (which is "
                                 f"{dest.size()})")
            if x.dtype != dest.dtype:
                raise TypeError("data type does not match")
            k = next((i for i, v in enumerate(vecs) if v is x), None)
            if k is None:
                vecs.append(x)
                k = len(vecs) - 1
            ops.append(_ExprOp(0, k, 0.0, 0.0))
        elif x.kind == "scalar":
            ops.append(_ExprOp(1, 0, x.args[0].real, x.args[0].imag))
        elif x.kind == "conj":
            emit(x.args[0])
            ops.append(_ExprOp(6, 0, 0.0, 0.0))
        else:
            emit(x.args[0])
            emit(x.args[1])
            ops.append(_ExprOp(_OPS[x.kind], 0, 0.0, 0.0))

    emit(_Expr.wrap(expr))
    arr = (_ExprOp * len(ops))(*ops)
    ptrs = (ctypes.c_void_p * max(1, len(vecs)))(*[v.data.data_ptr() for v in vecs])
    packs = (ctypes.c_int * max(1, len(vecs)))(*[v.pack_size for v in vecs])
    _lib.check(_lib.lib().pcx_vec_eval(_dtype_code(dest.dtype), _ptr(dest.data), dest.pack_size, dest.size(),
                                       ctypes.cast(arr, ctypes.c_void_p), len(ops), ptrs, packs, len(vecs),
                                       _stream_ptr(stream)))


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    if not t.is_cuda:
        raise ValueError("data must reside in CUDA device memory")
    return ctypes.c_void_p(t.data_ptr())


class fft_unit:
    """Plan of a power-of-two complex FFT (reference fft.hpp:565-2166).

    ``fft_unit(fft_size, sub_size=2048, dtype=torch.float32, order=fft_order.normal)``
    """

    def __init__(self, fft_size: int, sub_size: int = 2048, dtype: torch.dtype = torch.float32,
                 order: fft_order = fft_order.normal):
        self._dtype = dtype
        self._order = fft_order(order)
        self._plan = ctypes.c_void_p()
        L = _lib.lib()
        _lib.check(L.pcx_plan_create(ctypes.byref(self._plan), int(fft_size), _dtype_code(dtype), int(self._order),
                                     int(sub_size)))
        self._n = int(fft_size)

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib.lib().pcx_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def __copy__(self):
        raise TypeError("fft_unit is not assignable (reference fft.hpp:611-612)")

    # ---------------------------------------------------------------- info
    def size(self) -> int:
        return self._n

    @property
    def order(self) -> fft_order:
        return self._order

    @property
    def dtype(self) -> torch.dtype:
        return self._dtype

    def status(self) -> None:
        """Raise TimeoutError if a kernel gave up a bounded wait (pcx_plan_status)."""
        _lib.check(_lib.lib().pcx_plan_status(self._plan))

    def workspace_size(self, batch: int = 1) -> int:
        return int(_lib.lib().pcx_plan_workspace_size(self._plan, batch))

    FORMS = {0: "default", 1: "one-pass", 2: "one-launch four-step", 3: "chunked four-step"}

    def form(self) -> dict:
        """The plan's form (pcx_plan_form): name, tile distance in rounds, chunk scratch bytes."""
        f, r, c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_size_t(0)
        _lib.check(_lib.lib().pcx_plan_form(self._plan, ctypes.byref(f), ctypes.byref(r), ctypes.byref(c)))
        return {"form": self.FORMS.get(f.value, str(f.value)), "rounds": r.value, "chunk_bytes": c.value}

    def tuning(self) -> dict:
        """The plan's form and, for the one-launch four-step, its variant (pcx_plan_tuning):
        split N1 x N2, blocks per SM (tile shape), ring stages, dependency distance in rounds."""
        r = _lib.TuneResult()
        _lib.check(_lib.lib().pcx_plan_tuning(self._plan, ctypes.byref(r)))
        out = {"form": self.FORMS.get(r.form, str(r.form)), "rounds": r.rounds, "chunk_bytes": r.chunk_bytes}
        if r.log_n1 > 0 and r.form in (0, 2):
            out.update({"split": [1 << r.log_n1, 1 << r.log_n2], "blocks_per_sm": r.blocks_per_sm,
                        "stages": r.stages})
        return out

    def set_tuning(self, form: str = "one-launch four-step", *, split: tuple[int, int] | None = None,
                   blocks_per_sm: int = 0, stages: int = 0, rounds: int = 3, chunk_bytes: int = 0) -> None:
        """Choose a form (and four-step variant) without timing it (pcx_plan_set_tuning)."""
        codes = {v: k for k, v in self.FORMS.items()}
        r = _lib.TuneResult()
        r.form = codes[form]
        r.rounds = rounds
        r.chunk_bytes = chunk_bytes
        if split is not None:
            r.log_n1, r.log_n2 = (int(split[0]).bit_length() - 1, int(split[1]).bit_length() - 1)
            r.blocks_per_sm, r.stages = blocks_per_sm, stages
        _lib.check(_lib.lib().pcx_plan_set_tuning(self._plan, ctypes.byref(r)))

    def describe_form(self) -> str:
        """One line naming the form, its split and tile shape (for reports)."""
        t = self.tuning()
        if "split" in t and t["form"] in ("default", "one-launch four-step"):
            n1, n2 = t["split"]
            return (f"one-launch four-step {n1}x{n2}, {t['blocks_per_sm']} block(s)/SM "
                    f"({64 // t['blocks_per_sm']} KB tiles), {t['stages']} stages, distance {t['rounds']} rounds")
        if t["form"] == "chunked four-step":
            return f"chunked four-step, {t['chunk_bytes'] >> 20} MB scratch per buffer"
        return t["form"]

    def tune(self, batch: int = 1, stream=None) -> str:
        """Time this size's forms and four-step variants on `batch` rows and keep the fastest
        (pcx_plan_tune); returns describe_form()."""
        form = ctypes.c_int(0)
        _lib.check(_lib.lib().pcx_plan_tune(self._plan, batch, _stream_ptr(stream), ctypes.byref(form)))
        return self.describe_form()

    # ---------------------------------------------------------- raw calls
    def exec(self, dst: torch.Tensor, src: torch.Tensor, *, direction: int = 0, normalize: bool = True,
             batch: int = 1, pack_dst: int | None = None, pack_src: int | None = None, src_len: int = 0,
             dst_stride: int | None = None, src_stride: int | None = None, stream=None,
             workspace: torch.Tensor | None = None, check: bool = True) -> None:
        """Batched transform of `batch` rows of packed reals (pcx_fft_exec).

        With ``check`` (the default) the call waits for the stream and raises
        TimeoutError if a kernel gave up a bounded wait and left rows
        unwritten; ``check=False`` returns as soon as the work is queued, and
        the caller reads the flag later with :meth:`status`."""
        pd = pack_dst or default_pack_size(self._dtype)
        ps = pack_src or pd
        if dst.dtype != self._dtype or src.dtype != self._dtype:
            raise TypeError("data type does not match the fft_unit")
        ds = dst_stride if dst_stride is not None else real_size(self._n, pd)
        ss = src_stride if src_stride is not None else real_size(self._n, ps)
        L = _lib.lib()
        if workspace is None:
            rc = L.pcx_fft_exec(self._plan, _ptr(dst), _ptr(src), src_len, pd, ps, direction, int(normalize), batch,
                                ds, ss, _stream_ptr(stream))
        else:
            rc = L.pcx_fft_exec_ws(self._plan, _ptr(dst), _ptr(src), src_len, pd, ps, direction, int(normalize),
                                   batch, ds, ss, _ptr(workspace), workspace.numel() * workspace.element_size(),
                                   _stream_ptr(stream))
        _lib.check(rc)
        if check:
            self._wait_and_check(stream)

    def _wait_and_check(self, stream) -> None:
        (stream if stream is not None else torch.cuda.current_stream()).synchronize()
        self.status()

    def fft_raw(self, dest: torch.Tensor, source: torch.Tensor | None = None, source_size: int | None = None,
                pack_dest: int = 1, pack_src: int = 1) -> None:
        """fft_raw<PD,PS>(dest[, source[, source_size]]) (fft.hpp:624-681)."""
        src = dest if source is None else source
        self.exec(dest, src, direction=0, pack_dst=pack_dest, pack_src=pack_src, src_len=source_size or 0)

    def ifft_raw(self, dest: torch.Tensor, source: torch.Tensor | None = None, normalized: bool = True,
                 pack_dest: int = 1, pack_src: int = 1) -> None:
        """ifft_raw<Normalized,PD,PS>(dest[, source]) (fft.hpp:689-721)."""
        src = dest if source is None else source
        self.exec(dest, src, direction=1, normalize=normalized, pack_dst=pack_dest, pack_src=pack_src)

    # ------------------------------------------------------ vector calls
    def __call__(self, dest: vector, source: vector | None = None) -> None:
        """operator()(vector) in place, or operator()(dest, source) (fft.hpp:728-820)."""
        if source is None:
            if dest.size() != self._n:
                raise ValueError(f"input size (which is {dest.size()}) is not equal to fft size (which is "
                                 f"{self._n})")
            self.exec(dest.data, dest.data, direction=0, pack_dst=dest.pack_size, pack_src=dest.pack_size)
            return
        if dest.size() != self._n:
            raise ValueError(f"destination size (which is {dest.size()}) is not equal to fft size (which is "
                             f"{self._n})")
        if source.size() > self._n:
            raise ValueError(f"source size (which is {source.size()}) is bigger than fft size (which is "
                             f"{self._n})")
        self._check_repack(dest, source)
        self.exec(dest.data, source.data, direction=0, pack_dst=dest.pack_size, pack_src=source.pack_size,
                  src_len=source.size())

    def ifft(self, dest: vector, source: vector | None = None, normalized: bool = True) -> None:
        """ifft<Normalized>(vector) / ifft<Normalized>(dest, source) (fft.hpp:828-915)."""
        if source is None:
            if dest.size() != self._n:
                raise ValueError(f"input size (which is {dest.size()} is not equal to fft size (which is "
                                 f"{self._n})")
            self.exec(dest.data, dest.data, direction=1, normalize=normalized, pack_dst=dest.pack_size,
                      pack_src=dest.pack_size)
            return
        if dest.size() != self._n:
            raise ValueError(f"destination size (which is {dest.size()}) is not equal to fft size (which is "
                             f"{self._n})")
        if source.size() != self._n:
            raise ValueError(f"source size (which is {source.size()}) is not equal to fft size (which is "
                             f"{self._n})")
        self._check_repack(dest, source)
        self.exec(dest.data, source.data, direction=1, normalize=normalized, pack_dst=dest.pack_size,
                  pack_src=source.pack_size)

    def _check_repack(self, dest: vector, source: vector) -> None:
        # fft.hpp:783-792 — in-place repack with a pack wider than a register is refused
        reg = 32 // torch.empty((), dtype=self._dtype).element_size()
        if (dest.pack_size != source.pack_size and max(dest.pack_size, source.pack_size) > reg
                and dest.data.data_ptr() == source.data.data_ptr()):
            raise ValueError(f"cannot perform in-place repack from source pack size (which is {source.pack_size}) "
                             f"to destination pack size (which is {dest.pack_size})")

    def exec_tensor_core(self, dst: torch.Tensor, src: torch.Tensor, *, direction: int = 0, normalize: bool = True,
                         batch: int = 1, precision: str = "bf16", stream=None, check: bool = True) -> None:
        """Tensor-core form (pcx_tc_fft_exec): DFT-matrix stages with split operands, "bf16"
        (two parts, three products), "tf32" (two parts, three products) or "bf16x6" (three
        bf16 parts, six products).  ``check`` as in :meth:`exec`."""
        prec = {"bf16": 0, "tf32": 1, "bf16x6": 2}[precision]
        _lib.check(_lib.lib().pcx_tc_fft_exec(self._plan, _ptr(dst), _ptr(src), direction, int(normalize), batch,
                                              prec, _stream_ptr(stream)))
        if check:
            self._wait_and_check(stream)

    # ------------------------------------------------------------- adjoint
    def vjp(self, g_out: torch.Tensor, *, direction: int = 0, normalize: bool = True, batch: int = 1,
            pack: int | None = None, stream=None) -> torch.Tensor:
        """Cotangent of the input given the cotangent of the output (pcx_fft_vjp)."""
        p = pack or default_pack_size(self._dtype)
        g_in = torch.empty_like(g_out)
        _lib.check(_lib.lib().pcx_fft_vjp(self._plan, _ptr(g_in), _ptr(g_out), p, direction, int(normalize), batch,
                                          real_size(self._n, p), _stream_ptr(stream)))
        return g_in


class fft_unit_par(fft_unit):
    """Transform across vectors (reference fft.hpp:2167-2572).

    ``fft_unit_par(size, dtype=torch.float32, order=fft_order.normal)``;
    ``unit(dest, source)`` takes two sequences of ``size`` vectors of equal
    length L and, for every element position p < L, writes the transform of
    ``source[0][p] .. source[size-1][p]`` to ``dest[0][p] .. dest[size-1][p]``.
    """

    def __init__(self, size: int, dtype: torch.dtype = torch.float32, order: fft_order = fft_order.normal):
        super().__init__(size, 2048, dtype, order)

    def __call__(self, dest, source, *, inverse: bool = False, normalized: bool = True, stream=None) -> None:
        dest, source = list(dest), list(source)
        for name, vs in (("destination", dest), ("source", source)):
            if len(vs) != self._n:
                raise ValueError(f"{name} size (which is {len(vs)} is not equal to fft size (which is {self._n})")
        length = dest[0].size()
        for v in dest + source:
            if v.size() != length:
                raise ValueError("all vectors of a parallel transform have the same size")
            if v.dtype != self._dtype:
                raise TypeError("data type does not match the fft_unit_par")
        pd, ps = dest[0].pack_size, source[0].pack_size
        if any(v.pack_size != pd for v in dest) or any(v.pack_size != ps for v in source):
            raise ValueError("all vectors of one side share one pack size")
        arr = ctypes.c_void_p * self._n
        dptr = arr(*[v.data.data_ptr() for v in dest])
        sptr = arr(*[v.data.data_ptr() for v in source])
        _lib.check(_lib.lib().pcx_fft_par_exec(self._plan, dptr, sptr, self._n, length, pd, ps, int(inverse),
                                               int(normalized), _stream_ptr(stream)))


class fxcorr_unit:
    """Overlap-save cross-correlator (reference fxcorr.hpp:44-147).

    ``fxcorr_unit(g, fft_size)``: ``g`` is a :class:`vector` (device) or a
    complex array-like.  ``unit(x)`` correlates in place; ``unit(dest, src)``
    out of place (the reference leaves that overload empty, fxcorr.hpp:138-140).
    """

    def __init__(self, g, fft_size: int, dtype: torch.dtype | None = None):
        if not isinstance(g, vector):
            g = vector.from_complex(np.asarray(g), dtype=dtype or torch.float32)
        self._dtype = g.dtype
        self._k = g.size()
        self._pack_g = g.pack_size
        self._n = int(fft_size)
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().pcx_fxcorr_create(ctypes.byref(self._h), _ptr(g.data), self._k, g.pack_size, self._n,
                                                _dtype_code(self._dtype)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().pcx_fxcorr_destroy(h)
            except Exception:
                pass
            self._h = None

    def fft_size(self) -> int:
        return self._n

    def step(self, pack: int | None = None) -> int:
        """Outputs per overlap-save block: (N - (K-1)) rounded down to the pack."""
        p = pack or default_pack_size(self._dtype)
        return (self._n - (self._k - 1)) // p * p

    def status(self) -> None:
        """Raise TimeoutError if a block gave up a bounded wait (pcx_fxcorr_status)."""
        _lib.check(_lib.lib().pcx_fxcorr_status(self._h))

    def kernel_size(self) -> int:
        return self._k

    def exec(self, dst: torch.Tensor, src: torch.Tensor, length: int, *, channels: int = 1, pack: int | None = None,
             dst_stride: int | None = None, src_stride: int | None = None, stream=None,
             check: bool = True) -> None:
        """Correlate `channels` rows (pcx_fxcorr_exec).  With ``check`` (the default) the call
        waits for the stream and raises TimeoutError if a block gave up a bounded wait."""
        p = pack or default_pack_size(self._dtype)
        rs = real_size(length, p)
        _lib.check(_lib.lib().pcx_fxcorr_exec(self._h, _ptr(dst), _ptr(src), length, p, channels,
                                              dst_stride if dst_stride is not None else rs,
                                              src_stride if src_stride is not None else rs, _stream_ptr(stream)))
        if check:
            (stream if stream is not None else torch.cuda.current_stream()).synchronize()
            self.status()

    def __call__(self, dest: vector, source: vector | None = None) -> None:
        if source is None:
            self.exec(dest.data, dest.data, dest.size(), pack=dest.pack_size)
            return
        if dest.size() != source.size() or dest.pack_size != source.pack_size:
            raise ValueError("destination and source must have the same size and pack size")
        self.exec(dest.data, source.data, dest.size(), pack=dest.pack_size)

    def vjp(self, gy: torch.Tensor, x: torch.Tensor, length: int, *, channels: int = 1, pack: int | None = None,
            want_kernel_grad: bool = True, want_signal_grad: bool = True,
            stream=None) -> tuple[torch.Tensor | None, torch.Tensor | None]:
        """Cotangents of the signal and the kernel given the output's, `gy`
        (pcx_fxcorr_vjp); either may be skipped (returned as None)."""
        p = pack or default_pack_size(self._dtype)
        gx = torch.empty_like(gy) if want_signal_grad else None
        gg = (torch.empty(real_size(self._k, self._pack_g), dtype=self._dtype, device=gy.device)
              if want_kernel_grad else None)
        _lib.check(_lib.lib().pcx_fxcorr_vjp(self._h, _ptr(gx) if gx is not None else None,
                                             _ptr(gg) if gg is not None else None, _ptr(gy), _ptr(x), length, p,
                                             channels, real_size(length, p), _stream_ptr(stream)))
        return gx, gg


def correlation_fft_size(k: int, max_size: int = 16384) -> int:
    """FFT size for an overlap-save correlation with a k-tap kernel: the power
    of two N >= k + 7 that minimises the transform work per output sample,
    2 * N * log2(N) / (N - k + 1) (a forward and an inverse transform per
    block of N - k + 1 outputs), over 128 <= N <= max_size.  Sizes above 8192
    are taken only for kernels of more than 4096 taps, where they halve the
    block overlap; up to 8192 the ragged batch runs a correlation's blocks in
    its shared-memory ring."""
    best, best_cost = None, None
    n = 128
    while n <= max_size:
        if n >= k + 7 and (n <= 8192 or k > 4096):
            cost = 2 * n * (n.bit_length() - 1) / (n - k + 1)
            if best_cost is None or cost < best_cost:
                best, best_cost = n, cost
        n *= 2
    if best is None:
        raise ValueError(f"kernel size (which is {k}) needs an FFT size above {max_size}")
    return best


class ragged_batch:
    """Many FFTs of uneven power-of-two sizes and correlations in ONE
    persistent launch fed by a device work queue, replayed from a CUDA graph
    (pcx_ragged_*).  No counterpart in the reference.

    ``ffts``: list of ``(dst, src, n)`` — one complex64 transform each, pack 8
    (``n`` in 2^5..2^18).  ``xcorrs``: list of ``(dst, src, length, g, n_fft)``
    with ``g`` a :class:`vector` of kernel taps (out of place).  Pointers are
    fixed at construction; calling the object replays the graph.
    ``tensor_core`` ("bf16", "tf32" or "bf16x6", as ``fft_unit.exec_tensor_core``)
    runs the transforms of 2^8..2^12 points in the tensor-core form, a second
    persistent launch in the same graph (pcx_ragged_create_tc).
    """

    def __init__(self, ffts, xcorrs=(), direction: int = 0, normalize: bool = True,
                 tensor_core: str | None = None):
        n = len(ffts)
        m = len(xcorrs)
        sz = (ctypes.c_size_t * max(n, 1))(*[int(f[2]) for f in ffts])
        dsts = (ctypes.c_void_p * max(n, 1))(*[f[0].data_ptr() for f in ffts])
        srcs = (ctypes.c_void_p * max(n, 1))(*[f[1].data_ptr() for f in ffts])
        xl = (ctypes.c_size_t * max(m, 1))(*[int(x[2]) for x in xcorrs])
        xk = (ctypes.c_size_t * max(m, 1))(*[int(x[3].size()) for x in xcorrs])
        xg = (ctypes.c_void_p * max(m, 1))(*[x[3].data.data_ptr() for x in xcorrs])
        xn = (ctypes.c_size_t * max(m, 1))(*[int(x[4]) for x in xcorrs])
        xd = (ctypes.c_void_p * max(m, 1))(*[x[0].data_ptr() for x in xcorrs])
        xs = (ctypes.c_void_p * max(m, 1))(*[x[1].data_ptr() for x in xcorrs])
        self._keep = (ffts, xcorrs)
        self._h = ctypes.c_void_p()
        tc = -1 if tensor_core is None else {"bf16": 0, "tf32": 1, "bf16x6": 2}[tensor_core]
        _lib.check(_lib.lib().pcx_ragged_create_tc(ctypes.byref(self._h), _lib.PCX_F32, n, sz, dsts, srcs,
                                                   direction, int(normalize), m, xl, xk, xg, xn, xd, xs, tc))

    def __call__(self, stream=None) -> None:
        _lib.check(_lib.lib().pcx_ragged_exec(self._h, _stream_ptr(stream)))

    def status(self) -> None:
        _lib.check(_lib.lib().pcx_ragged_status(self._h))

    def items(self) -> int:
        return int(_lib.lib().pcx_ragged_items(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().pcx_ragged_destroy(h)
            except Exception:
                pass
            self._h = None
