"""pcx_fft_exec_noalloc: the batched FFT for callers that cannot allocate
device memory while running (a fixed budget set at start-up, memory handed
out only by their own pool).  It runs the same kernels as pcx_fft_exec but
takes its four-step scratch from a fixed 8 MiB device array instead of an
allocation.  Called through the C ABI on a fresh plan (before the plan has
any scratch of its own) and checked against pcx_fft_exec on two calls in a
row; after one set-up call, further calls must leave the device's free
memory unchanged.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

from packed_b200 import _lib, fft_unit, real_size
from tests._util import TOL

pytestmark = pytest.mark.gpu

SCRATCH = 8 << 20


def _noalloc(unit, dst, src, batch, direction=0, normalize=1, src_len=0):
    p = 8 if unit.dtype == torch.float32 else 4
    row = real_size(unit.size(), p)
    rc = _lib.lib().pcx_fft_exec_noalloc(unit._plan, ctypes.c_void_p(dst.data_ptr()),
                                         ctypes.c_void_p(src.data_ptr()), src_len, p, p, direction, normalize, batch,
                                         row, row, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)


def _free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _rel(a, b):
    a, b = a.double(), b.double()
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("log_n,batch,dtype", [(16, 5, torch.float32), (14, 70, torch.float32),
                                               (13, 9, torch.float32), (20, 3, torch.float32),
                                               (12, 7, torch.float32), (19, 2, torch.float64)])
def test_noalloc_matches_allocating_entry_point(log_n, batch, dtype):
    n = 1 << log_n
    p = 8 if dtype == torch.float32 else 4
    tol = TOL[np.float32 if dtype == torch.float32 else np.float64]
    g = torch.Generator(device="cuda").manual_seed(log_n)
    xs = [torch.randn(batch * real_size(n, p), device="cuda", dtype=dtype, generator=g) for _ in range(2)]
    got = [torch.full_like(x, float("nan")) for x in xs]
    want = [torch.empty_like(x) for x in xs]
    # a fresh plan that has never run pcx_fft_exec, so it holds no scratch of
    # its own: the no-alloc call must not fall back to plan scratch
    unit = fft_unit(n, dtype=dtype)
    _noalloc(unit, got[0], xs[0], batch)    # set-up call on this device
    unit.status()
    free0 = _free_bytes()
    # two calls in a row, different inputs and directions: the second runs on
    # the array the first one left behind
    for call in range(2):
        _noalloc(unit, got[call], xs[call], batch, direction=call % 2)
        unit.status()
        assert _free_bytes() == free0, "the allocation-free entry point changed the device's free memory"
    ref = fft_unit(n, dtype=dtype)
    for call in range(2):
        ref.exec(want[call], xs[call], batch=batch, direction=call % 2)
        assert _rel(got[call], want[call]) < tol


def test_noalloc_rejects_oversize_transform():
    # fp64 at 2^20 needs 16 MiB of scratch per transform: more than the array holds
    unit = fft_unit(1 << 20, dtype=torch.float64)
    x = torch.zeros(real_size(1 << 20, 4), device="cuda", dtype=torch.float64)
    with pytest.raises(NotImplementedError, match="scratch per transform"):
        _noalloc(unit, x, x, 1)
    assert _lib.lib().pcx_fft_exec_noalloc(None, None, None, 0, 8, 8, 0, 1, 1, 0, 0, None) == _lib.PCX_ERR_INVALID
