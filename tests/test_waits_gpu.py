"""The kernels' bounded device waits give up and report instead of hanging.

Every spin in the kernels (an mbarrier phase, another block's completion
counter) has a time limit, after which the kernel records an error the host
reads (pcx_plan_status and friends) and returns.  Here one GPU thread runs
those waits on conditions that never come true; both must give up, and the
context must stay usable for a normal transform afterwards."""
import ctypes
import time

import numpy as np
import pytest
import torch

import oracle as O
from packed_b200 import _lib, fft_unit
from tests._util import TOL, rel_l2

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_the_context_stays_usable():
    mbar, ctr = ctypes.c_int(-1), ctypes.c_int(-1)
    t0 = time.perf_counter()
    _lib.check(_lib.lib().pcx_selftest_waits(50_000_000, ctypes.byref(mbar), ctypes.byref(ctr)))
    dt = time.perf_counter() - t0
    assert mbar.value == 0 and ctr.value == 0
    assert dt < 30    # ~1 s of counter wait, plus start-up
    # the GPU still answers: a transform right after matches numpy
    n, b = 1 << 16, 3
    z = np.random.default_rng(7).standard_normal((b, n)) + 1j * np.random.default_rng(8).standard_normal((b, n))
    x = torch.as_tensor(O.pack(z, 8)).cuda()
    y = torch.empty_like(x)
    u = fft_unit(n)
    u.exec(y, x, batch=b)
    u.status()
    assert rel_l2(O.unpack(y.cpu().numpy(), n, 8), np.fft.fft(z, axis=-1)) < TOL[np.float32]
