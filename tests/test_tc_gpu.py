"""Tensor-core form (tcgen05 split-precision DFT-matrix stages): accuracy
against the FP64 oracle per size, and agreement with the plain FP32 path.
The two-part bf16 form (three products) is held to its own measured bound
(the dropped lo*lo product is up to 2^-18 of each term); the tf32 form and
the three-part bf16 form (six products) to the FP32 bar."""
import numpy as np
import pytest
import torch

import oracle as O
from packed_b200 import fft_unit
from tests._util import TOL, rel_l2

pytestmark = pytest.mark.gpu

BF16_BOUND = 1e-4


def c4_input(rng, b, n):
    # N(0,1) plus a 1e-3 tone at a seeded bin
    z = rng.standard_normal((b, n)) + 1j * rng.standard_normal((b, n))
    k = rng.integers(0, n, b)
    z += 1e-3 * np.exp(2j * np.pi * k[:, None] * np.arange(n)[None, :] / n)
    return z, k


@pytest.mark.parametrize("log_n", [8, 9, 10, 11, 12, 13, 14, 15, 16])
@pytest.mark.parametrize("precision", ["bf16", "tf32", "bf16x6"])
def test_tc_fft_accuracy(log_n, precision):
    n = 1 << log_n
    b = 33
    rng = np.random.default_rng(4)
    z, k = c4_input(rng, b, n)
    x = torch.as_tensor(O.pack(z, 8)).cuda()
    y = torch.full_like(x, float("nan"))
    unit = fft_unit(n)
    unit.exec_tensor_core(y, x, batch=b, precision=precision)
    torch.cuda.synchronize()
    unit.status()
    got = O.unpack(y.cpu().numpy(), n, 8)
    want = np.fft.fft(z, axis=-1)
    err = rel_l2(got, want)
    bound = BF16_BOUND if precision == "bf16" else TOL[np.float32]
    assert err < bound, f"{precision} N={n}: rel L2 {err:.3e}"
    # the tone bin keeps its value
    tone = np.abs(got[np.arange(b), k] - want[np.arange(b), k]).max()
    assert tone < 1e-2
    # inverse round trip
    back = torch.empty_like(y)
    unit.exec_tensor_core(back, y, batch=b, direction=1, precision=precision)
    assert rel_l2(O.unpack(back.cpu().numpy(), n, 8), z) < 2 * bound


@pytest.mark.parametrize("log_n", [14, 16])
def test_tc_two_pass_matches_plain_and_chunks(log_n):
    """The two-pass form agrees with the plain path, in place, and across
    scratch chunks (a batch several times the chunk)."""
    n = 1 << log_n
    b = 3 * ((24 << 20) // (8 * n)) + 5    # several 24 MB chunks and a ragged last one
    g = torch.Generator(device="cuda").manual_seed(14)
    x = torch.randn(b * 2 * n, device="cuda", generator=g)
    unit = fft_unit(n)
    want = torch.empty_like(x)
    unit.exec(want, x, batch=b)
    y = x.clone()
    unit.exec_tensor_core(y, y, batch=b, precision="tf32")    # in place
    torch.cuda.synchronize()
    unit.status()
    err = (torch.linalg.vector_norm(y.double() - want.double()) / torch.linalg.vector_norm(want.double())).item()
    assert err < TOL[np.float32]


def test_tc_sizes_outside_the_form_are_refused():
    for n in (128, 1 << 17):
        unit = fft_unit(n)
        x = torch.zeros(2 * n, device="cuda")
        with pytest.raises(NotImplementedError, match="tensor-core form"):
            unit.exec_tensor_core(x, x, batch=1)


@pytest.mark.parametrize("log_n,b", [(8, 20000), (10, 3001), (12, 1500)])
def test_tc_persistent_many_items_per_cta(log_n, b):
    """Whole-row sizes run as a persistent launch: with a batch of several
    items per resident CTA (items of 4096 points, the last one partial) every
    row must match the plain FP32 transform to the split form's accuracy."""
    n = 1 << log_n
    x = torch.randn(b, 2 * n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(log_n + b))
    unit = fft_unit(n)
    want = torch.empty_like(x)
    unit.exec(want, x, batch=b)
    for precision in ("bf16x6", "tf32"):
        y = torch.full_like(x, float("nan"))
        unit.exec_tensor_core(y, x, batch=b, precision=precision)
        torch.cuda.synchronize()
        unit.status()
        d = (y - want).double()
        rel = (d.norm(dim=1) / want.double().norm(dim=1)).max().item()
        assert rel < TOL[np.float32], (precision, rel)
