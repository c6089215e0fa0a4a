"""GPU parity of the FFT path (libpcx_cuda.so through its C ABI) against the
CPU oracle and the reference's golden outputs.  Bar: relative L2 2e-6 (FP32),
1e-13 (FP64)."""
import re
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle as O
from packed_b200 import fft_order, fft_unit, real_size, vector
from tests._util import TOL, golden, normal_cx, rel_l2

pytestmark = pytest.mark.gpu

F32, F64 = torch.float32, torch.float64
NPD = {F32: np.float32, F64: np.float64}


def to_dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).cuda()


def run(unit, src_packed, batch, **kw):
    src = to_dev(src_packed, unit.dtype)
    dst = torch.empty_like(src) if kw.pop("inplace", False) is False else src
    unit.exec(dst, src, batch=batch, **kw)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def rows_for(n):
    return max(1, min(6, (1 << 16) // n)) if n <= 4096 else (7 if n >= (1 << 19) else 3)


@pytest.mark.parametrize("log_n", list(range(1, 21)))
@pytest.mark.parametrize("order", [0, 1, 2])
def test_forward_inverse_parity_f32(log_n, order):
    n = 1 << log_n
    if order == 2 and n < 16:
        pytest.skip("unordered defined for n >= 16")
    rng = np.random.default_rng(100 + log_n)
    b = rows_for(n)
    p = min(8, n)
    z = normal_cx(rng, b, n)
    x = O.pack(z, p)
    unit = fft_unit(n, dtype=F32, order=order)
    got = run(unit, x, b, direction=0, pack_dst=p, pack_src=p)
    want = O.fft_packed(x, n, order=order, pack_src=p, pack_dst=p)
    assert rel_l2(O.unpack(got, n, p), O.unpack(want, n, p)) < TOL[np.float32]
    back = run(unit, want.astype(np.float32), b, direction=1, pack_dst=p, pack_src=p)
    assert rel_l2(O.unpack(back, n, p), z) < TOL[np.float32]


@pytest.mark.parametrize("log_n", [4, 6, 10, 12, 13, 16, 20])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_parity_f64(log_n, order):
    n = 1 << log_n
    rng = np.random.default_rng(200 + log_n)
    b = 2 if n >= 4096 else 4
    z = normal_cx(rng, b, n)
    x = O.pack(z, 4, np.float64)
    unit = fft_unit(n, dtype=F64, order=order)
    got = run(unit, x, b, direction=0, pack_dst=4, pack_src=4)
    want = O.fft_packed(x, n, order=order, pack_src=4, pack_dst=4, dtype=np.float64)
    assert rel_l2(O.unpack(got, n, 4), O.unpack(want, n, 4)) < TOL[np.float64]
    back = run(unit, want, b, direction=1, pack_dst=4, pack_src=4)
    assert rel_l2(O.unpack(back, n, 4), z) < TOL[np.float64]


def test_fp64_template_check_c2():
    # FP64 template check of the size sweep: N=2^12, batch 4096, pack 4, N(0,1) seed 1
    n, b = 4096, 4096
    rng = np.random.default_rng(1)
    z = normal_cx(rng, b, n)
    x = O.pack(z, 4, np.float64)
    unit = fft_unit(n, dtype=F64)
    got = O.unpack(run(unit, x, b, direction=0, pack_dst=4, pack_src=4), n, 4)
    want = np.fft.fft(z, axis=-1)
    assert rel_l2(got, want) < TOL[np.float64]


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_matches_reference_golden(n, order):
    G = golden()
    unit = fft_unit(n, order=order)
    got = run(unit, G[f"x_{n}"], 1, direction=0)
    assert rel_l2(O.unpack(got, n, 8), O.unpack(G[f"fwd_{n}_o{order}"], n, 8)) < TOL[np.float32]
    inv = run(unit, G[f"fwd_{n}_o{order}"], 1, direction=1)
    assert rel_l2(O.unpack(inv, n, 8), O.unpack(G[f"inv_{n}_o{order}"], n, 8)) < TOL[np.float32]
    if order:
        raw = run(unit, G[f"fwd_{n}_o{order}"], 1, direction=1, normalize=False)
        assert rel_l2(O.unpack(raw, n, 8), O.unpack(G[f"invraw_{n}_o{order}"], n, 8)) < TOL[np.float32]


def test_c1_config_against_reference_and_fp64():
    # N=1024, batch 64, U[-1,1) seed 0; forward then inverse (1/N)
    G = golden()
    rng = np.random.default_rng(0)
    z = np.stack([(rng.uniform(-1, 1, 1024) + 1j * rng.uniform(-1, 1, 1024)).astype(np.complex64)
                  for _ in range(64)])
    x = O.pack(z, 8)
    unit = fft_unit(1024)
    fwd = run(unit, x, 64, direction=0)
    inv = run(unit, fwd, 64, direction=1)
    assert rel_l2(O.unpack(fwd[:4], 1024, 8), O.unpack(G["c1_fwd"], 1024, 8)) < TOL[np.float32]
    assert rel_l2(O.unpack(inv[:4], 1024, 8), O.unpack(G["c1_inv"], 1024, 8)) < TOL[np.float32]
    assert rel_l2(O.unpack(fwd, 1024, 8), O.dft(z.astype(np.complex128))) < TOL[np.float32]
    assert rel_l2(O.unpack(inv, 1024, 8), z) < TOL[np.float32]


def test_reference_tone_input():
    G = golden()
    got = run(fft_unit(1024), G["tone_x_1024"], 1)
    assert rel_l2(O.unpack(got, 1024, 8), O.unpack(G["tone_fwd_1024"], 1024, 8)) < TOL[np.float32]


@pytest.mark.parametrize("n", [1024, 1 << 14])
def test_zero_extended_source(n):
    rng = np.random.default_rng(5)
    for order in (0, 1, 2):
        for src_len in (1, 700 * n // 1024, n - 3):
            z = normal_cx(rng, src_len)
            src = to_dev(O.pack(z, 8), F32)
            dst = torch.full((2 * n,), float("nan"), device="cuda")
            fft_unit(n, order=order).exec(dst, src, src_len=src_len)
            want = O.fft_packed(O.pack(z, 8), n, order=order, src_len=src_len)
            assert rel_l2(O.unpack(dst.cpu().numpy(), n, 8), O.unpack(want, n, 8)) < TOL[np.float32]
    G = golden()
    got = torch.empty(2048, device="cuda")
    fft_unit(1024, order=1).exec(got, to_dev(G["zx_src_700"], F32), src_len=700)
    assert rel_l2(O.unpack(got.cpu().numpy(), 1024, 8), O.unpack(G["zx_fwd_1024_o1"], 1024, 8)) < 2e-6


@pytest.mark.parametrize("n", [256, 4096, 1 << 15])
def test_pack_conversion_and_strides(n):
    rng = np.random.default_rng(9)
    b = 3
    z = normal_cx(rng, b, n)
    unit = fft_unit(n)
    want = np.fft.fft(z, axis=-1)
    for ps, pd in ((1, 8), (8, 1), (2, 4), (4, 4), (8, 8), (16, 8), (8, 16), (16, 16), (1, 16), (16, 2)):
        pad_s, pad_d = 16, 48
        rs, rd = real_size(n, ps) + pad_s, real_size(n, pd) + pad_d
        src = np.zeros((b, rs), np.float32)
        src[:, : real_size(n, ps)] = O.pack(z, ps)
        s = to_dev(src, F32)
        d = torch.zeros((b, rd), device="cuda")
        unit.exec(d, s, batch=b, pack_src=ps, pack_dst=pd, src_stride=rs, dst_stride=rd)
        out = d.cpu().numpy()
        assert rel_l2(O.unpack(out[:, : real_size(n, pd)], n, pd), want) < TOL[np.float32]
        assert np.all(out[:, real_size(n, pd):] == 0), "wrote outside the rows"


@pytest.mark.parametrize("n", [64, 4096, 1 << 17])
def test_in_place(n):
    rng = np.random.default_rng(11)
    z = normal_cx(rng, 2, n)
    x = to_dev(O.pack(z, 8), F32)
    unit = fft_unit(n, order=fft_order.bit_reversed)
    unit.exec(x, x, batch=2)
    want = O.fft_packed(O.pack(z, 8), n, order=1)
    assert rel_l2(O.unpack(x.cpu().numpy(), n, 8), O.unpack(want, n, 8)) < TOL[np.float32]
    unit.exec(x, x, batch=2, direction=1)
    assert rel_l2(O.unpack(x.cpu().numpy(), n, 8), z) < TOL[np.float32]


def test_vector_api_and_errors():
    n = 512
    rng = np.random.default_rng(2)
    z = normal_cx(rng, n)
    v = vector.from_complex(z)
    unit = fft_unit(n)
    unit(v)
    assert rel_l2(v.to_complex(), np.fft.fft(z)) < TOL[np.float32]
    unit.ifft(v)
    assert rel_l2(v.to_complex(), z) < TOL[np.float32]
    # out-of-place with a shorter source (zero extension) and another pack width
    s = vector.from_complex(z[:300], pack=4)
    d = vector(n)
    unit(d, s)
    zz = np.zeros(n, complex)
    zz[:300] = z[:300]
    assert rel_l2(d.to_complex(), np.fft.fft(zz)) < TOL[np.float32]
    # out-of-place inverse is the correct inverse (the reference's is not)
    back = vector(n, pack=2)
    unit.ifft(back, d)
    assert rel_l2(back.to_complex(), zz) < TOL[np.float32]
    with pytest.raises(ValueError, match="is not equal to fft size"):
        unit(vector(n // 2))
    with pytest.raises(ValueError, match="is bigger than fft size"):
        unit(vector(n), vector(n * 2))
    with pytest.raises(ValueError, match="in-place repack"):
        unit(vector(n, pack=16, data=d.data), vector(n, pack=8, data=d.data))


def test_unnormalized_inverse_all_orders():
    n = 2048
    rng = np.random.default_rng(4)
    z = normal_cx(rng, n)
    for order in (0, 1, 2):
        unit = fft_unit(n, order=order)
        y = O.fft_packed(O.pack(z, 8), n, order=order)
        got = run(unit, y, 1, direction=1, normalize=False)
        assert rel_l2(O.unpack(got, n, 8), z * n) < TOL[np.float32]


@pytest.mark.parametrize("log_n", [6, 12, 14, 20])
def test_vjp_adjoint_identity(log_n):
    # <F x, y> == <x, F^H y> for the forward and the normalised inverse
    n = 1 << log_n
    rng = np.random.default_rng(log_n)
    x, y = normal_cx(rng, n), normal_cx(rng, n)
    for order in (0, 1):
        unit = fft_unit(n, dtype=F64, order=order)
        for direction, norm in ((0, True), (1, True), (1, False)):
            xd = to_dev(O.pack(x, 4, np.float64), F64)
            fx = torch.empty_like(xd)
            unit.exec(fx, xd, direction=direction, normalize=norm)
            gy = to_dev(O.pack(y, 4, np.float64), F64)
            gx = unit.vjp(gy, direction=direction, normalize=norm)
            lhs = np.vdot(O.unpack(fx.cpu().numpy(), n, 4), y)
            rhs = np.vdot(x, O.unpack(gx.cpu().numpy(), n, 4))
            assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("log_n", [10, 16])
def test_vjp_vs_central_fd(log_n):
    """pcx_fft_vjp (FP64 plan) against FP64 central finite differences of
    L = sum w |Y|^2, Y = the plan's forward, normalised inverse or unnormalised
    inverse of x, w ~ U[0,1): 32 coordinates, real and imaginary directions,
    |fd - grad| <= 1e-6 * max(1, |fd|).  Y is linear in x, so the perturbed
    outputs are Y +- h*dY with dY the transform of the unit step, and the
    difference is summed term by term.  L is quadratic, so the central
    difference has no truncation error at any step; h = 1e-3 keeps its
    rounding noise near 1e-9 (at h = 1e-6 forming Y +- h*dY from |Y| ~ sqrt(n)
    leaves up to ~2e-6 on coordinates whose gradient is small)."""
    n, batch, h = 1 << log_n, 2, 1e-3
    rng = np.random.default_rng(log_n + 100)
    z = normal_cx(rng, batch, n)
    w = rng.uniform(0, 1, (batch, n))
    unit = fft_unit(n, dtype=F64)
    k = np.arange(n)
    for direction, norm in ((0, True), (1, True), (1, False)):
        scale = 1.0 / n if (direction == 1 and norm) else 1.0
        Y = (np.fft.fft(z, axis=-1) if direction == 0 else np.fft.ifft(z, axis=-1) * n) * scale
        gy = to_dev(O.pack(2 * w * Y, 4, np.float64), F64)    # dL/dRe Y + i dL/dIm Y
        gx = O.unpack(unit.vjp(gy, direction=direction, normalize=norm, batch=batch).cpu().numpy(), n, 4)
        sign = -1.0 if direction == 0 else 1.0
        for b, i in zip(rng.integers(0, batch, 32), rng.integers(0, n, 32)):
            col = np.exp(sign * 2j * np.pi * ((i * k) % n) / n) * scale    # transform of e_i
            for u, an in ((1.0, gx[b, i].real), (1j, gx[b, i].imag)):
                dy = u * col
                fd = float(np.sum(w[b] * (np.abs(Y[b] + h * dy) ** 2 - np.abs(Y[b] - h * dy) ** 2)) / (2 * h))
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (direction, norm, fd, an)


@pytest.mark.slow
@pytest.mark.parametrize("log_n", [6, 10, 12, 13, 16, 18, 20])
def test_full_size_roundtrip_and_parseval(log_n):
    # C2 size: 1 GiB of complex64 per buffer, N(0,1) seed 1 — size-independent
    # properties: Parseval and forward->inverse round trip
    n = 1 << log_n
    b = (1 << 27) // n
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(b * 2 * n, device="cuda", generator=g)
    y = torch.empty_like(x)
    unit = fft_unit(n)
    unit.exec(y, x, batch=b)
    ex = (x.double() ** 2).view(b, -1).sum(1)
    ey = (y.double() ** 2).view(b, -1).sum(1) / n
    assert torch.max(torch.abs(ey / ex - 1)).item() < 1e-5
    unit.exec(y, y, batch=b, direction=1)
    err = torch.linalg.norm((y - x).double()) / torch.linalg.norm(x.double())
    assert err.item() < 2e-6
    # the first rows against the oracle
    rows = x[: 2 * n * min(b, 2)].cpu().numpy().reshape(-1, 2 * n)
    got = torch.empty(rows.size, device="cuda")
    unit.exec(got, to_dev(rows, F32), batch=rows.shape[0])
    want = O.fft_packed(rows, n)
    assert rel_l2(O.unpack(got.cpu().numpy().reshape(rows.shape), n, 8), O.unpack(want, n, 8)) < 2e-6


@pytest.mark.parametrize("log_n,batch", [(14, 1), (14, 300), (15, 37), (16, 64), (17, 5), (18, 9), (19, 3), (20, 6),
                                         (20, 1)])
@pytest.mark.parametrize("dtype", [F32, F64])
def test_one_launch_four_step_matches_chunked(log_n, batch, dtype, monkeypatch):
    """The one-launch four-step (all chunks in one persistent grid, device
    dependency counters, a copy warp per CTA) against the chunked two-launch
    pipeline: the same arithmetic, so bit-identical, and both against the
    oracle on a few rows."""
    n = 1 << log_n
    if dtype == F64 and batch > 16:
        batch = 16
    p = 8 if dtype == F32 else 4
    rng = np.random.default_rng(300 + log_n)
    z = normal_cx(rng, batch, n)
    x = O.pack(z, p, NPD[dtype])
    unit = fft_unit(n, dtype=dtype)
    # the chunked passes use the plan's own split (the longer sub-transform
    # first); the one-launch kernel is pinned to a variant of that split, so
    # the arithmetic is the same
    l1, l2 = (log_n + 1) // 2, log_n // 2
    v = next(v for v in _variants() if v[0] == dtype and v[1:3] == (l1, l2))
    unit.set_tuning("one-launch four-step", split=(1 << l1, 1 << l2), blocks_per_sm=v[3], stages=v[4])
    outs = {}
    for mode in ("chunked", "one-launch"):
        if mode == "chunked":
            monkeypatch.setenv("PCX_FOURSTEP", "chunked")
        else:
            monkeypatch.delenv("PCX_FOURSTEP", raising=False)
        fwd = run(unit, x, batch, direction=0)
        inv = run(unit, fwd, batch, direction=1)
        outs[mode] = (fwd, inv)
        unit.status()
    assert np.array_equal(outs["chunked"][0], outs["one-launch"][0])
    assert np.array_equal(outs["chunked"][1], outs["one-launch"][1])
    k = min(batch, 2)
    want = O.fft_packed(x[:k], n, pack_src=p, pack_dst=p, dtype=NPD[dtype])
    tol = TOL[NPD[dtype]]
    assert rel_l2(O.unpack(outs["one-launch"][0][:k], n, p), O.unpack(want, n, p)) < tol
    assert rel_l2(O.unpack(outs["one-launch"][1], n, p), z) < tol


@pytest.mark.parametrize("log_n,batch", [(13, 64), (14, 40), (16, 8), (20, 3)])
def test_tune_picks_a_form_and_keeps_parity(log_n, batch):
    """pcx_plan_tune times the forms of the size and keeps the fastest; the
    transform stays within the FP32 bar of the oracle whatever it picked."""
    n = 1 << log_n
    unit = fft_unit(n, dtype=F32)
    form = unit.tune(batch)
    assert re.match(r"(one-pass|one-launch four-step \d+x\d+|chunked four-step)\b", form), form
    rng = np.random.default_rng(400 + log_n)
    z = normal_cx(rng, batch, n)
    x = O.pack(z, 8)
    got = run(unit, x, batch, direction=0)
    unit.status()
    k = min(batch, 2)
    want = O.fft_packed(x[:k], n, pack_src=8, pack_dst=8)
    assert rel_l2(O.unpack(got[:k], n, 8), O.unpack(want, n, 8)) < TOL[np.float32]
    back = run(unit, got, batch, direction=1)
    assert rel_l2(O.unpack(back, n, 8), z) < TOL[np.float32]


def _variants():
    from packed_b200 import _lib as L
    import re
    text = (Path(__file__).resolve().parents[1] / "packed_b200" / "csrc" / "pcx_host.hpp").read_text()
    out = []
    for name, dt in (("kFsVariantsF32", F32), ("kFsVariantsF64", F64)):
        body = text[text.index(name):]
        body = body[: body.index("};")]
        out += [(dt, *map(int, m)) for m in re.findall(r"\{(\d+), (\d+), (\d+), (\d+)\}", body)]
    return out


@pytest.mark.parametrize("dtype,l1,l2,minb,st", _variants())
def test_every_fourstep_variant_matches_oracle(dtype, l1, l2, minb, st):
    """Every built-in variant of the one-launch four-step (split, blocks per
    SM, ring stages), chosen explicitly through pcx_plan_set_tuning, against
    the oracle: forward and inverse, a ragged batch."""
    n = 1 << (l1 + l2)
    p = 8 if dtype == F32 else 4
    batch = 5 if n <= (1 << 16) else 2
    rng = np.random.default_rng(l1 * 100 + l2 * 10 + minb + st)
    z = normal_cx(rng, batch, n)
    x = O.pack(z, p, NPD[dtype])
    unit = fft_unit(n, dtype=dtype)
    unit.set_tuning("one-launch four-step", split=(1 << l1, 1 << l2), blocks_per_sm=minb, stages=st, rounds=2)
    t = unit.tuning()
    assert t["split"] == [1 << l1, 1 << l2] and t["blocks_per_sm"] == minb and t["stages"] == st
    fwd = run(unit, x, batch, direction=0)
    back = run(unit, fwd, batch, direction=1)
    unit.status()
    tol = TOL[NPD[dtype]]
    want = np.fft.fft(z, axis=-1)
    assert rel_l2(O.unpack(fwd, n, p), want) < tol
    assert rel_l2(O.unpack(back, n, p), z) < tol


def test_set_tuning_rejects_unbuilt_variant():
    unit = fft_unit(1 << 16)
    with pytest.raises(NotImplementedError):
        unit.set_tuning("one-launch four-step", split=(1024, 64), blocks_per_sm=1, stages=3)


def test_tune_small_size_has_one_form():
    assert fft_unit(1024).tune(16) == "default"


@pytest.mark.parametrize("n,length,pd,ps,dtype", [(64, 37, 8, 8, F32), (1024, 100, 1, 8, F32), (16384, 9, 8, 2, F32),
                                                  (8, 5, 4, 4, F32), (256, 33, 4, 1, F64)])
def test_fft_unit_par_across_vectors(n, length, pd, ps, dtype):
    """fft_unit_par (reference fft.hpp:2167): for every element position p the
    n-point transform runs across the n vectors; checked against numpy's FP64
    FFT along that axis, forward and normalised inverse, mixed pack widths."""
    from packed_b200 import fft_unit_par
    npd = np.float64 if dtype == F64 else np.float32
    rng = np.random.default_rng(500 + n + length)
    z = normal_cx(rng, n, length)
    src = [vector.from_complex(z[i], dtype=dtype, pack=ps) for i in range(n)]
    dst = [vector(length, dtype=dtype, pack=pd) for _ in range(n)]
    unit = fft_unit_par(n, dtype=dtype)
    unit(dst, src)
    torch.cuda.synchronize()
    got = np.stack([v.to_complex() for v in dst])
    want = np.fft.fft(z, axis=0)
    assert rel_l2(got, want) < TOL[npd]
    back = [vector(length, dtype=dtype, pack=ps) for _ in range(n)]
    unit(back, dst, inverse=True)
    torch.cuda.synchronize()
    assert rel_l2(np.stack([v.to_complex() for v in back]), z) < TOL[npd]


def test_fft_unit_par_errors():
    from packed_b200 import fft_unit_par
    unit = fft_unit_par(16)
    with pytest.raises(ValueError, match="is not equal to fft size"):
        unit([vector(4) for _ in range(15)], [vector(4) for _ in range(16)])


@pytest.mark.parametrize("dtype", [F32, F64])
def test_vector_expressions_on_device(dtype):
    """pcxo::vector expression templates (reference vector_arithm.hpp:405-1140,
    the binary-operator table of tests/test_op.cpp:116-131): +, -, *, / between
    vectors and scalars and conj, evaluated on the device (pcx_vec_eval), mixed
    pack widths, against numpy."""
    from packed_b200 import conj
    npd = np.float64 if dtype == F64 else np.float32
    rng = np.random.default_rng(600)
    n = 1000
    za, zb, zc = (normal_cx(rng, n) for _ in range(3))
    zb += 2.0    # keep divisors away from zero
    a = vector.from_complex(za, dtype=dtype, pack=8 if dtype == F32 else 4)
    b = vector.from_complex(zb, dtype=dtype, pack=1)
    c = vector.from_complex(zc, dtype=dtype, pack=2)
    s = 0.5 - 1.5j
    cases = [
        (lambda: a + b, za + zb), (lambda: a - b, za - zb), (lambda: a * b, za * zb), (lambda: a / b, za / zb),
        (lambda: a + conj(b), za + np.conj(zb)), (lambda: conj(a) * b, np.conj(za) * zb),
        (lambda: conj(a) / conj(b), np.conj(za) / np.conj(zb)), (lambda: a * s + c, za * s + zc),
        (lambda: s / b - conj(c * a), s / zb - np.conj(zc * za)), (lambda: (a + b) * (a - c) / (b * b), (za + zb) * (za - zc) / (zb * zb)),
    ]
    out = vector(n, dtype=dtype, pack=4)
    for expr, want in cases:
        out.assign(expr())
        torch.cuda.synchronize()
        assert rel_l2(out.to_complex(), want) < TOL[npd]
    a.assign(a * a)    # destination among the operands, same pack
    torch.cuda.synchronize()
    assert rel_l2(a.to_complex(), za * za) < TOL[npd]
    with pytest.raises(ValueError, match="not equal to subrange size"):
        out.assign(a + vector(n + 1, dtype=dtype))


@pytest.mark.parametrize("n", [8192, 1 << 14, 1 << 17])
def test_pack16_two_pass_sizes(n):
    """Pack widths above the four-step kernels' own (8 reals for float, 4 for
    double) are repacked around the transform: FP32 and FP64, in place and
    out of place, forward and inverse."""
    rng = np.random.default_rng(16)
    b = 2
    z = normal_cx(rng, b, n)
    want = np.fft.fft(z, axis=-1)
    for dt, npd, packs in ((F32, np.float32, ((16, 16), (16, 4), (2, 16))), (F64, np.float64, ((8, 8), (16, 4), (4, 16)))):
        unit = fft_unit(n, dtype=dt)
        tol = TOL[npd]
        for ps, pd in packs:
            x = to_dev(O.pack(z, ps, npd), dt)
            y = torch.empty((b, real_size(n, pd)), dtype=dt, device="cuda")
            unit.exec(y, x, batch=b, pack_src=ps, pack_dst=pd)
            assert rel_l2(O.unpack(y.cpu().numpy(), n, pd), want) < tol, (dt, ps, pd)
            back = torch.empty((b, real_size(n, ps)), dtype=dt, device="cuda")
            unit.exec(back, y, batch=b, direction=1, pack_src=pd, pack_dst=ps)
            assert rel_l2(O.unpack(back.cpu().numpy(), n, ps), z) < tol, (dt, ps, pd)
            if ps == pd:    # in place
                unit.exec(x, x, batch=b, pack_src=ps, pack_dst=pd)
                assert rel_l2(O.unpack(x.cpu().numpy(), n, pd), want) < tol, (dt, ps, pd)
        with pytest.raises(NotImplementedError, match="pack sizes above 16"):
            big = torch.zeros(2 * n, dtype=dt, device="cuda")
            unit.exec(big, big, pack_src=32, pack_dst=32)
