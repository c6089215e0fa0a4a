"""GPU parity of the fused overlap-save correlator and its adjoint against the
CPU oracle (direct FP64 sums, overlap-save restatement) and the reference's
golden outputs."""
import numpy as np
import pytest
import torch

import oracle as O
from packed_b200 import fxcorr_unit, real_size, vector
from packed_b200.autograd import FxcorrFunction
from tests._util import TOL, golden, normal_cx, rel_l2

pytestmark = pytest.mark.gpu

F32, F64 = torch.float32, torch.float64


def dev(a, dtype=F32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).cuda()


def corr(z, g, n_fft, pack=8, inplace=True, dtype=F32, channels=1):
    npd = np.float32 if dtype == F32 else np.float64
    s = z.shape[-1]
    unit = fxcorr_unit(vector.from_complex(g, dtype=dtype), n_fft)
    x = dev(O.pack(z, pack, npd), dtype)
    y = x if inplace else torch.full_like(x, float("nan"))
    unit.exec(y, x, s, channels=channels, pack=pack)
    torch.cuda.synchronize()
    if inplace:
        unit.status()
    return O.unpack(y.cpu().numpy(), s, pack)


def test_reference_single_block_golden():
    G = golden()
    for tag, k, n, s in (("xc1", 128, 256, 128), ("xc2", 512, 1024, 512)):
        z, g = O.unpack(G[f"{tag}_x"], s, 8), O.unpack(G[f"{tag}_g"], k, 8)
        got = corr(z, g, n)
        assert rel_l2(got, O.unpack(G[f"{tag}_y"], s, 8)) < 1e-5
        assert rel_l2(got, O.xcorr_direct(z, g)) < TOL[np.float32]


def test_multi_block_against_corrected_reference():
    G = golden()
    z, g = O.unpack(G["xc3_x"], 3000, 8), O.unpack(G["xc3_g"], 100, 8)
    got = corr(z, g, 512)
    assert rel_l2(got, O.unpack(G["xc3_y"], 3000, 8)) < TOL[np.float32]
    assert rel_l2(got, O.xcorr_direct(z, g)) < TOL[np.float32]


@pytest.mark.parametrize("s,k,n", [(1, 1, 64), (100, 13, 64), (777, 60, 128), (5000, 200, 1024), (4096, 1, 256),
                                   (20000, 1000, 2048), (33333, 3000, 4096), (70000, 4000, 8192),
                                   (100000, 4096, 16384), (50000, 12000, 16384)])
@pytest.mark.parametrize("inplace", [True, False])
def test_against_direct_sum(s, k, n, inplace):
    rng = np.random.default_rng(s + k)
    z, g = normal_cx(rng, s), normal_cx(rng, k, sigma=1 / np.sqrt(k))
    got = corr(z, g, n, inplace=inplace)
    want = O.xcorr_ols(z, g, n) if s * k > 5e7 else O.xcorr_direct(z, g)
    assert rel_l2(got, want) < TOL[np.float32]


@pytest.mark.parametrize("pack", [1, 2, 4, 8, 16])
def test_pack_widths_and_channels(pack):
    rng = np.random.default_rng(pack)
    ch, s, k, n = 3, 3001, 77, 512
    z, g = normal_cx(rng, ch, s), normal_cx(rng, k)
    unit = fxcorr_unit(vector.from_complex(g), n)
    x = dev(O.pack(z, pack))
    unit.exec(x, x, s, channels=ch, pack=pack)
    got = O.unpack(x.cpu().numpy(), s, pack)
    for c in range(ch):
        assert rel_l2(got[c], O.xcorr_direct(z[c], g)) < TOL[np.float32]


def test_fp64():
    rng = np.random.default_rng(64)
    z, g = normal_cx(rng, 20000), normal_cx(rng, 700)
    got = corr(z, g, 2048, pack=4, dtype=F64)
    assert rel_l2(got, O.xcorr_ols(z, g, 2048, 4)) < TOL[np.float64]


def test_c3_shape_reduced_channels():
    # C3 parameters (K=4096, N_fft=16384, step 12288) on 4 channels of 2^18
    rng = np.random.default_rng(2)
    ch, s, k, n = 4, 1 << 18, 4096, 16384
    z = normal_cx(rng, ch, s).astype(np.complex64)
    g = normal_cx(rng, k, sigma=1 / 64).astype(np.complex64)
    unit = fxcorr_unit(vector.from_complex(g), n)
    assert unit.step() == 12288
    x = dev(O.pack(z, 8))
    unit.exec(x, x, s, channels=ch)
    unit.status()
    got = O.unpack(x.cpu().numpy(), s, 8)
    for c in range(ch):
        assert rel_l2(got[c], O.xcorr_ols(z[c], g, n)) < TOL[np.float32]


@pytest.mark.slow
def test_c3_full_size_all_channels():
    """Full C3 (256 channels x 2^20, K 4096, N_fft 16384, in place): every
    output of every channel against an FP64 reference computed on the device
    from the same FP32 inputs (linear correlation by a 2^21-point torch.fft in
    complex128, the checker); each channel within the FP32 bar of 2e-6
    relative L2."""
    ch, s, k, n = 256, 1 << 20, 4096, 16384
    gen = torch.Generator(device="cuda").manual_seed(2)
    x = torch.randn(ch * 2 * s, device="cuda", generator=gen)
    rng = np.random.default_rng(3)
    g = normal_cx(rng, k, sigma=1 / 64).astype(np.complex64)
    unit = fxcorr_unit(vector.from_complex(g), n)
    orig = x.clone()
    unit.exec(x, x, s, channels=ch)
    unit.status()

    def rows(t, m):    # pack-8 rows -> complex128 [rows, m]
        v = t.reshape(-1, m // 8, 2, 8).double()
        return torch.complex(v[:, :, 0, :].reshape(-1, m), v[:, :, 1, :].reshape(-1, m))

    L = 1 << 21    # >= s + k - 1: the circular correlation is the linear one on [0, s)
    gs = torch.conj(torch.fft.fft(torch.as_tensor(g.astype(np.complex128), device="cuda"), L))
    worst = 0.0
    for c0 in range(0, ch, 16):
        want = torch.fft.ifft(torch.fft.fft(rows(orig[c0 * 2 * s:(c0 + 16) * 2 * s], s), L) * gs)[:, :s]
        got = rows(x[c0 * 2 * s:(c0 + 16) * 2 * s], s)
        err = torch.linalg.vector_norm(got - want, dim=-1) / torch.linalg.vector_norm(want, dim=-1)
        worst = max(worst, float(err.max()))
        assert float(err.max()) < TOL[np.float32], (c0, float(err.max()))
    print(f"C3 full size: worst channel relative L2 {worst:.3g}")


def test_vjp_against_oracle():
    rng = np.random.default_rng(11)
    ch, s, k, n = 2, 9000, 300, 1024
    z, g = normal_cx(rng, ch, s), normal_cx(rng, k)
    gy = normal_cx(rng, ch, s)
    unit = fxcorr_unit(vector.from_complex(g), n)
    gx, gg = unit.vjp(dev(O.pack(gy, 8)), dev(O.pack(z, 8)), s, channels=ch)
    gx = O.unpack(gx.cpu().numpy(), s, 8)
    gg = O.unpack(gg.cpu().numpy(), k, 8)
    gg_want = np.zeros(k, complex)
    for c in range(ch):
        gxw, ggw = O.xcorr_vjp_direct(z[c], g, gy[c])
        assert rel_l2(gx[c], gxw) < TOL[np.float32]
        gg_want += ggw
    assert rel_l2(gg, gg_want) < TOL[np.float32]


def _c3_like_problem(dtype, s=1 << 16, k=4096):
    """One channel with C3's kernel shape and distributions: signal N(0,1)
    (seed 2), kernel N(0,1/4096) (seed 3), loss weight U[0,1) (seed 6)."""
    z = normal_cx(np.random.default_rng(2), s)
    g = normal_cx(np.random.default_rng(3), k, sigma=1 / 64)
    w = np.random.default_rng(6).uniform(0, 1, s)
    if dtype == F32:    # the FP64 side sees exactly the FP32 inputs
        z, g = z.astype(np.complex64).astype(complex), g.astype(np.complex64).astype(complex)
    return z, g, w


def _autograd_grads(z, g, w, n, dtype):
    """d(sum w |y|^2)/dx and /dg through FxcorrFunction (pcx_fxcorr_vjp)."""
    s, k = z.size, g.size
    p = 8 if dtype == F32 else 4
    npd = np.float32 if dtype == F32 else np.float64
    x = dev(O.pack(z, p, npd), dtype).requires_grad_(True)
    gt = dev(O.pack(g, p, npd), dtype).requires_grad_(True)
    y = FxcorrFunction.apply(x, gt, n, s, k, 1)
    wt = dev(O.pack(w.astype(complex), p, npd), dtype)
    wr = wt.clone()
    wr.view(-1, 2, p)[:, 1, :] = wt.view(-1, 2, p)[:, 0, :]    # weight both re and im
    (wr * y * y).sum().backward()
    return O.unpack(x.grad.cpu().numpy(), s, p), O.unpack(gt.grad.cpu().numpy(), k, p)


def _central_fd(z, g, w, n, coords_x, coords_g, h=1e-6):
    """FP64 central finite differences (step h) of L = sum w |y|^2, y the
    correlation of z with g, at the given signal and kernel coordinates, in
    the real and the imaginary direction.  y is linear in z and in conj(g), so
    the perturbed outputs are formed exactly as y +- h*dy (dy the outputs'
    change per unit step, from the definition y[m] = sum_j z[m+j] conj(g[j])),
    and L(+h) - L(-h) is summed term by term over the affected outputs: the
    difference quotient then carries ~1e-9 of rounding noise instead of the
    ~1e-6 that subtracting two separately summed losses of ~3e4 would."""
    s, k = z.size, g.size
    y = O.xcorr_ols(z, g, n)

    def fd(lo, dy):
        yy, ww = y[lo:lo + dy.size], w[lo:lo + dy.size]
        return float(np.sum(ww * (np.abs(yy + h * dy) ** 2 - np.abs(yy - h * dy) ** 2)) / (2 * h))

    out_x, out_g = [], []
    for i in coords_x:
        lo = max(0, i - k + 1)
        m = np.arange(lo, i + 1)
        for u in (1.0, 1j):
            out_x.append(fd(lo, u * np.conj(g[i - m])))
    for j in coords_g:
        m = np.arange(0, s - j)
        for u in (1.0, 1j):
            out_g.append(fd(0, z[m + j] * np.conj(u)))
    return np.array(out_x), np.array(out_g)


def _parts(v, coords):
    return np.array([c for i in coords for c in (v[i].real, v[i].imag)])


def test_adjoint_fp64_vs_central_fd():
    """FP64 correlator (K = 4096, N_fft = 8192: the largest FP64 correlator
    size) against FP64 central finite differences at 64 signal and 64 kernel
    coordinates: |fd - grad| <= 1e-6 * max(1, |fd|), nothing added."""
    n = 8192
    z, g, w = _c3_like_problem(F64)
    gx, gg = _autograd_grads(z, g, w, n, F64)
    rng = np.random.default_rng(64)
    cx, cg = rng.integers(0, z.size, 64), rng.integers(0, g.size, 64)
    fdx, fdg = _central_fd(z, g, w, n, cx, cg)
    for fd, an in ((fdx, _parts(gx, cx)), (fdg, _parts(gg, cg))):
        assert np.all(np.abs(fd - an) <= 1e-6 * np.maximum(1.0, np.abs(fd))), np.max(np.abs(fd - an))
    # and the whole gradients against the FP64 reference gradient (direct sums)
    yd = O.xcorr_direct(z, g)
    gxw, ggw = O.xcorr_vjp_direct(z, g, 2 * w * yd)
    assert rel_l2(gx, gxw) < 1e-12 and rel_l2(gg, ggw) < 1e-12


def test_adjoint_fp32_c3_vs_central_fd():
    """FP32 correlator at C3's shape (K = 4096, N_fft = 16384) against the same
    FP64 central differences.  An FP32 gradient carries the FP32 parity error
    (relative L2 <= 2e-6 of the gradient vector), so each coordinate is held to
    |fd - grad| <= 2e-5 * rms(grad): ten times the vector bar, per coordinate."""
    n = 16384
    z, g, w = _c3_like_problem(F32)
    gx, gg = _autograd_grads(z, g, w, n, F32)
    rng = np.random.default_rng(64)
    cx, cg = rng.integers(0, z.size, 64), rng.integers(0, g.size, 64)
    fdx, fdg = _central_fd(z, g, w, n, cx, cg)
    for fd, full, an in ((fdx, gx, _parts(gx, cx)), (fdg, gg, _parts(gg, cg))):
        rms = np.sqrt(np.mean(np.abs(full) ** 2))
        assert np.all(np.abs(fd - an) <= 2e-5 * rms), np.max(np.abs(fd - an)) / rms
    yd = O.xcorr_direct(z, g)
    gxw, ggw = O.xcorr_vjp_direct(z, g, 2 * w * yd)
    assert rel_l2(gx, gxw) < TOL[np.float32] and rel_l2(gg, ggw) < TOL[np.float32]


def test_errors():
    g = vector.from_complex(np.ones(100))
    with pytest.raises(ValueError, match="power of two"):
        fxcorr_unit(g, 1000)
    with pytest.raises(ValueError):
        fxcorr_unit(g, 64)
    unit = fxcorr_unit(g, 128)
    x = torch.zeros(real_size(100, 8), device="cuda")
    with pytest.raises(ValueError):
        unit.exec(x, x, 100, pack=3)


@pytest.mark.parametrize("n,s,k,ch,inplace", [(16384, 100000, 4096, 1, True), (16384, 12288 * 3, 4096, 3, False),
                                              (16384, 5000, 64, 2, True), (8192, 70001, 4000, 2, True),
                                              (8192, 8191, 1, 1, False), (16384, 1 << 17, 9, 4, True)])
def test_four_step_form_matches_general_kernel(n, s, k, ch, inplace, monkeypatch):
    """FP32 correlators of 2^13 and 2^14 points run as a four-step inside each
    CTA; the general one-pass kernel (selected at creation by PCX_XC_GENERAL)
    and the overlap-save oracle must agree with it, on ragged lengths, several
    channels, in and out of place."""
    rng = np.random.default_rng(n + s + k)
    z = normal_cx(rng, ch, s).astype(np.complex64)
    g = normal_cx(rng, k, sigma=1 / 64).astype(np.complex64)
    got = corr(z, g, n, inplace=inplace, channels=ch)
    monkeypatch.setenv("PCX_XC_GENERAL", "1")
    ref = corr(z, g, n, inplace=inplace, channels=ch)
    for c in range(ch):
        want = O.xcorr_ols(z[c], g, n)
        assert rel_l2(got[c], want) < TOL[np.float32]
        assert rel_l2(ref[c], want) < TOL[np.float32]
        assert rel_l2(got[c], ref[c]) < TOL[np.float32]


@pytest.mark.parametrize("n,s,k,ch", [(16384, 40000, 4096, 2), (16384, 30001, 4097, 1), (16384, 9000, 12000, 3),
                                      (8192, 30000, 4000, 2), (8192, 20000, 9, 1), (16384, 16384, 1, 1),
                                      (16384, 100, 300, 2)])
def test_adjoint_four_step_form(n, s, k, ch, monkeypatch):
    """Both halves of the adjoint at 2^13 and 2^14 points run in the in-CTA
    four-step form: the signal gradient (a convolution with the kernel, its
    windows starting K-1 rounded up to whole packs before each block) and the
    kernel gradient (per-thread block spectra kept in tensor memory).  They
    must agree with the general kernels (PCX_XC_GENERAL at creation) and the
    direct-sum oracle."""
    rng = np.random.default_rng(n + s + k + 1)
    z = normal_cx(rng, ch, s).astype(np.complex64)
    g = normal_cx(rng, k, sigma=1 / 64).astype(np.complex64)
    gy = normal_cx(rng, ch, s).astype(np.complex64)
    dz, dgy = dev(np.stack([O.pack(r, 8) for r in z])), dev(np.stack([O.pack(r, 8) for r in gy]))

    def grads():
        unit = fxcorr_unit(vector.from_complex(g), n)
        gx, gg = unit.vjp(dgy, dz, s, channels=ch)
        torch.cuda.synchronize()
        unit.status()
        return [O.unpack(r, s, 8) for r in gx.cpu().numpy()], O.unpack(gg.cpu().numpy(), k, 8)

    got_x, got_g = grads()
    monkeypatch.setenv("PCX_XC_GENERAL", "1")
    ref_x, ref_g = grads()
    want_g = np.zeros(k, complex)
    for c in range(ch):
        want_x, wg = O.xcorr_vjp_direct(z[c], g, gy[c])
        want_g += wg
        assert rel_l2(got_x[c], want_x) < TOL[np.float32], c
        assert rel_l2(ref_x[c], want_x) < TOL[np.float32], c
        assert rel_l2(got_x[c], ref_x[c]) < TOL[np.float32], c
    assert rel_l2(got_g, want_g) < TOL[np.float32]
    assert rel_l2(ref_g, want_g) < TOL[np.float32]
    assert rel_l2(got_g, ref_g) < TOL[np.float32]
