"""The CPU oracle pinned against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference headers) and against
direct FP64/long-double sums.  CPU only."""
import numpy as np
import pytest

import oracle as O
from tests._util import TOL, golden, normal_cx, rel_l2

G = golden()

# The reference fft_unit<float> is within ~3e-7 of the exact DFT; its
# difference from the double-precision oracle is bounded by the FP32 bar.
REF_TOL = TOL[np.float32]


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_oracle_forward_matches_reference(n, order):
    x = G[f"x_{n}"]
    got = O.fft_packed(x, n, order=order, direction=0)
    assert rel_l2(O.unpack(got, n, 8), O.unpack(G[f"fwd_{n}_o{order}"], n, 8)) < REF_TOL


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_oracle_inverse_matches_reference(n, order):
    y = G[f"fwd_{n}_o{order}"]
    got = O.fft_packed(y, n, order=order, direction=1, normalize=True)
    assert rel_l2(O.unpack(got, n, 8), O.unpack(G[f"inv_{n}_o{order}"], n, 8)) < REF_TOL
    if order:
        raw = O.fft_packed(y, n, order=order, direction=1, normalize=False)
        assert rel_l2(O.unpack(raw, n, 8), O.unpack(G[f"invraw_{n}_o{order}"], n, 8)) < REF_TOL


def test_oracle_large_and_tone():
    n = 16384
    got = O.fft_packed(G[f"x_{n}"], n)
    assert rel_l2(O.unpack(got, n, 8), O.unpack(G[f"fwd_{n}_o0"], n, 8)) < REF_TOL
    got = O.fft_packed(G["tone_x_1024"], 1024)
    assert rel_l2(O.unpack(got, 1024, 8), O.unpack(G["tone_fwd_1024"], 1024, 8)) < REF_TOL


def test_oracle_zero_extension():
    got = O.fft_packed(G["zx_src_700"], 1024, order=1, src_len=700)
    assert rel_l2(O.unpack(got, 1024, 8), O.unpack(G["zx_fwd_1024_o1"], 1024, 8)) < REF_TOL


def test_oracle_c1_rows():
    rng = np.random.default_rng(0)
    c1 = np.stack([(rng.uniform(-1, 1, 1024) + 1j * rng.uniform(-1, 1, 1024)).astype(np.complex64)
                   for _ in range(64)])
    x = O.pack(c1[:4], 8)
    np.testing.assert_array_equal(x, G["c1_x"])    # same generator, same bits
    fwd = O.fft_packed(x, 1024)
    inv = O.fft_packed(G["c1_fwd"], 1024, direction=1)
    assert rel_l2(O.unpack(fwd, 1024, 8), O.unpack(G["c1_fwd"], 1024, 8)) < REF_TOL
    assert rel_l2(O.unpack(inv, 1024, 8), O.unpack(G["c1_inv"], 1024, 8)) < REF_TOL


def test_unordered_permutation_is_the_references():
    # position p of an unordered forward output holds frequency bitrev(sigma(p))
    for n in (64, 256, 1024, 4096):
        pos = O.order_pos(n, 2)
        z = O.unpack(G[f"x_{n}"], n, 8)
        nat = np.fft.fft(z)
        ref = O.unpack(G[f"fwd_{n}_o2"], n, 8)
        assert rel_l2(ref[pos], nat) < REF_TOL


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref (the reference compiled here) not built")
@pytest.mark.parametrize("sub", [64, 128, 512, 4096])
@pytest.mark.parametrize("order", [1, 2])
def test_order_permutation_does_not_depend_on_sub_size(order, sub):
    # The reference's unordered (and bit_reversed) output order, run through
    # the reference itself at several sub_size values: position p holds
    # frequency bitrev(sigma(p)) (bitrev(p)) whatever the sub_size, which is
    # what order_pos implements and the GPU kernels use.
    rng = np.random.default_rng(sub + order)
    for n in (64, 256, 1024, 4096, 16384, 32768):
        z = normal_cx(rng, n)
        got = O.unpack(O.ref_fft(O.pack(z, 8), n, order, 0, True, sub), n, 8)
        assert rel_l2(got[O.order_pos(n, order)], np.fft.fft(z)) < REF_TOL


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128])
def test_oracle_fft_matches_direct_dft(n):
    rng = np.random.default_rng(n)
    z = normal_cx(rng, n)
    assert rel_l2(O.fft(z), O.dft(z)) < 1e-14
    assert rel_l2(O.fft(z, inverse=True), O.dft(z, inverse=True)) < 1e-14


def test_xcorr_single_block_matches_reference():
    for tag, k, n, s in (("xc1", 128, 256, 128), ("xc2", 512, 1024, 512)):
        x = O.unpack(G[f"{tag}_x"], s, 8)
        g = O.unpack(G[f"{tag}_g"], k, 8)
        y = O.xcorr_direct(x, g)
        assert rel_l2(O.unpack(G[f"{tag}_y"], s, 8), y) < 1e-5


def test_xcorr_multi_block_matches_corrected_reference():
    x = O.unpack(G["xc3_x"], 3000, 8)
    g = O.unpack(G["xc3_g"], 100, 8)
    y = O.xcorr_direct(x, g)
    assert rel_l2(O.xcorr_ols(x, g, 512), y) < 1e-13
    assert rel_l2(O.unpack(G["xc3_y"], 3000, 8), y) < REF_TOL
    # the shipped fxcorr_unit is wrong past the first block (fxcorr.hpp:112-129)
    assert rel_l2(O.unpack(G["xc3_y_shipped"], 3000, 8), y) > 0.1


def test_xcorr_vjp_matches_finite_differences():
    rng = np.random.default_rng(7)
    s, k = 200, 17
    x, g = normal_cx(rng, s), normal_cx(rng, k)
    w = rng.uniform(0, 1, s)

    def loss(x_, g_):
        y = O.xcorr_direct(x_, g_)
        return float(np.sum(w * np.abs(y) ** 2))

    y = O.xcorr_direct(x, g)
    gy = 2 * w * y    # d/dRe + i d/dIm of sum w |y|^2
    gx, gg = O.xcorr_vjp_direct(x, g, gy)
    h = 1e-6
    for idx in rng.integers(0, s, 5):
        for part, unit in ((0, 1.0), (1, 1j)):
            xp, xm = x.copy(), x.copy()
            xp[idx] += h * unit
            xm[idx] -= h * unit
            fd = (loss(xp, g) - loss(xm, g)) / (2 * h)
            an = gx[idx].real if part == 0 else gx[idx].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))
    for idx in rng.integers(0, k, 5):
        for part, unit in ((0, 1.0), (1, 1j)):
            gp, gm = g.copy(), g.copy()
            gp[idx] += h * unit
            gm[idx] -= h * unit
            fd = (loss(x, gp) - loss(x, gm)) / (2 * h)
            an = gg[idx].real if part == 0 else gg[idx].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def test_pack_layout_roundtrip():
    rng = np.random.default_rng(3)
    for p in (1, 2, 4, 8, 16):
        for n in (5, 16, 33):
            z = normal_cx(rng, n)
            a = O.pack(z, p)
            assert a.shape[-1] == O.real_size(n, p)
            np.testing.assert_allclose(O.unpack(a, n, p), z.astype(np.complex64))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n", [64, 1024, 16384])
def test_oracle_pack_conversions_match_reference(n):
    """The reference's own fft_raw<PD, PS> (its pack conversions in the FFT's
    loads and stores) against the oracle, natural and bit-reversed order."""
    rng = np.random.default_rng(n + 3)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for order in (0, 1):
        for ps, pd in ((1, 8), (8, 1), (2, 4), (4, 2), (1, 1), (2, 8)):
            x = O.pack(z, ps)
            got = O.ref_fft_raw_packs(x, n, pd, ps, order=order)
            want = O.fft_packed(x, n, order=order, pack_src=ps, pack_dst=pd)
            assert rel_l2(O.unpack(got, n, pd), O.unpack(want, n, pd)) < REF_TOL, (order, ps, pd)
