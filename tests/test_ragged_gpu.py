"""Ragged persistent batch (one launch, device work queue, CUDA graph):
every transform and correlation checked against the CPU oracle, on two
replays of the graph."""
import numpy as np
import pytest
import torch

import oracle as O
from packed_b200 import fft_unit, ragged_batch, vector
from tests._util import TOL, normal_cx, rel_l2

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("seed", [5, 6])
def test_ragged_batch_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    sizes = [1 << int(v) for v in rng.integers(5, 19, 40)] + [1 << 18, 1 << 13, 1 << 12, 1 << 5]
    zs, ffts = [], []
    for n in sizes:
        z = normal_cx(rng, n)
        zs.append(z)
        ffts.append((torch.full((2 * n,), float("nan"), device="cuda"), dev(O.pack(z, 8)), n))
    xcs, xin = [], []
    # correlations of 128..8192 points (on the ring) and one of 16384 points
    # (its own path through the whole ring); the fixed ones give 4096-point
    # items with a zero second window (3 blocks; 1 block) and an 8192-point one
    fixed = [(50000, 5000, 16384), (7676, 1500, 4096), (1200, 1100, 4096), (20000, 3000, 8192)]
    for q in range(6 + len(fixed)):
        if q < 6:
            s, k = int(2 ** rng.uniform(12, 17)), int(2 ** rng.uniform(6, 12))
            nf = max(128, 1 << int(np.ceil(np.log2(2 * k))))
        else:
            s, k, nf = fixed[q - 6]
        x, g = normal_cx(rng, s), normal_cx(rng, k)
        xin.append((x, g, nf))
        xcs.append((torch.full((len(O.pack(x, 8)),), float("nan"), device="cuda"), dev(O.pack(x, 8)), s,
                    vector.from_complex(g), nf))
    batch = ragged_batch(ffts, xcs)
    assert batch.items() > len(sizes)
    for replay in range(2):
        for d, _, _ in ffts:
            d.fill_(float("nan"))
        batch()
        torch.cuda.synchronize()
        batch.status()
        for (d, _, n), z in zip(ffts, zs):
            assert rel_l2(O.unpack(d.cpu().numpy(), n, 8), np.fft.fft(z)) < TOL[np.float32], (replay, n)
        for (d, _, s, _, nf), (x, g, _) in zip(xcs, xin):
            assert rel_l2(O.unpack(d.cpu().numpy(), s, 8), O.xcorr_ols(x, g, nf)) < TOL[np.float32], (replay, s)


def test_ragged_matches_plain_launch_bits():
    # same kernels' arithmetic as the per-size plain launches for N <= 4096 rows
    rng = np.random.default_rng(9)
    n = 1024
    z = normal_cx(rng, 5, n)
    src = [dev(O.pack(z[i], 8)) for i in range(5)]
    dst = [torch.empty_like(s) for s in src]
    ragged_batch([(dst[i], src[i], n) for i in range(5)])()
    ref = torch.empty(5 * 2 * n, device="cuda")
    fft_unit(n).exec(ref, torch.cat(src), batch=5)
    torch.cuda.synchronize()
    got = torch.cat(dst)
    assert rel_l2(O.unpack(got.cpu().numpy().reshape(5, -1), n, 8),
                  O.unpack(ref.cpu().numpy().reshape(5, -1), n, 8)) < TOL[np.float32]


def _unpack_rows(t: torch.Tensor, n: int) -> torch.Tensor:
    """Pack-8 rows of n points (n a multiple of 8) -> complex128 [rows, n], on the device."""
    v = t.reshape(-1, n // 8, 2, 8).double()
    return torch.complex(v[:, :, 0, :].reshape(-1, n), v[:, :, 1, :].reshape(-1, n))


def _row_rel_l2(got: torch.Tensor, want: torch.Tensor) -> torch.Tensor:
    return torch.linalg.vector_norm(got - want, dim=-1) / torch.linalg.vector_norm(want, dim=-1)


def test_full_c5_scale_against_fp64():
    """The full C5 configuration (10,000 FFTs of 2^8..2^18 points and 500
    correlations, seed 5, as the benchmark builds it) in one graph replay,
    every transform and every correlation against an FP64 reference computed
    on the device from the same FP32 inputs (torch.fft as the checker): each
    one within the FP32 bar of 2e-6 relative L2."""
    from packed_b200 import correlation_fft_size

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    lgs = np.floor(rng.uniform(8, 19, 10000)).astype(int)
    groups, ffts = {}, []
    for lg in sorted(set(lgs.tolist())):
        cnt, n = int((lgs == lg).sum()), 1 << lg
        src = torch.randn(cnt * 2 * n, device=dev)
        dst = torch.full_like(src, float("nan"))
        groups[lg] = (cnt, src, dst)
        ffts += [(dst[i * 2 * n:(i + 1) * 2 * n], src[i * 2 * n:(i + 1) * 2 * n], n) for i in range(cnt)]
    s_all = np.floor(2 ** rng.uniform(12, 20, 500)).astype(int) // 8 * 8
    k_all = np.floor(2 ** rng.uniform(6, 13, 500)).astype(int)
    xcs = []
    for s, k in zip(s_all, k_all):
        taps = vector.from_complex(rng.standard_normal(k) + 1j * rng.standard_normal(k), device=dev)
        x = torch.randn(2 * int(s), device=dev)
        xcs.append((torch.full_like(x, float("nan")), x, int(s), taps, correlation_fft_size(int(k))))
    batch = ragged_batch(ffts, xcs)
    batch()
    for _, _, d in groups.values():
        d.fill_(float("nan"))
    for y, _, _, _, _ in xcs:
        y.fill_(float("nan"))
    batch()    # the second replay is checked
    torch.cuda.synchronize()
    batch.status()
    worst = 0.0
    for lg, (cnt, src, dst) in groups.items():
        n = 1 << lg
        for r0 in range(0, cnt, 128):    # bounded FP64 working set
            r1 = min(cnt, r0 + 128)
            want = torch.fft.fft(_unpack_rows(src[r0 * 2 * n:r1 * 2 * n], n))
            err = _row_rel_l2(_unpack_rows(dst[r0 * 2 * n:r1 * 2 * n], n), want)
            assert not torch.isnan(err).any(), (n, r0)
            worst = max(worst, float(err.max()))
            assert float(err.max()) < TOL[np.float32], (n, r0, float(err.max()))
    for y, x, s, taps, nf in xcs:
        k = taps.size()
        g = _unpack_rows(taps.data[: 2 * ((k + 7) // 8 * 8)], (k + 7) // 8 * 8)[0, :k]
        L = 1 << int(np.ceil(np.log2(s + k)))
        want = torch.fft.ifft(torch.fft.fft(_unpack_rows(x, s)[0], L) * torch.conj(torch.fft.fft(g, L)))[:s]
        err = float(_row_rel_l2(_unpack_rows(y, s)[0], want))
        worst = max(worst, err)
        assert err < TOL[np.float32], (s, k, nf, err)
    print(f"full C5: worst relative L2 {worst:.3g}")


@pytest.mark.parametrize("log_n", [10, 14, 16, 18])
def test_ragged_inverse_one_size(log_n):
    """An inverse ragged batch (normalised: every transform of one size, as
    pcx_ragged_create requires) against numpy's inverse FFT."""
    n = 1 << log_n
    cnt = max(3, min(40, (1 << 21) // n))
    rng = np.random.default_rng(700 + log_n)
    z = normal_cx(rng, cnt, n)
    src = [dev(O.pack(z[i], 8)) for i in range(cnt)]
    dst = [torch.full_like(s, float("nan")) for s in src]
    batch = ragged_batch([(dst[i], src[i], n) for i in range(cnt)], direction=1)
    batch()
    torch.cuda.synchronize()
    batch.status()
    for i in range(cnt):
        assert rel_l2(O.unpack(dst[i].cpu().numpy(), n, 8), np.fft.ifft(z[i])) < TOL[np.float32], i


def test_ragged_rejects_mixed_normalised_inverse_and_misaligned_buffers():
    rng = np.random.default_rng(8)
    a, b = dev(O.pack(normal_cx(rng, 256), 8)), dev(O.pack(normal_cx(rng, 512), 8))
    with pytest.raises(NotImplementedError):
        ragged_batch([(torch.empty_like(a), a, 256), (torch.empty_like(b), b, 512)], direction=1)
    c = torch.zeros(2 * 1024 + 2, device="cuda")
    with pytest.raises(ValueError):
        ragged_batch([(c[2:], c[2:], 1024)])    # 8-byte offset: not 16-byte aligned


@pytest.mark.parametrize("precision", ["bf16x6", "tf32"])
def test_ragged_tensor_core_form(precision):
    """With tensor_core set, the transforms of 2^8..2^12 points run in the
    persistent tensor-core form beside the ragged launch (one graph): every
    transform of a mixed batch (all sizes 2^5..2^14, ragged counts per size,
    plus correlations) and a normalised inverse of one size against the
    oracle at the FP32 bar."""
    rng = np.random.default_rng(900)
    sizes = [1 << int(v) for v in rng.integers(5, 15, 70)] + [256] * 17 + [4096] * 3
    zs, ffts = [], []
    for n in sizes:
        z = normal_cx(rng, n)
        zs.append(z)
        ffts.append((torch.full((2 * n,), float("nan"), device="cuda"), dev(O.pack(z, 8)), n))
    x, g = normal_cx(rng, 20000), normal_cx(rng, 700)
    xc = (torch.full((len(O.pack(x, 8)),), float("nan"), device="cuda"), dev(O.pack(x, 8)), 20000,
          vector.from_complex(g), 2048)
    batch = ragged_batch(ffts, [xc], tensor_core=precision)
    for replay in range(2):
        batch()
        torch.cuda.synchronize()
        batch.status()
        for (d, _, n), z in zip(ffts, zs):
            assert rel_l2(O.unpack(d.cpu().numpy(), n, 8), np.fft.fft(z)) < TOL[np.float32], (replay, n)
        assert rel_l2(O.unpack(xc[0].cpu().numpy(), 20000, 8), O.xcorr_ols(x, g, 2048)) < TOL[np.float32]
    # inverse, normalised, one size in the tensor-core range
    n = 1024
    z = normal_cx(rng, 11, n)
    src = [dev(O.pack(z[i], 8)) for i in range(11)]
    dst = [torch.full_like(s, float("nan")) for s in src]
    inv = ragged_batch([(dst[i], src[i], n) for i in range(11)], direction=1, tensor_core=precision)
    inv()
    torch.cuda.synchronize()
    inv.status()
    for i in range(11):
        assert rel_l2(O.unpack(dst[i].cpu().numpy(), n, 8), np.fft.ifft(z[i])) < TOL[np.float32], i
