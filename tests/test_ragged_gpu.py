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
    # (its own path through the whole ring)
    for q in range(7):
        s = int(2 ** rng.uniform(12, 17)) if q < 6 else 50000
        k = int(2 ** rng.uniform(6, 12)) if q < 6 else 5000
        nf = max(128, 1 << int(np.ceil(np.log2(2 * k))))
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
