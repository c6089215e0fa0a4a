"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs the reference library's own fft_unit<float> / fxcorr_unit<float>
(compiled from its headers by oracle/Makefile into oracle/_ref/libpcx_ref.so)
on seeded inputs and stores inputs and outputs in ``fft_golden.npz``.  Run it
where the reference sources are present:

    make -C oracle && python tests/golden/make_golden.py

Inputs come from numpy's PCG64 generator (``np.random.default_rng(seed)``),
the one generator every harness in this repository uses.  All arrays are
float32 packed split-complex rows at pack width 8.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "fft_golden.npz"


def uniform_cx(rng, n):
    return (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libpcx_ref.so missing: build it with the reference sources present")
    d: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(1234)
    # 1) every order, forward and inverse, per size
    for n in (64, 256, 1024, 4096):
        x = O.pack(uniform_cx(rng, n), 8)
        d[f"x_{n}"] = x
        for order in (0, 1, 2):
            y = O.ref_fft(x, n, order, 0)
            d[f"fwd_{n}_o{order}"] = y
            d[f"inv_{n}_o{order}"] = O.ref_fft(y, n, order, 1, True)
            if order:
                d[f"invraw_{n}_o{order}"] = O.ref_fft(y, n, order, 1, False)
    n = 16384
    x = O.pack(uniform_cx(rng, n), 8)
    d[f"x_{n}"] = x
    d[f"fwd_{n}_o0"] = O.ref_fft(x, n, 0, 0)
    # 2) the reference test's own input: exp(i*2*pi*i/N*13.37) in float (tests/test_fft.cpp:300)
    n = 1024
    i = np.arange(n, dtype=np.float32)
    tone = np.exp(1j * (np.float32(2 * np.pi) * i / np.float32(n) * np.float32(13.37)).astype(np.float32))
    d["tone_x_1024"] = O.pack(tone.astype(np.complex64), 8)
    d["tone_fwd_1024"] = O.ref_fft(d["tone_x_1024"], n, 0, 0)
    # 3) zero-extended source (fft.hpp:759-820): bit_reversed, src 700 of 1024
    src = O.pack(uniform_cx(rng, 700), 8)
    d["zx_src_700"] = src
    d["zx_fwd_1024_o1"] = O.ref_fft_oop(src, 1024, 700, 1, 0)
    # 4) config C1 (N=1024, batch 64, U[-1,1) seed 0): the first 4 rows, fwd then inverse
    rng0 = np.random.default_rng(0)
    c1 = np.stack([uniform_cx(rng0, 1024) for _ in range(64)])
    rows = O.pack(c1[:4], 8)
    d["c1_x"] = rows
    d["c1_fwd"] = np.stack([O.ref_fft(r, 1024, 0, 0) for r in rows])
    d["c1_inv"] = np.stack([O.ref_fft(r, 1024, 0, 1) for r in d["c1_fwd"]])
    # 5) correlation: single block through the shipped fxcorr_unit (exact there),
    #    multi block through the corrected overlap-save on the reference fft_unit
    bark = np.array([1, 1, 1, 1, 1, -1, -1, 1, 1, -1, 1, -1, 1], dtype=np.complex64)
    g = np.zeros(128, np.complex64)
    g[:13] = bark
    f = rng.integers(-3, 4, 128).astype(np.complex64) * 1j
    f[109:122] += bark
    d["xc1_g"], d["xc1_x"] = O.pack(g, 8), O.pack(f, 8)
    d["xc1_y"] = O.ref_fxcorr(d["xc1_g"], 128, 256, d["xc1_x"], 128, fixed=False)
    g2 = np.exp(1j * rng.integers(-3, 3, 512)).astype(np.complex64)
    x2 = np.exp(1j * rng.integers(-3, 3, 512)).astype(np.complex64)
    d["xc2_g"], d["xc2_x"] = O.pack(g2, 8), O.pack(x2, 8)
    d["xc2_y"] = O.ref_fxcorr(d["xc2_g"], 512, 1024, d["xc2_x"], 512, fixed=False)
    g3 = (rng.standard_normal(100) + 1j * rng.standard_normal(100)).astype(np.complex64)
    x3 = (rng.standard_normal(3000) + 1j * rng.standard_normal(3000)).astype(np.complex64)
    d["xc3_g"], d["xc3_x"] = O.pack(g3, 8), O.pack(x3, 8)
    d["xc3_y"] = O.ref_fxcorr(d["xc3_g"], 100, 512, d["xc3_x"], 3000, fixed=True)
    d["xc3_y_shipped"] = O.ref_fxcorr(d["xc3_g"], 100, 512, d["xc3_x"], 3000, fixed=False)
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(d)} arrays)")


if __name__ == "__main__":
    main()
