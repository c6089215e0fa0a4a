"""torch.autograd.Function wrappers over the hand-written adjoints.

Tensors are packed split-complex reals (the library layout); the gradient of a
real loss with respect to a packed real is exactly the library's complex
cotangent convention (d/dRe + i d/dIm stored at the same packed positions).

* ``FFTFunction.apply(x, unit, direction, normalize, batch)``: y = fft(x)
  (or the inverse); backward is pcx_fft_vjp.
* ``FxcorrFunction.apply(x, g, fft_size, length, channels)``: y = x (*) g,
  the overlap-save correlation; backward is pcx_fxcorr_vjp (convolution with
  g for x, correlation of the output gradient with x for g).
"""
from __future__ import annotations

import torch

from .fft import default_pack_size, fft_unit, fxcorr_unit, real_size, vector


class FFTFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, unit: fft_unit, direction: int = 0, normalize: bool = True,
                batch: int = 1):
        y = torch.empty_like(x)
        unit.exec(y, x.contiguous(), direction=direction, normalize=normalize, batch=batch)
        ctx.unit, ctx.direction, ctx.normalize, ctx.batch = unit, direction, normalize, batch
        return y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        gx = ctx.unit.vjp(gy.contiguous(), direction=ctx.direction, normalize=ctx.normalize, batch=ctx.batch)
        return gx, None, None, None, None


class FxcorrFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, g: torch.Tensor, fft_size: int, length: int, k: int, channels: int = 1):
        p = default_pack_size(x.dtype)
        unit = fxcorr_unit(vector(k, dtype=g.dtype, data=g.detach().contiguous()), fft_size)
        y = torch.empty_like(x)
        unit.exec(y, x.contiguous(), length, channels=channels, pack=p)
        ctx.unit, ctx.length, ctx.channels = unit, length, channels
        ctx.save_for_backward(x)
        return y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        (x,) = ctx.saved_tensors
        gx, gg = ctx.unit.vjp(gy.contiguous(), x.contiguous(), ctx.length, channels=ctx.channels,
                              want_kernel_grad=ctx.needs_input_grad[1])
        return gx, gg, None, None, None, None


def packed_reals(n: int, dtype: torch.dtype = torch.float32) -> int:
    return real_size(n, default_pack_size(dtype))
