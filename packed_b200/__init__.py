"""packed-b200: B200 (sm_100a) implementation of the FFT hot path of the
Dooez/packed library — fft_unit, fxcorr_unit and the packed split-complex
vector — over the C ABI of libpcx_cuda.so (include/pcx_cuda.h)."""
from .fft import (conj, correlation_fft_size, default_pack_size, evaluate, fft_order, fft_unit, fft_unit_par,
                  fxcorr_unit, ragged_batch, real_size, vector)

__all__ = ["fft_order", "default_pack_size", "real_size", "vector", "fft_unit", "fft_unit_par", "fxcorr_unit", "ragged_batch",
           "conj", "evaluate", "correlation_fft_size"]
__version__ = "0.1.0"
