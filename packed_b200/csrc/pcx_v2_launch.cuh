// Launch helpers for the hot-path kernels of pcx_fft_v2.cuh.  Each of the
// pcx_v2_*.cu units instantiates one kernel family so they compile in parallel.
#pragma once

#include "pcx_fft_v2.cuh"
#include "pcx_host.hpp"

#include <algorithm>

namespace pcxg {

template<class T>
struct v2cfg {
    static constexpr int TILE = 65536 / (int)sizeof(cpx<T>);    // elements per four-step tile
    static constexpr int G8   = 64 / (2 * (int)sizeof(T));      // elements per 64-byte segment
    static constexpr int LP   = G8 == 8 ? 3 : 2;                // default pack width (32 bytes of reals)
};

template<class K>
inline cudaError_t set_smem(K kern, int bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// Grid for a persistent launch: resident CTAs, at most one per tile.
template<class K>
inline cudaError_t persistent_grid(K kern, int nt, int bytes, long long tiles, int sms, unsigned* grid) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, bytes);
    if (e != cudaSuccess) return e;
    const long long g = std::min<long long>(tiles, (long long)std::max(per_sm, 1) * sms);
    *grid             = (unsigned)std::max<long long>(g, 1);
    return cudaSuccess;
}

}    // namespace pcxg
