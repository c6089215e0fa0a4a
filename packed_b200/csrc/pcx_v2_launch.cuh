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
    cudaError_t e = occupancy_cached(reinterpret_cast<const void*>(kern), nt, bytes, &per_sm);
    if (e != cudaSuccess) return e;
    const long long g = std::min<long long>(tiles, (long long)std::max(per_sm, 1) * sms);
    *grid             = (unsigned)std::max<long long>(g, 1);
    return cudaSuccess;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
inline cudaError_t encode_tensor_map(CUtensorMap* map, bool f64, int rank, void* base, const cuuint64_t* dims,
                                     const cuuint64_t* strides, const cuuint32_t* box, const cuuint32_t* estr) {
    using fn_t     = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static fn_t fn = nullptr;
    if (!fn) {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || !p) return e != cudaSuccess ? e : cudaErrorNotSupported;
        fn = reinterpret_cast<fn_t>(p);
    }
    const CUresult r = fn(map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, base, dims,
                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}    // namespace pcxg
