// Launch of one variant of the one-launch four-step kernel (k_fourstep), and
// the macro the variant translation units (pcx_fs_part*.cu) instantiate it
// with.  The variants are split over several files only to build in parallel.
#pragma once

#include "pcx_fourstep.cuh"
#include "pcx_host.hpp"
#include "pcx_v2_launch.cuh"

#include <type_traits>

namespace pcxg {

template<class T, int LOGN1, int LOGN2, int MINB, int ST>
cudaError_t launch_fs(const fs_args& a, cudaStream_t st, int sms, bool attr_only, int* tc, int* tr, int* per_sm) {
    using F = fs_cfg<T, LOGN1, LOGN2, MINB, ST>;
    static_assert(F::SMEM <= 232448, "shared memory per block");
    static_assert(F::MINB * (F::SMEM + 1024 + 256) <= 233472, "blocks per SM fit the shared memory");
    static_assert(F::STAGE % 128 == 0, "TMA destinations stay 128-byte aligned");
    auto kern = k_fourstep<T, LOGN1, LOGN2, MINB, ST>;
    if (tc) *tc = F::TC;
    if (tr) *tr = F::TR;
    if (attr_only) {
        cudaError_t e = set_smem(kern, F::SMEM);
        if (e == cudaSuccess && per_sm) e = occupancy_cached(reinterpret_cast<const void*>(kern), F::NT + 64, F::SMEM, per_sm);
        return e;
    }
    const long long items = a.batch * (F::TC + F::TR);
    if (items == 0) return cudaSuccess;
    if (items >= (1LL << 31)) return cudaErrorInvalidValue;    // the kernel counts items in 32 bits
    // 3-D view of the source: [transform][n1][2*N2 reals], box = 2*C reals x min(N1, 256) rows
    CUtensorMap      map;
    const cuuint64_t dims[3]    = {(cuuint64_t)2 << LOGN2, (cuuint64_t)1 << LOGN1, (cuuint64_t)a.batch};
    const long long  ss         = a.batch > 1 ? a.src_stride : (2LL << (LOGN1 + LOGN2));    // unused when 1 row
    const cuuint64_t strides[2] = {((cuuint64_t)2 << LOGN2) * sizeof(T), (cuuint64_t)ss * sizeof(T)};
    const cuuint32_t box[3]     = {(cuuint32_t)(2 * F::C), (cuuint32_t)F::BOXY, 1};
    const cuuint32_t estr[3]    = {1, 1, 1};
    cudaError_t      e = encode_tensor_map(&map, sizeof(T) == 8, 3, const_cast<void*>(a.src), dims, strides, box, estr);
    if (e != cudaSuccess) return e;
    unsigned grid = 0;
    e             = persistent_grid(kern, F::NT + 64, F::SMEM, items, sms, &grid);
    if (e != cudaSuccess) return e;
    kern<<<grid, F::NT + 64, F::SMEM, st>>>(map, a);
    return cudaGetLastError();
}

}    // namespace pcxg

// Inside a part function (f64, v, a, st, sms, attr_only, tc, tr, per_sm in scope).
#define PCX_FS_VARIANT(T, L1, L2, M, S)                                                                    \
    if (f64 == std::is_same<T, double>::value && v.l1 == L1 && v.l2 == L2 && v.minb == M && v.st == S) { \
        return pcxg::launch_fs<T, L1, L2, M, S>(a, st, sms, attr_only, tc, tr, per_sm);                   \
    }

#define PCX_FS_PART(NAME)                                                                                     \
    cudaError_t NAME(bool f64, const pcxg::fs_variant& v, const pcxg::fs_args& a, cudaStream_t st, int sms, \
                     bool attr_only, int* tc, int* tr, int* per_sm)
