// Instantiations and launch of the four-step column pass (k_col2).
#include "pcx_v2_launch.cuh"

namespace pcxg {

template<class T, int LOGN1, int LOGN2>
static cudaError_t launch(const v2_args& a, cudaStream_t st, int sms, bool attr_only) {
    constexpr int C     = std::max(v2cfg<T>::G8, v2cfg<T>::TILE >> LOGN1);
    constexpr int NT    = C * splan<LOGN1>::TT;
    constexpr int bytes = xch_interleaved<(1 << LOGN1), C>::size * (int)sizeof(cpx<T>);
    auto          kern  = k_col2<T, LOGN1, LOGN2, v2cfg<T>::LP, C, NT>;
    if (attr_only) return set_smem(kern, bytes);
    const long long tiles = a.batch * ((1 << LOGN2) / C);
    if (tiles == 0) return cudaSuccess;
    unsigned    grid = 0;
    cudaError_t e    = persistent_grid(kern, NT, bytes, tiles, sms, &grid);
    if (e != cudaSuccess) return e;
    kern<<<grid, NT, bytes, st>>>(a);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch(int l1, int l2, const v2_args& a, cudaStream_t st, int sms, bool attr_only) {
    switch (l1 * 32 + l2) {
    case 7 * 32 + 6: return launch<T, 7, 6>(a, st, sms, attr_only);
    case 7 * 32 + 7: return launch<T, 7, 7>(a, st, sms, attr_only);
    case 8 * 32 + 7: return launch<T, 8, 7>(a, st, sms, attr_only);
    case 8 * 32 + 8: return launch<T, 8, 8>(a, st, sms, attr_only);
    case 9 * 32 + 8: return launch<T, 9, 8>(a, st, sms, attr_only);
    case 9 * 32 + 9: return launch<T, 9, 9>(a, st, sms, attr_only);
    case 10 * 32 + 9: return launch<T, 10, 9>(a, st, sms, attr_only);
    case 10 * 32 + 10: return launch<T, 10, 10>(a, st, sms, attr_only);
    default: return cudaErrorNotSupported;
    }
}

template<class T, int LOGN1, int LOGN2>
static cudaError_t launch3(const v2_args& a, long long total_rows, long long row0, int* err, cudaStream_t st, int sms,
                           bool attr_only) {
    constexpr int C     = std::max(v2cfg<T>::G8, v2cfg<T>::TILE >> LOGN1);
    constexpr int NT    = C * splan<LOGN1>::TT;
    constexpr int bytes = col3_smem<T, LOGN1, C>();
    auto          kern  = k_col3<T, LOGN1, LOGN2, v2cfg<T>::LP, C, NT>;
    if (attr_only) return set_smem(kern, bytes);
    const long long tiles = a.batch * ((1 << LOGN2) / C);
    if (tiles == 0) return cudaSuccess;
    // 3-D view of the source: [row][n1][2*N2 reals], box = N1 (<= 256) x one 64-byte segment
    CUtensorMap     map;
    const cuuint64_t dims[3]    = {(cuuint64_t)2 << LOGN2, (cuuint64_t)1 << LOGN1, (cuuint64_t)total_rows};
    const cuuint64_t strides[2] = {((cuuint64_t)2 << LOGN2) * sizeof(T), (cuuint64_t)a.src_stride * sizeof(T)};
    const cuuint32_t box[3]     = {(cuuint32_t)(2 * C), (cuuint32_t)col3_boxy<T, LOGN1>(), 1};
    const cuuint32_t estr[3]    = {1, 1, 1};
    cudaError_t      e          = encode_tensor_map(&map, sizeof(T) == 8, 3, const_cast<void*>(a.src), dims, strides, box, estr);
    if (e != cudaSuccess) return e;
    unsigned grid = 0;
    e             = persistent_grid(kern, NT, bytes, tiles, sms, &grid);
    if (e != cudaSuccess) return e;
    v3_pass_args pa{a, row0, err};
    kern<<<grid, NT, bytes, st>>>(map, pa);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch3(int l1, int l2, const v2_args& a, long long total_rows, long long row0, int* err,
                             cudaStream_t st, int sms, bool attr_only) {
    switch (l1 * 32 + l2) {
    case 7 * 32 + 6: return launch3<T, 7, 6>(a, total_rows, row0, err, st, sms, attr_only);
    case 7 * 32 + 7: return launch3<T, 7, 7>(a, total_rows, row0, err, st, sms, attr_only);
    case 8 * 32 + 7: return launch3<T, 8, 7>(a, total_rows, row0, err, st, sms, attr_only);
    case 8 * 32 + 8: return launch3<T, 8, 8>(a, total_rows, row0, err, st, sms, attr_only);
    case 9 * 32 + 8: return launch3<T, 9, 8>(a, total_rows, row0, err, st, sms, attr_only);
    case 9 * 32 + 9: return launch3<T, 9, 9>(a, total_rows, row0, err, st, sms, attr_only);
    case 10 * 32 + 9: return launch3<T, 10, 9>(a, total_rows, row0, err, st, sms, attr_only);
    case 10 * 32 + 10: return launch3<T, 10, 10>(a, total_rows, row0, err, st, sms, attr_only);
    default: return cudaErrorNotSupported;
    }
}

}    // namespace pcxg

cudaError_t pcx_v3_col(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, long long total_rows, long long row0,
                       int* err, cudaStream_t st, int sms, bool attr_only) {
    return f64 ? pcxg::dispatch3<double>(log_n1, log_n2, a, total_rows, row0, err, st, sms, attr_only)
               : pcxg::dispatch3<float>(log_n1, log_n2, a, total_rows, row0, err, st, sms, attr_only);
}

cudaError_t pcx_v2_col(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, cudaStream_t st, int sms,
                       bool attr_only) {
    return f64 ? pcxg::dispatch<double>(log_n1, log_n2, a, st, sms, attr_only)
               : pcxg::dispatch<float>(log_n1, log_n2, a, st, sms, attr_only);
}
