// Instantiations and launch of the single-pass hot-path kernel (k_single2).
#include "pcx_v2_launch.cuh"

namespace pcxg {

template<class T, int LOGL>
static cudaError_t launch(const v2_args& a, cudaStream_t st, bool attr_only) {
    constexpr int NT    = 256;
    using P             = splan<LOGL>;
    constexpr int M     = NT / P::TT;
    constexpr int bytes = xch_blocked<P::L, M>::size * (int)sizeof(cpx<T>);
    auto          kern  = k_single2<T, LOGL, v2cfg<T>::LP, NT>;
    if (attr_only) return set_smem(kern, bytes);
    if (a.batch == 0) return cudaSuccess;
    kern<<<(unsigned)((a.batch + M - 1) / M), NT, bytes, st>>>(a);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch(int log_n, const v2_args& a, cudaStream_t st, bool attr_only) {
    switch (log_n) {
    case 7: return launch<T, 7>(a, st, attr_only);
    case 8: return launch<T, 8>(a, st, attr_only);
    case 9: return launch<T, 9>(a, st, attr_only);
    case 10: return launch<T, 10>(a, st, attr_only);
    case 11: return launch<T, 11>(a, st, attr_only);
    case 12: return launch<T, 12>(a, st, attr_only);
    default: return cudaErrorNotSupported;
    }
}

template<class T, int LOGL>
static cudaError_t launch3(const v3_args& a, cudaStream_t st, int sms, bool attr_only) {
    constexpr int NT    = LOGL >= 13 ? 512 : 256;    // 16 elements per thread
    constexpr int M     = NT / splan<LOGL>::TT;
    constexpr int bytes = single3_smem<T, LOGL, NT>();
    auto          kern  = k_single3<T, LOGL, v2cfg<T>::LP, NT>;
    if (attr_only) return set_smem(kern, bytes);
    const long long tiles = (a.batch + M - 1) / M;
    if (tiles == 0) return cudaSuccess;
    unsigned    grid = 0;
    cudaError_t e    = persistent_grid(kern, NT, bytes, tiles, sms, &grid);
    if (e != cudaSuccess) return e;
    kern<<<grid, NT, bytes, st>>>(a);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch3(int log_n, const v3_args& a, cudaStream_t st, int sms, bool attr_only) {
    switch (log_n) {
    case 5: return launch3<T, 5>(a, st, sms, attr_only);
    case 6: return launch3<T, 6>(a, st, sms, attr_only);
    case 7: return launch3<T, 7>(a, st, sms, attr_only);
    case 8: return launch3<T, 8>(a, st, sms, attr_only);
    case 9: return launch3<T, 9>(a, st, sms, attr_only);
    case 10: return launch3<T, 10>(a, st, sms, attr_only);
    case 11: return launch3<T, 11>(a, st, sms, attr_only);
    case 12: return launch3<T, 12>(a, st, sms, attr_only);
    case 13:
        if constexpr (sizeof(T) == 4) return launch3<T, 13>(a, st, sms, attr_only);    // 64 KB per row
        return cudaErrorNotSupported;
    default: return cudaErrorNotSupported;
    }
}

}    // namespace pcxg

cudaError_t pcx_v3_single(bool f64, int log_n, const pcxg::v3_args& a, cudaStream_t st, int sms, bool attr_only) {
    return f64 ? pcxg::dispatch3<double>(log_n, a, st, sms, attr_only)
               : pcxg::dispatch3<float>(log_n, a, st, sms, attr_only);
}

cudaError_t pcx_v2_single(bool f64, int log_n, const pcxg::v2_args& a, cudaStream_t st, bool attr_only) {
    return f64 ? pcxg::dispatch<double>(log_n, a, st, attr_only) : pcxg::dispatch<float>(log_n, a, st, attr_only);
}
