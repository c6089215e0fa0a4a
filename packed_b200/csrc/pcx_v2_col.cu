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

}    // namespace pcxg

cudaError_t pcx_v2_col(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, cudaStream_t st, int sms,
                       bool attr_only) {
    return f64 ? pcxg::dispatch<double>(log_n1, log_n2, a, st, sms, attr_only)
               : pcxg::dispatch<float>(log_n1, log_n2, a, st, sms, attr_only);
}
