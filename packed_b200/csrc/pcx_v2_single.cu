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

}    // namespace pcxg

cudaError_t pcx_v2_single(bool f64, int log_n, const pcxg::v2_args& a, cudaStream_t st, bool attr_only) {
    return f64 ? pcxg::dispatch<double>(log_n, a, st, attr_only) : pcxg::dispatch<float>(log_n, a, st, attr_only);
}
