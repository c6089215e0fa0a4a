// Instantiations and launch of the four-step row pass (k_row2).
#include "pcx_v2_launch.cuh"

namespace pcxg {

template<class T, int LOGN1, int LOGN2>
static cudaError_t launch(const v2_args& a, cudaStream_t st, int sms, bool attr_only) {
    constexpr int G8    = v2cfg<T>::G8;
    constexpr int CR    = std::max(G8, v2cfg<T>::TILE >> LOGN2);
    constexpr int NT    = CR * splan<LOGN2>::TT;
    constexpr int bytes = xch_grouped<(1 << LOGN2), CR, G8>::size * (int)sizeof(cpx<T>);
    auto          kern  = k_row2<T, LOGN1, LOGN2, v2cfg<T>::LP, CR, G8, NT>;
    if (attr_only) return set_smem(kern, bytes);
    const long long tiles = a.batch * ((1 << LOGN1) / CR);
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
static cudaError_t launch3(const v2_args& a, int* err, cudaStream_t st, int sms, bool attr_only) {
    constexpr int G8    = v2cfg<T>::G8;
    constexpr int CR    = std::max(G8, v2cfg<T>::TILE >> LOGN2);
    constexpr int NT    = CR * splan<LOGN2>::TT;
    constexpr int bytes = row3_smem<T, LOGN2, CR, G8>();
    auto          kern  = k_row3<T, LOGN1, LOGN2, v2cfg<T>::LP, CR, G8, NT>;
    if (attr_only) return set_smem(kern, bytes);
    const long long tiles = a.batch * ((1 << LOGN1) / CR);
    if (tiles == 0) return cudaSuccess;
    unsigned    grid = 0;
    cudaError_t e    = persistent_grid(kern, NT, bytes, tiles, sms, &grid);
    if (e != cudaSuccess) return e;
    v3_pass_args pa{a, 0, err};
    kern<<<grid, NT, bytes, st>>>(pa);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch3(int l1, int l2, const v2_args& a, int* err, cudaStream_t st, int sms, bool attr_only) {
    switch (l1 * 32 + l2) {
    case 7 * 32 + 6: return launch3<T, 7, 6>(a, err, st, sms, attr_only);
    case 7 * 32 + 7: return launch3<T, 7, 7>(a, err, st, sms, attr_only);
    case 8 * 32 + 7: return launch3<T, 8, 7>(a, err, st, sms, attr_only);
    case 8 * 32 + 8: return launch3<T, 8, 8>(a, err, st, sms, attr_only);
    case 9 * 32 + 8: return launch3<T, 9, 8>(a, err, st, sms, attr_only);
    case 9 * 32 + 9: return launch3<T, 9, 9>(a, err, st, sms, attr_only);
    case 10 * 32 + 9: return launch3<T, 10, 9>(a, err, st, sms, attr_only);
    case 10 * 32 + 10: return launch3<T, 10, 10>(a, err, st, sms, attr_only);
    default: return cudaErrorNotSupported;
    }
}

}    // namespace pcxg

cudaError_t pcx_v3_row(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, int* err, cudaStream_t st, int sms,
                       bool attr_only) {
    return f64 ? pcxg::dispatch3<double>(log_n1, log_n2, a, err, st, sms, attr_only)
               : pcxg::dispatch3<float>(log_n1, log_n2, a, err, st, sms, attr_only);
}

cudaError_t pcx_v2_row(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, cudaStream_t st, int sms,
                       bool attr_only) {
    return f64 ? pcxg::dispatch<double>(log_n1, log_n2, a, st, sms, attr_only)
               : pcxg::dispatch<float>(log_n1, log_n2, a, st, sms, attr_only);
}

// Stage-twiddle tables (shared by the three families): entries and generation.
namespace {
template<int LOGL>
constexpr int tw_entries() {
    return pcxg::stage_tw_size<pcxg::splan<LOGL>>();
}
template<int LOGL, class T>
cudaError_t gen_stage(void* out, cudaStream_t st) {
    using P = pcxg::splan<LOGL>;
    for (int s = 1; s < P::NST; ++s) {
        const int ns = 1 << P::nsbits(s), nq = pcxg::stw_q(P::rbits(s));
        auto*     o  = static_cast<pcxg::cpx<T>*>(out) + pcxg::stage_tw_offset<P>(s);
        pcxg::k_stage_twiddles<T><<<(ns * nq + 255) / 256, 256, 0, st>>>(o, ns, P::rbits(s), P::nsbits(s) + P::rbits(s));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
template<int LOGL>
cudaError_t stage_dispatch(void* out, bool f64, cudaStream_t st, int* entries) {
    *entries = tw_entries<LOGL>();
    if (!out) return cudaSuccess;
    return f64 ? gen_stage<LOGL, double>(out, st) : gen_stage<LOGL, float>(out, st);
}
}    // namespace

cudaError_t pcx_v2_stage_twiddles(int log_l, void* out, bool f64, cudaStream_t st, int* entries) {
    switch (log_l) {
    case 1: return stage_dispatch<1>(out, f64, st, entries);
    case 2: return stage_dispatch<2>(out, f64, st, entries);
    case 3: return stage_dispatch<3>(out, f64, st, entries);
    case 4: return stage_dispatch<4>(out, f64, st, entries);
    case 5: return stage_dispatch<5>(out, f64, st, entries);
    case 6: return stage_dispatch<6>(out, f64, st, entries);
    case 7: return stage_dispatch<7>(out, f64, st, entries);
    case 8: return stage_dispatch<8>(out, f64, st, entries);
    case 9: return stage_dispatch<9>(out, f64, st, entries);
    case 10: return stage_dispatch<10>(out, f64, st, entries);
    case 11: return stage_dispatch<11>(out, f64, st, entries);
    case 12: return stage_dispatch<12>(out, f64, st, entries);
    case 13: return stage_dispatch<13>(out, f64, st, entries);
    case 14: return stage_dispatch<14>(out, f64, st, entries);
    default: return cudaErrorNotSupported;
    }
}
