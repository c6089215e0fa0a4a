// Host side of the overlap-save correlator: handle creation (kernel spectrum
// computed on the device), the fused correlation launch and its adjoint.
#include "pcx_fxcorr2d.cuh"
#include "pcx_fxcorr_kernels.cuh"
#include "pcx_host.hpp"
#include "pcx_v2_launch.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

using namespace pcxg;

struct pcx_fxcorr_s {
    int         dtype  = PCX_F32;
    size_t      k      = 0;
    size_t      n      = 0;
    int         log_n  = 0;
    int         pack_g = 8;
    pcx_plan_s* plan   = nullptr;    // natural-order N-point FFT (kernel spectrum, gradient inverse)
    void*       tw     = nullptr;    // W_N^i, i < N
    void*       kspec  = nullptr;    // FFT(g)/N, interleaved complex, natural order
    unsigned*   ctl    = nullptr;    // [0] work counter, [1] error flag, [2..] flags
    size_t      flags_cap = 0;
    unsigned    epoch     = 0;
    void*       gscratch  = nullptr;    // kernel-gradient accumulators
    size_t      gscratch_bytes = 0;
    int         sms            = 0;
    int         device         = 0;
    // FP32, N = 2^13 or 2^14: in-CTA four-step form (pcx_fxcorr2d.cuh)
    void*       x2d            = nullptr;    // one allocation: K permuted | stage tables | twiddles
    const void* x2_kperm       = nullptr;
    const void* x2_stw1        = nullptr;
    const void* x2_stw2        = nullptr;
    const void* x2_tws         = nullptr;
};

namespace {

constexpr int XC_SINGLE_NT = 256;

template<class T, int LOGN>
struct xcfg {
    static constexpr int EPT = LOGN >= 14 ? 32 : 16;
    using P                  = splan<LOGN, EPT>;
    static constexpr int M   = P::TT >= XC_SINGLE_NT ? 1 : XC_SINGLE_NT / P::TT;
    static constexpr int NT  = M * P::TT;
};

template<class T, int LOGN>
int launch_xc(const xc_args& a, const void* tw, cudaStream_t st, int sms, bool attr_only) {
    using C             = xcfg<T, LOGN>;
    constexpr int bytes = fxcorr_smem_bytes<T, LOGN, C::EPT, C::M>();
    auto          kern  = k_fxcorr<T, LOGN, C::EPT, C::M>;
    if (attr_only) {
        PCX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        return PCX_OK;
    }
    int per_sm = 0;
    PCX_CUDA_TRY(occupancy_cached(reinterpret_cast<const void*>(kern), C::NT, bytes, &per_sm));
    const long long groups = (a.total + C::M - 1) / C::M;
    const long long grid   = std::max<long long>(1, std::min<long long>(groups, (long long)std::max(per_sm, 1) * sms));
    kern<<<(unsigned)grid, C::NT, bytes, st>>>(a, reinterpret_cast<const cpx<T>*>(tw));
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}

template<class T, int LOGN>
int launch_kg(const kg_args& a, const void* tw, cudaStream_t st, int grid, bool attr_only) {
    using C             = xcfg<T, LOGN>;
    constexpr int bytes = fxcorr_smem_bytes<T, LOGN, C::EPT, 1>();
    auto          kern  = k_fxcorr_kgrad<T, LOGN, C::EPT>;
    if (attr_only) {
        PCX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        return PCX_OK;
    }
    kern<<<(unsigned)grid, C::P::TT, bytes, st>>>(a, reinterpret_cast<const cpx<T>*>(tw));
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}

template<class T>
int dispatch_xc(int log_n, const xc_args& a, const void* tw, cudaStream_t st, int sms, bool attr_only) {
    switch (log_n) {
    case 6: return launch_xc<T, 6>(a, tw, st, sms, attr_only);
    case 7: return launch_xc<T, 7>(a, tw, st, sms, attr_only);
    case 8: return launch_xc<T, 8>(a, tw, st, sms, attr_only);
    case 9: return launch_xc<T, 9>(a, tw, st, sms, attr_only);
    case 10: return launch_xc<T, 10>(a, tw, st, sms, attr_only);
    case 11: return launch_xc<T, 11>(a, tw, st, sms, attr_only);
    case 12: return launch_xc<T, 12>(a, tw, st, sms, attr_only);
    case 13: return launch_xc<T, 13>(a, tw, st, sms, attr_only);
    case 14:
        if constexpr (sizeof(T) == 4) return launch_xc<T, 14>(a, tw, st, sms, attr_only);
        [[fallthrough]];
    default: return pcx_fail(PCX_ERR_UNSUPPORTED, "fft size not supported by the fused correlator");
    }
}

template<class T>
int dispatch_kg(int log_n, const kg_args& a, const void* tw, cudaStream_t st, int grid, bool attr_only) {
    switch (log_n) {
    case 6: return launch_kg<T, 6>(a, tw, st, grid, attr_only);
    case 7: return launch_kg<T, 7>(a, tw, st, grid, attr_only);
    case 8: return launch_kg<T, 8>(a, tw, st, grid, attr_only);
    case 9: return launch_kg<T, 9>(a, tw, st, grid, attr_only);
    case 10: return launch_kg<T, 10>(a, tw, st, grid, attr_only);
    case 11: return launch_kg<T, 11>(a, tw, st, grid, attr_only);
    case 12: return launch_kg<T, 12>(a, tw, st, grid, attr_only);
    case 13: return launch_kg<T, 13>(a, tw, st, grid, attr_only);
    case 14:
        if constexpr (sizeof(T) == 4) return launch_kg<T, 14>(a, tw, st, grid, attr_only);
        [[fallthrough]];
    default: return pcx_fail(PCX_ERR_UNSUPPORTED, "fft size not supported by the fused correlator");
    }
}

template<class T>
__global__ void k_scale_pack(const cpx<T>* __restrict__ src, int k, int lp, T* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const int P = 1 << lp;
    const int o = ((i >> lp) << (lp + 1)) + (i & (P - 1));
    dst[o]      = src[i].re;
    dst[o + P]  = src[i].im;
}

// K / N from natural order k = k1 + N1*k2 to row-major [k1][k2].
__global__ void k_perm_spectrum(const cpx<float>* __restrict__ ks, cpx<float>* __restrict__ kp, int log_n1,
                                int log_n2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (1 << (log_n1 + log_n2))) return;
    const int k1 = q >> log_n2, k2 = q & ((1 << log_n2) - 1);
    kp[q]        = ks[k1 + (k2 << log_n1)];
}

}    // namespace

// The spectrum K[k1 + N1*k2] stored at [k1*N2 + k2] (the (k1, k2) order of the
// in-CTA four-step correlator's rows), on `st`.
cudaError_t pcx_xc2_perm_spectrum(const void* ks, void* kp, int log_n1, int log_n2, cudaStream_t st) {
    const int n = 1 << (log_n1 + log_n2);
    k_perm_spectrum<<<(n + 255) / 256, 256, 0, st>>>(static_cast<const cpx<float>*>(ks), static_cast<cpx<float>*>(kp),
                                                      log_n1, log_n2);
    return cudaGetLastError();
}

namespace {

template<int LOGN>
int launch_xc2(const xc2_args& a, cudaStream_t st, int sms, bool attr_only) {
    using C   = xc2_cfg<LOGN>;
    auto kern = k_fxcorr2d<LOGN>;
    if (attr_only) {
        PCX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        return PCX_OK;
    }
    int per_sm = 0;
    PCX_CUDA_TRY(occupancy_cached(reinterpret_cast<const void*>(kern), C::NT, C::SMEM, &per_sm));
    const long long grid = std::max<long long>(1, std::min<long long>(a.base.total, (long long)std::max(per_sm, 1) * sms));
    kern<<<(unsigned)grid, C::NT, C::SMEM, st>>>(a);
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}

template<int LOGN>
int launch_xc2_kg(const xc2_kg_args& a, cudaStream_t st, int grid, bool attr_only) {
    using C   = xc2_cfg<LOGN>;
    auto kern = k_fxcorr2d_kgrad<LOGN>;
    if (attr_only) {
        PCX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        return PCX_OK;
    }
    kern<<<(unsigned)grid, C::NT, C::SMEM, st>>>(a);
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}

// Tables of the in-CTA four-step form; false when it does not apply.
template<int LOGN>
int init_xc2(pcx_fxcorr_s* h) {
    using C         = xc2_cfg<LOGN>;
    int e1 = 0, e2 = 0;
    // full stage tables of the two sub-transforms (one entry per twiddle)
    PCX_CUDA_TRY(pcx_fourstep_tables(C::LOGN1, nullptr, false, 0, &e1));
    PCX_CUDA_TRY(pcx_fourstep_tables(C::LOGN2, nullptr, false, 0, &e2));
    e1                  = (e1 + 1) / 2 * 2;    // 16-byte sections
    e2                  = (e2 + 1) / 2 * 2;
    const size_t ntw    = (size_t)C::NB + C::N2 + C::N1;
    const size_t entries = (size_t)C::N + e1 + e2 + ntw;
    PCX_CUDA_TRY(cudaMalloc(&h->x2d, entries * sizeof(cpx<float>)));
    auto* base   = static_cast<cpx<float>*>(h->x2d);
    auto* kp     = base;
    auto* s1     = kp + C::N;
    auto* s2     = s1 + e1;
    auto* tws    = s2 + e2;
    PCX_CUDA_TRY(pcx_xc2_perm_spectrum(h->kspec, kp, C::LOGN1, C::LOGN2, 0));
    PCX_CUDA_TRY(pcx_fourstep_tables(C::LOGN1, s1, false, 0, &e1));
    PCX_CUDA_TRY(pcx_fourstep_tables(C::LOGN2, s2, false, 0, &e2));
    PCX_CUDA_TRY(pcx_gen_twiddles(tws, C::NB, LOGN, 1, false, 0));
    PCX_CUDA_TRY(pcx_gen_twiddles(tws + C::NB, C::N2, LOGN, C::TT1, false, 0));
    PCX_CUDA_TRY(pcx_gen_twiddles(tws + C::NB + C::N2, C::N1, LOGN, C::TT2, false, 0));
    h->x2_kperm = kp;
    h->x2_stw1  = s1;
    h->x2_stw2  = s2;
    h->x2_tws   = tws;
    if (int rc = launch_xc2_kg<LOGN>(xc2_kg_args{}, 0, 0, true)) return rc;
    return launch_xc2<LOGN>(xc2_args{}, 0, 0, true);
}

int check_pack(int pack) {
    if (pack < 1 || (pack & (pack - 1)) != 0) {
        return pcx_fail(PCX_ERR_INVALID, "pack size (which is " + std::to_string(pack) + ") is not a power of two");
    }
    return PCX_OK;
}

int ensure_flags(pcx_fxcorr_s* h, size_t items) {
    if (h->ctl && h->flags_cap >= items) return PCX_OK;
    if (h->ctl) cudaFree(h->ctl);
    h->ctl       = nullptr;
    h->flags_cap = 0;
    const size_t cap = std::max<size_t>(items, 1024);
    PCX_CUDA_TRY(cudaMalloc(&h->ctl, (cap + 2) * sizeof(unsigned)));
    PCX_CUDA_TRY(cudaMemset(h->ctl, 0, (cap + 2) * sizeof(unsigned)));
    h->flags_cap = cap;
    h->epoch     = 0;
    return PCX_OK;
}

int run_xc(pcx_fxcorr_s* h, void* dst, const void* src, size_t len, int pack, size_t channels, size_t dstride,
           size_t sstride, bool convolve, cudaStream_t st) {
    if (int rc = check_pack(pack)) return rc;
    const size_t n = h->n;
    if ((size_t)pack > n) return pcx_fail(PCX_ERR_UNSUPPORTED, "pack size larger than fft size");
    const size_t step = (n - (h->k - 1)) / pack * pack;
    if (step == 0) {
        return pcx_fail(PCX_ERR_INVALID, "kernel size (which is " + std::to_string(h->k) +
                                             ") leaves no output per block for fft size " + std::to_string(n));
    }
    if (len == 0 || channels == 0) return PCX_OK;
    if (!dst || !src) return pcx_fail(PCX_ERR_INVALID, "null data pointer");
    const size_t row = (len + pack - 1) / pack * 2 * pack;
    if (channels > 1 && (dstride < row || sstride < row)) return pcx_fail(PCX_ERR_INVALID, "channel stride smaller than a row");
    const size_t nblk  = (len + step - 1) / step;
    const size_t total = nblk * channels;
    if (total >= (size_t(1) << 31)) return pcx_fail(PCX_ERR_UNSUPPORTED, "too many blocks in one call");
    const bool inplace = dst == src;
    if (inplace && convolve) return pcx_fail(PCX_ERR_INVALID, "the adjoint needs distinct input and output buffers");
    if (int rc = ensure_flags(h, inplace ? total : 1)) return rc;
    if (++h->epoch == 0) {
        PCX_CUDA_TRY(cudaMemsetAsync(h->ctl + 2, 0, h->flags_cap * sizeof(unsigned), st));
        h->epoch = 1;
    }
    PCX_CUDA_TRY(cudaMemsetAsync(h->ctl, 0, sizeof(unsigned), st));

    xc_args a{};
    a.src         = src;
    a.dst         = dst;
    a.src_stride  = (long long)sstride;
    a.dst_stride  = (long long)dstride;
    a.len         = (long long)len;
    a.lp          = __builtin_ctz(pack);
    a.step        = (int)step;
    a.nblk        = (int)nblk;
    a.total       = (long long)total;
    // convolution (the adjoint): window b starts `shift` samples before
    // output b*step, and output m of the block is circular index m + shift.
    // Any shift >= K-1 with step + shift <= N gives the same outputs; at pack 8
    // K-1 rounded up to whole packs is one (step = N - shift), and it keeps
    // the windows on whole packs, as the four-step form below needs.
    const size_t shift = pack == 8 ? (h->k - 1 + 7) / 8 * 8 : h->k - 1;
    a.in_shift    = convolve ? (int)shift : 0;
    a.out_shift   = convolve ? (int)shift : 0;
    a.conj_kernel = convolve ? 0 : 1;
    a.inplace     = inplace ? 1 : 0;
    a.hwait       = (int)((n + step - 1) / step) - 1;
    a.epoch       = h->epoch;
    a.flags       = h->ctl + 2;
    a.counter     = h->ctl;
    a.error       = reinterpret_cast<int*>(h->ctl + 1);
    a.kspec       = h->kspec;
    // in-CTA four-step form: FP32, pack 8, windows on whole packs, rows of
    // packs 16-byte aligned
    const bool x2 = h->x2d && pack == 8 && a.in_shift % 8 == 0 &&
                    (channels == 1 || sstride % 4 == 0) && reinterpret_cast<uintptr_t>(src) % 16 == 0;
    if (x2) {
        xc2_args b{};
        b.base  = a;
        b.kperm = h->x2_kperm;
        b.stw1  = h->x2_stw1;
        b.stw2  = h->x2_stw2;
        b.tws   = h->x2_tws;
        return h->log_n == 14 ? launch_xc2<14>(b, st, h->sms, false) : launch_xc2<13>(b, st, h->sms, false);
    }
    return h->dtype == PCX_F64 ? dispatch_xc<double>(h->log_n, a, h->tw, st, h->sms, false)
                               : dispatch_xc<float>(h->log_n, a, h->tw, st, h->sms, false);
}

}    // namespace

extern "C" int pcx_fxcorr_create(pcx_fxcorr* out, const void* g, size_t k, int pack_g, size_t n_fft, int dtype) {
    return pcx_guard([&]() -> int {
        if (!out) return pcx_fail(PCX_ERR_INVALID, "handle pointer is null");
        *out = nullptr;
        if (n_fft <= 1 || (n_fft & (n_fft - 1)) != 0) {
            return pcx_fail(PCX_ERR_INVALID, "fft_size (which is " + std::to_string(n_fft) +
                                                 ") is not a power of two or less than 2");
        }
        if (dtype != PCX_F32 && dtype != PCX_F64) return pcx_fail(PCX_ERR_INVALID, "unknown dtype");
        if (int rc = check_pack(pack_g)) return rc;
        if (k == 0 || k > n_fft) {
            return pcx_fail(PCX_ERR_INVALID, "kernel size (which is " + std::to_string(k) +
                                                 ") must be in 1..fft size (which is " + std::to_string(n_fft) + ")");
        }
        const int log_n = __builtin_ctzll(n_fft);
        const int maxlog = dtype == PCX_F64 ? 13 : 14;
        if (log_n < 6 || log_n > maxlog) {
            return pcx_fail(PCX_ERR_UNSUPPORTED, "fused correlator supports fft sizes 2^6..2^" + std::to_string(maxlog));
        }
        if (!g) return pcx_fail(PCX_ERR_INVALID, "null kernel pointer");
        auto h    = new pcx_fxcorr_s{};
        h->dtype  = dtype;
        h->k      = k;
        h->n      = n_fft;
        h->log_n  = log_n;
        h->pack_g = pack_g;
        cudaGetDevice(&h->device);
        auto fail = [&](int rc) {
            pcx_fxcorr_destroy(h);
            return rc;
        };
        PCX_CUDA_TRY(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device));
        int rc = pcx_plan_create(&h->plan, n_fft, dtype, PCX_ORDER_NORMAL, 2048);
        if (rc) return fail(rc);
        const size_t eb = dtype == PCX_F64 ? 16 : 8;
        cudaError_t  e  = cudaMalloc(&h->tw, n_fft * eb);
        if (e == cudaSuccess) e = cudaMalloc(&h->kspec, n_fft * eb);
        if (e == cudaSuccess) e = pcx_gen_twiddles(h->tw, (int)n_fft, log_n, 1, dtype == PCX_F64, 0);
        if (e != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        // K = FFT(g zero-padded to N) / N, natural order, interleaved (fxcorr.hpp:62-69)
        rc = pcx_fft_run(h->plan, h->kspec, g, k, 1, pack_g, PCX_FORWARD, 0, 1, 2 * n_fft,
                         (k + pack_g - 1) / pack_g * 2 * pack_g, nullptr, 0, 0, 1.0 / (double)n_fft);
        if (rc) return fail(rc);
        rc = dtype == PCX_F64 ? dispatch_xc<double>(log_n, xc_args{}, nullptr, 0, 0, true)
                              : dispatch_xc<float>(log_n, xc_args{}, nullptr, 0, 0, true);
        if (rc) return fail(rc);
        rc = dtype == PCX_F64 ? dispatch_kg<double>(log_n, kg_args{}, nullptr, 0, 0, true)
                              : dispatch_kg<float>(log_n, kg_args{}, nullptr, 0, 0, true);
        if (rc) return fail(rc);
        if (dtype == PCX_F32 && (log_n == 13 || log_n == 14) && std::getenv("PCX_XC_GENERAL") == nullptr) {
            rc = log_n == 14 ? init_xc2<14>(h) : init_xc2<13>(h);
            if (rc) return fail(rc);
        }
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        *out = h;
        return PCX_OK;
    });
}

extern "C" int pcx_fxcorr_destroy(pcx_fxcorr h) {
    if (!h) return PCX_OK;
    if (h->plan) pcx_plan_destroy(h->plan);
    if (h->tw) cudaFree(h->tw);
    if (h->kspec) cudaFree(h->kspec);
    if (h->ctl) cudaFree(h->ctl);
    if (h->gscratch) cudaFree(h->gscratch);
    if (h->x2d) cudaFree(h->x2d);
    delete h;
    return PCX_OK;
}

extern "C" int pcx_fxcorr_exec(pcx_fxcorr h, void* dst, const void* src, size_t len, int pack, size_t channels,
                               size_t dst_stride, size_t src_stride, void* stream) {
    return pcx_guard([&]() -> int {
        if (!h) return pcx_fail(PCX_ERR_INVALID, "handle is null");
        return run_xc(h, dst, src, len, pack, channels, dst_stride, src_stride, false,
                      static_cast<cudaStream_t>(stream));
    });
}

extern "C" int pcx_fxcorr_status(pcx_fxcorr h) {
    return pcx_guard([&]() -> int {
        if (!h) return pcx_fail(PCX_ERR_INVALID, "handle is null");
        if (!h->ctl) return PCX_OK;
        unsigned err = 0;
        PCX_CUDA_TRY(cudaMemcpy(&err, h->ctl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (err) {
            PCX_CUDA_TRY(cudaMemset(h->ctl + 1, 0, sizeof(unsigned)));
            return pcx_fail(PCX_ERR_TIMEOUT, "a correlation block gave up a bounded wait (for its input copy or, in place, for its predecessor)");
        }
        return PCX_OK;
    });
}

extern "C" int pcx_fxcorr_vjp(pcx_fxcorr h, void* gx, void* gg, const void* gy, const void* x, size_t len, int pack,
                              size_t channels, size_t stride, void* stream) {
    return pcx_guard([&]() -> int {
        if (!h) return pcx_fail(PCX_ERR_INVALID, "handle is null");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // d/dx: convolution of gy with g
        if (gx) {
            int rc = run_xc(h, gx, gy, len, pack, channels, stride, stride, true, st);
            if (rc) return rc;
        }
        if (!gg) return PCX_OK;
        if (!x) return pcx_fail(PCX_ERR_INVALID, "kernel gradient needs the forward input x");
        if (int rc = check_pack(pack)) return rc;
        const size_t n    = h->n;
        const size_t step = (n - (h->k - 1)) / pack * pack;
        if (step == 0 || len == 0 || channels == 0) return pcx_fail(PCX_ERR_INVALID, "nothing to differentiate");
        const size_t nblk  = (len + step - 1) / step;
        const size_t total = nblk * channels;
        const size_t eb    = h->dtype == PCX_F64 ? 16 : 8;
        const int    grid  = (int)std::min<size_t>(total, (size_t)h->sms);
        const size_t need  = ((size_t)grid * 2 + 2) * n * eb;
        if (h->gscratch_bytes < need) {
            if (h->gscratch) cudaFree(h->gscratch);
            h->gscratch       = nullptr;
            h->gscratch_bytes = 0;
            PCX_CUDA_TRY(cudaMalloc(&h->gscratch, need));
            h->gscratch_bytes = need;
        }
        if (int rc = ensure_flags(h, 1)) return rc;
        PCX_CUDA_TRY(cudaMemsetAsync(h->ctl, 0, sizeof(unsigned), st));
        char*   base  = static_cast<char*>(h->gscratch);
        kg_args a{};
        a.x       = x;
        a.gy      = gy;
        a.stride  = (long long)stride;
        a.len     = (long long)len;
        a.lp      = __builtin_ctz(pack);
        a.step    = (int)step;
        a.nblk    = (int)nblk;
        a.total   = (long long)total;
        a.counter = h->ctl;
        a.error   = reinterpret_cast<int*>(h->ctl + 1);
        a.acc     = base;
        a.xspec   = base + (size_t)grid * n * eb;
        void* sum = base + (size_t)grid * 2 * n * eb;
        void* inv = base + ((size_t)grid * 2 + 1) * n * eb;
        // FP32 2^13 / 2^14 at pack 8 on 16-byte aligned rows: the in-CTA
        // four-step form with the per-thread spectra in tensor memory
        const bool x2 = h->x2d && pack == 8 && (channels == 1 || stride % 4 == 0) &&
                        (reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(gy)) % 16 == 0;
        int rc;
        if (x2) {
            xc2_kg_args b{};
            b.base = a;
            b.stw1 = h->x2_stw1;
            b.stw2 = h->x2_stw2;
            b.tws  = h->x2_tws;
            rc     = h->log_n == 14 ? launch_xc2_kg<14>(b, st, grid, false) : launch_xc2_kg<13>(b, st, grid, false);
        } else {
            rc = h->dtype == PCX_F64 ? dispatch_kg<double>(h->log_n, a, h->tw, st, grid, false)
                                     : dispatch_kg<float>(h->log_n, a, h->tw, st, grid, false);
        }
        if (rc) return rc;
        if (h->dtype == PCX_F64) {
            k_kgrad_reduce<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
                static_cast<const cpx<double>*>(a.acc), grid, (int)n, static_cast<cpx<double>*>(sum));
        } else {
            k_kgrad_reduce<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
                static_cast<const cpx<float>*>(a.acc), grid, (int)n, static_cast<cpx<float>*>(sum));
        }
        PCX_CUDA_TRY(cudaGetLastError());
        // gg[j] = (1/N) sum_k S[k] e^{+2 pi i jk/N}, j < K
        rc = pcx_fft_run(h->plan, inv, sum, 0, 1, 1, PCX_INVERSE, 1, 1, 2 * n, 2 * n, nullptr, 0, st, 1.0);
        if (rc) return rc;
        const int lpg = __builtin_ctz(h->pack_g);
        if (h->dtype == PCX_F64) {
            k_scale_pack<double><<<(unsigned)((h->k + 255) / 256), 256, 0, st>>>(
                static_cast<const cpx<double>*>(inv), (int)h->k, lpg, static_cast<double*>(gg));
        } else {
            k_scale_pack<float><<<(unsigned)((h->k + 255) / 256), 256, 0, st>>>(
                static_cast<const cpx<float>*>(inv), (int)h->k, lpg, static_cast<float*>(gg));
        }
        PCX_CUDA_TRY(cudaGetLastError());
        return PCX_OK;
    });
}
