// Host side of the FFT: plans (twiddle tables generated on the device in
// FP64), the launch schedule for the single-pass and four-step paths, and the
// FFT entry points of the C ABI (include/pcx_cuda.h).
#include "pcx_fft_kernels.cuh"
#include "pcx_fft_v2.cuh"
#include "pcx_fourstep.cuh"
#include "pcx_host.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>
#include <string>

namespace pcxg {

// ---------------------------------------------------------------- twiddles
template<class T>
__global__ void k_twiddles(cpx<T>* out, int count, int log_n, long long mult) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long e = ((long long)i * mult) & ((1LL << log_n) - 1);
    double          s, c;
    // exp(-2 pi i e / N): the argument 2e/N is exact, sincospi reduces it exactly.
    sincospi(2.0 * (double)e / (double)(1LL << log_n), &s, &c);
    out[i] = {T(c), T(-s)};
}

template<class T>
static cudaError_t gen_twiddles(void* out, int count, int log_n, long long mult, cudaStream_t st) {
    k_twiddles<T><<<(count + 255) / 256, 256, 0, st>>>(reinterpret_cast<cpx<T>*>(out), count, log_n, mult);
    return cudaGetLastError();
}

// ------------------------------------------------------- launch selection
constexpr int SINGLE_NT = 256;

template<class T>
struct kcfg {
    // elements per four-step tile: 64 KB of complex data
    static constexpr int TILE = 65536 / (int)sizeof(cpx<T>);
    static constexpr int NT   = TILE / 16;
    static constexpr int CMIN = 64 / (2 * (int)sizeof(T));    // one 64-byte row segment
};

template<class T, int LOGL>
static cudaError_t launch_single(const io_args& a, const void* tw, cudaStream_t st, bool set_attr) {
    constexpr int M     = SINGLE_NT / splan<LOGL>::TT;
    constexpr int bytes = single_smem_bytes<T, LOGL, SINGLE_NT>();
    auto          kern  = k_single<T, LOGL, SINGLE_NT>;
    if (set_attr) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    if (a.batch == 0) return cudaSuccess;
    const long long grid = (a.batch + M - 1) / M;
    kern<<<(unsigned)grid, SINGLE_NT, bytes, st>>>(a, reinterpret_cast<const cpx<T>*>(tw));
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch_single(int log_n, const io_args& a, const void* tw, cudaStream_t st, bool set_attr) {
    switch (log_n) {
    case 1: return launch_single<T, 1>(a, tw, st, set_attr);
    case 2: return launch_single<T, 2>(a, tw, st, set_attr);
    case 3: return launch_single<T, 3>(a, tw, st, set_attr);
    case 4: return launch_single<T, 4>(a, tw, st, set_attr);
    case 5: return launch_single<T, 5>(a, tw, st, set_attr);
    case 6: return launch_single<T, 6>(a, tw, st, set_attr);
    case 7: return launch_single<T, 7>(a, tw, st, set_attr);
    case 8: return launch_single<T, 8>(a, tw, st, set_attr);
    case 9: return launch_single<T, 9>(a, tw, st, set_attr);
    case 10: return launch_single<T, 10>(a, tw, st, set_attr);
    case 11: return launch_single<T, 11>(a, tw, st, set_attr);
    case 12: return launch_single<T, 12>(a, tw, st, set_attr);
    default: return cudaErrorInvalidValue;
    }
}

template<class T, int LOGL>
static cudaError_t launch_col(const pass_args& a, long long rows, const void* tw, cudaStream_t st, bool set_attr) {
    constexpr int C  = std::max(kcfg<T>::CMIN, kcfg<T>::TILE >> LOGL);
    constexpr int NT = C * splan<LOGL>::TT;
    static_assert(NT == kcfg<T>::NT || C == kcfg<T>::CMIN, "tile shape");
    constexpr int xb    = xch_interleaved<(1 << LOGL), C>::size * (int)sizeof(cpx<T>);
    constexpr int rb    = (1 << LOGL) * 2 * C * (int)sizeof(T);
    constexpr int bytes = xb > rb ? xb : rb;
    auto          kern  = k_colpass<T, LOGL, C, NT>;
    if (set_attr) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    if (rows == 0) return cudaSuccess;
    pass_args b     = a;
    b.tiles_per_row = (1 << a.log_n2) / C;
    kern<<<(unsigned)(rows * b.tiles_per_row), NT, bytes, st>>>(b, reinterpret_cast<const cpx<T>*>(tw));
    return cudaGetLastError();
}

template<class T, int LOGL>
static cudaError_t launch_row(const pass_args& a, long long rows, const void* tw, cudaStream_t st, bool set_attr) {
    constexpr int CR    = std::max(kcfg<T>::CMIN, kcfg<T>::TILE >> LOGL);
    constexpr int NT    = CR * splan<LOGL>::TT;
    constexpr int xb    = xch_blocked<(1 << LOGL), CR>::size * (int)sizeof(cpx<T>);
    constexpr int rb    = CR * 2 * (1 << LOGL) * (int)sizeof(T);
    constexpr int tb    = (1 << LOGL) * (2 * CR + 1) * (int)sizeof(T);
    constexpr int b1    = xb > rb ? xb : rb;
    constexpr int bytes = b1 > tb ? b1 : tb;
    auto          kern  = k_rowpass<T, LOGL, CR, NT>;
    if (set_attr) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    if (rows == 0) return cudaSuccess;
    pass_args b     = a;
    b.tiles_per_row = (1 << a.log_n1) / CR;
    kern<<<(unsigned)(rows * b.tiles_per_row), NT, bytes, st>>>(b, reinterpret_cast<const cpx<T>*>(tw));
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch_col(int logl, const pass_args& a, long long rows, const void* tw, cudaStream_t st,
                                bool set_attr) {
    switch (logl) {
    case 6: return launch_col<T, 6>(a, rows, tw, st, set_attr);
    case 7: return launch_col<T, 7>(a, rows, tw, st, set_attr);
    case 8: return launch_col<T, 8>(a, rows, tw, st, set_attr);
    case 9: return launch_col<T, 9>(a, rows, tw, st, set_attr);
    case 10: return launch_col<T, 10>(a, rows, tw, st, set_attr);
    default: return cudaErrorInvalidValue;
    }
}
template<class T>
static cudaError_t dispatch_row(int logl, const pass_args& a, long long rows, const void* tw, cudaStream_t st,
                                bool set_attr) {
    switch (logl) {
    case 6: return launch_row<T, 6>(a, rows, tw, st, set_attr);
    case 7: return launch_row<T, 7>(a, rows, tw, st, set_attr);
    case 8: return launch_row<T, 8>(a, rows, tw, st, set_attr);
    case 9: return launch_row<T, 9>(a, rows, tw, st, set_attr);
    case 10: return launch_row<T, 10>(a, rows, tw, st, set_attr);
    default: return cudaErrorInvalidValue;
    }
}

}    // namespace pcxg

using namespace pcxg;

cudaError_t pcx_gen_twiddles(void* out, int count, int log_n, long long mult, bool f64, cudaStream_t st) {
    return f64 ? gen_twiddles<double>(out, count, log_n, mult, st) : gen_twiddles<float>(out, count, log_n, mult, st);
}

// ------------------------------------------------------------------- plans
static size_t scratch_cap_bytes() {
    static size_t cap = [] {
        const char* e = std::getenv("PCX_SCRATCH_MB");
        long        v = e ? std::atol(e) : 0;
        return (size_t)(v > 0 ? v : 24) << 20;
    }();
    return cap;
}

size_t pcx_plan_s::chunk_rows(size_t batch) const {
    if (!two_pass) return 0;
    const size_t per = n * elem_bytes();
    size_t       c   = std::max<size_t>(1, scratch_cap_bytes() / per);
    return std::min(c, std::max<size_t>(batch, 1));
}

// Make `v` the plan's one-launch four-step variant: its split's tables (W_N
// tables, W_{16 N2}, full stage tables), generated again only when the split
// changes, and its tile counts and resident blocks per SM.
static int fs_select(pcx_plan_s* p, const fs_variant& v) {
    const bool f64 = p->dtype == PCX_F64;
    if (v.l1 + v.l2 != p->log_n) return pcx_fail(PCX_ERR_INVALID, "four-step variant of another size");
    int tc = 0, tr = 0, per_sm = 0;
    const cudaError_t ea = pcx_fourstep(f64, v, fs_args{}, 0, p->sms, true, &tc, &tr, &per_sm);
    if (ea != cudaSuccess) {
        cudaGetLastError();
        return pcx_fail(ea == cudaErrorNotSupported ? PCX_ERR_UNSUPPORTED : PCX_ERR_CUDA,
                        std::string("four-step variant: ") + cudaGetErrorString(ea));
    }
    if (p->fs_tab_l1 != v.l1 || !p->fs_mem) {
        const size_t eb = p->elem_bytes();
        const int    n1 = 1 << v.l1, n2 = 1 << v.l2;
        int          f1 = 0, f2 = 0;
        PCX_CUDA_TRY(pcx_fourstep_tables(v.l1, nullptr, f64, 0, &f1));
        PCX_CUDA_TRY(pcx_fourstep_tables(v.l2, nullptr, f64, 0, &f2));
        if (p->fs_mem) cudaFree(p->fs_mem);
        p->fs_mem    = nullptr;
        p->fs_tab_l1 = 0;
        const size_t ent = (size_t)n1 + 2 * (size_t)n2 + f1 + f2;
        PCX_CUDA_TRY(cudaMalloc(&p->fs_mem, ent * eb));
        char* b    = static_cast<char*>(p->fs_mem);
        p->fs_thi  = b;
        p->fs_tlo  = b + (size_t)n1 * eb;
        p->fs_tb   = b + ((size_t)n1 + n2) * eb;
        p->fs_st1  = b + ((size_t)n1 + 2 * n2) * eb;
        p->fs_st2  = b + ((size_t)n1 + 2 * n2 + f1) * eb;
        PCX_CUDA_TRY(pcx_gen_twiddles(p->fs_thi, n1, p->log_n, n2, f64, 0));
        PCX_CUDA_TRY(pcx_gen_twiddles(p->fs_tlo, n2, p->log_n, 1, f64, 0));
        PCX_CUDA_TRY(pcx_gen_twiddles(p->fs_tb, n2, v.l2 + 4, 1, f64, 0));
        PCX_CUDA_TRY(pcx_fourstep_tables(v.l1, p->fs_st1, f64, 0, &f1));
        PCX_CUDA_TRY(pcx_fourstep_tables(v.l2, p->fs_st2, f64, 0, &f2));
        p->fs_tab_l1 = v.l1;
    }
    p->fs_var    = v;
    p->fs_tc     = tc;
    p->fs_tr     = tr;
    p->fs_per_sm = per_sm;
    return PCX_OK;
}

// The built-in variants of the one-launch four-step for this plan's size.
static std::vector<fs_variant> fs_candidates(const pcx_plan_s* p) {
    std::vector<fs_variant> out;
    if (p->dtype == PCX_F64) {
        for (const auto& v: kFsVariantsF64) if (v.l1 + v.l2 == p->log_n) out.push_back(v);
    } else {
        for (const auto& v: kFsVariantsF32) if (v.l1 + v.l2 == p->log_n) out.push_back(v);
    }
    return out;
}

static int plan_init_tables(pcx_plan_s* p) {
    const int  log_n = p->log_n;
    const bool f64   = p->dtype == PCX_F64;
    auto       gen   = [&](void* out, int count, int lg, long long mult) {
        return f64 ? gen_twiddles<double>(out, count, lg, mult, 0) : gen_twiddles<float>(out, count, lg, mult, 0);
    };
    const size_t eb = p->elem_bytes();
    if (!p->two_pass) {
        p->tw_bytes = (size_t)p->n * eb;
        PCX_CUDA_TRY(cudaMalloc(&p->tw, p->tw_bytes));
        p->twL = p->tw;
        PCX_CUDA_TRY(gen(p->twL, (int)p->n, log_n, 1));
        PCX_CUDA_TRY(f64 ? dispatch_single<double>(log_n, io_args{}, nullptr, 0, true)
                         : dispatch_single<float>(log_n, io_args{}, nullptr, 0, true));
    } else {
        const int n1 = 1 << p->log_n1, n2 = 1 << p->log_n2;
        p->tw_bytes  = (size_t)(n1 + n2 + n2 + n1) * eb;
        PCX_CUDA_TRY(cudaMalloc(&p->tw, p->tw_bytes));
        char* base = static_cast<char*>(p->tw);
        p->twN1    = base;
        p->twN2    = base + n1 * eb;
        p->tw_lo   = base + (n1 + n2) * eb;
        p->tw_hi   = base + (n1 + 2 * n2) * eb;
        PCX_CUDA_TRY(gen(p->twN1, n1, p->log_n1, 1));
        PCX_CUDA_TRY(gen(p->twN2, n2, p->log_n2, 1));
        PCX_CUDA_TRY(gen(p->tw_lo, n2, log_n, 1));
        PCX_CUDA_TRY(gen(p->tw_hi, n1, log_n, n2));
        pass_args z{};
        z.log_n1 = p->log_n1;
        z.log_n2 = p->log_n2;
        for (int lg: {p->log_n1, p->log_n2}) {
            PCX_CUDA_TRY(f64 ? dispatch_col<double>(lg, z, 0, nullptr, 0, true)
                             : dispatch_col<float>(lg, z, 0, nullptr, 0, true));
            PCX_CUDA_TRY(f64 ? dispatch_row<double>(lg, z, 0, nullptr, 0, true)
                             : dispatch_row<float>(lg, z, 0, nullptr, 0, true));
        }
    }
    PCX_CUDA_TRY(cudaMalloc(&p->err, sizeof(int)));
    PCX_CUDA_TRY(cudaMemset(p->err, 0, sizeof(int)));
    // hot-path tables: stage twiddles per sub-transform, W_{16*N2}^m
    {
        int e1 = 0, e2 = 0;
        if (!p->two_pass) {
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(log_n, nullptr, f64, 0, &e1));
            PCX_CUDA_TRY(cudaMalloc(&p->stw, (size_t)std::max(e1, 2) * eb));
            p->stwL = p->stw;
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(log_n, p->stwL, f64, 0, &e1));
            v2_args z{};
            cudaError_t e = pcx_v2_single(f64, log_n, z, 0, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
            v3_args z3{};
            e = pcx_v3_single(f64, log_n, z3, 0, p->sms, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
        } else {
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(p->log_n1, nullptr, f64, 0, &e1));
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(p->log_n2, nullptr, f64, 0, &e2));
            const size_t nb = (size_t)16 << p->log_n2;
            PCX_CUDA_TRY(cudaMalloc(&p->stw, ((size_t)e1 + e2 + nb) * eb));
            char* base = static_cast<char*>(p->stw);
            p->stw1    = base;
            p->stw2    = base + (size_t)e1 * eb;
            p->tw_b    = base + ((size_t)e1 + e2) * eb;
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(p->log_n1, p->stw1, f64, 0, &e1));
            PCX_CUDA_TRY(pcx_v2_stage_twiddles(p->log_n2, p->stw2, f64, 0, &e2));
            PCX_CUDA_TRY(gen(p->tw_b, (int)nb, p->log_n2 + 4, 1));
            v2_args     z{};
            cudaError_t e = pcx_v2_col(f64, p->log_n1, p->log_n2, z, 0, p->sms, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
            e = pcx_v2_row(f64, p->log_n1, p->log_n2, z, 0, p->sms, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
            e = pcx_v3_col(f64, p->log_n1, p->log_n2, z, 0, 0, nullptr, 0, p->sms, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
            e = pcx_v3_row(f64, p->log_n1, p->log_n2, z, nullptr, 0, p->sms, true);
            if (e != cudaErrorNotSupported) PCX_CUDA_TRY(e);
            PCX_CUDA_TRY(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
            for (int i = 0; i < 2; ++i) {
                PCX_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_col[i], cudaEventDisableTiming));
                PCX_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_row[i], cudaEventDisableTiming));
            }
            PCX_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
            // one launch for all chunks of a batch
            // one launch for a whole batch: the size's first built-in variant
            p->fs_tc = p->fs_tr = 0;
            for (const fs_variant& v: fs_candidates(p)) {
                if (fs_select(p, v) == PCX_OK) break;
                p->fs_tc = p->fs_tr = 0;
            }
            // full stage tables of the two sub-transforms (the TMA-fed passes)
            int f1 = 0, f2 = 0;
            PCX_CUDA_TRY(pcx_fourstep_tables(p->log_n1, nullptr, f64, 0, &f1));
            PCX_CUDA_TRY(pcx_fourstep_tables(p->log_n2, nullptr, f64, 0, &f2));
            PCX_CUDA_TRY(cudaMalloc(&p->fst, ((size_t)f1 + f2) * eb));
            p->fst1 = p->fst;
            p->fst2 = static_cast<char*>(p->fst) + (size_t)f1 * eb;
            PCX_CUDA_TRY(pcx_fourstep_tables(p->log_n1, p->fst1, f64, 0, &f1));
            PCX_CUDA_TRY(pcx_fourstep_tables(p->log_n2, p->fst2, f64, 0, &f2));
            // N = 8192 in FP32 also has a one-pass form (64 KB rows in shared memory)
            v3_args z3{};
            if (pcx_v3_single(f64, log_n, z3, 0, p->sms, true) == cudaSuccess) {
                int e3 = 0;
                PCX_CUDA_TRY(pcx_v2_stage_twiddles(log_n, nullptr, f64, 0, &e3));
                PCX_CUDA_TRY(cudaMalloc(&p->stw_one, (size_t)std::max(e3, 2) * eb));
                PCX_CUDA_TRY(pcx_v2_stage_twiddles(log_n, p->stw_one, f64, 0, &e3));
            }
        }
    }
    PCX_CUDA_TRY(cudaDeviceSynchronize());
    return PCX_OK;
}

extern "C" int pcx_plan_create(pcx_plan* plan, size_t n, int dtype, int order, size_t sub_size) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan pointer is null");
        *plan = nullptr;
        // reference check_size (fft.hpp:1806-1812)
        if (n <= 1 || (n & (n - 1)) != 0) {
            return pcx_fail(PCX_ERR_INVALID, "fft_size (which is " + std::to_string(n) +
                                                 ") is not a power of two or less than 2");
        }
        // reference check_sub_size (fft.hpp:1814-1826)
        if (sub_size < 8 || (sub_size & (sub_size - 1)) != 0) {
            return pcx_fail(PCX_ERR_INVALID, "sub_size (which is " + std::to_string(sub_size) +
                                                 ") is not a power of two or less than 8");
        }
        if (dtype != PCX_F32 && dtype != PCX_F64) return pcx_fail(PCX_ERR_INVALID, "unknown dtype");
        if (order < 0 || order > 2) return pcx_fail(PCX_ERR_INVALID, "unknown fft_order");
        if (n > (size_t(1) << 20)) {
            return pcx_fail(PCX_ERR_UNSUPPORTED,
                            "fft_size (which is " + std::to_string(n) + ") exceeds the largest size built (2^20)");
        }
        if (order == PCX_ORDER_UNORDERED && n < 16) {
            return pcx_fail(PCX_ERR_UNSUPPORTED, "unordered order needs fft_size >= 16");
        }
        auto p      = new pcx_plan_s{};
        p->n        = n;
        p->dtype    = dtype;
        p->order    = order;
        p->sub_size = sub_size;
        p->log_n    = __builtin_ctzll(n);
        p->two_pass = p->log_n > 12;
        p->log_n1   = (p->log_n + 1) / 2;
        p->log_n2   = p->log_n / 2;
        cudaGetDevice(&p->device);
        if (cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess) {
            (void)cudaGetLastError();
            p->sms = 148;
        }
        int rc = plan_init_tables(p);
        if (rc != PCX_OK) {
            p->release();
            delete p;
            return rc;
        }
        *plan = p;
        return PCX_OK;
    });
}

void pcx_plan_s::release() {
    if (tw) cudaFree(tw);
    if (stw) cudaFree(stw);
    if (stw_one) cudaFree(stw_one);
    if (fst) cudaFree(fst);
    if (fs_mem) cudaFree(fs_mem);
    fs_mem    = nullptr;
    fs_tab_l1 = 0;
    if (fs_ctr) cudaFree(fs_ctr);
    if (par_buf) cudaFree(par_buf);
    par_buf   = nullptr;
    par_bytes = 0;
    if (scratch) cudaFree(scratch);
    if (side) cudaStreamDestroy(side);
    for (int i = 0; i < 2; ++i) {
        if (ev_col[i]) cudaEventDestroy(ev_col[i]);
        if (ev_row[i]) cudaEventDestroy(ev_row[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (err) cudaFree(err);
    err = nullptr;
    tw      = nullptr;
    stw     = nullptr;
    stw_one  = nullptr;
    fst      = nullptr;
    fst1     = nullptr;
    fst2     = nullptr;
    fs_ctr   = nullptr;
    fs_ctr_n = 0;
    scratch  = nullptr;
    side    = nullptr;
}

extern "C" int pcx_plan_destroy(pcx_plan plan) {
    return pcx_guard([&]() -> int {
        if (!plan) return PCX_OK;
        plan->release();
        delete plan;
        return PCX_OK;
    });
}

extern "C" size_t pcx_plan_size(pcx_plan plan) { return plan ? plan->n : 0; }

extern "C" int pcx_plan_status(pcx_plan plan) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        int err = 0;
        PCX_CUDA_TRY(cudaMemcpy(&err, plan->err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) {
            PCX_CUDA_TRY(cudaMemset(plan->err, 0, sizeof(int)));
            return pcx_fail(PCX_ERR_TIMEOUT, "a transform of this plan gave up waiting for its input copy");
        }
        return PCX_OK;
    });
}

namespace {
// Name of the current device, the tuning cache's GPU key.
std::string gpu_name() {
    int            dev = 0;
    cudaDeviceProp pr{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    return pr.name;
}

// The plan's current choice as a cache / report record.
pcx_tune_result plan_choice(const pcx_plan_s* p, double ms) {
    pcx_tune_result r{};
    r.form          = p->form;
    r.rounds        = p->fs_rounds;
    r.chunk_bytes   = p->chunk_bytes;
    r.log_n1        = p->fs_var.l1;
    r.log_n2        = p->fs_var.l2;
    r.blocks_per_sm = p->fs_var.minb;
    r.stages        = p->fs_var.st;
    r.ms            = ms;
    return r;
}

// Apply a tuning record to the plan; false if it names a variant not built here.
bool apply_choice(pcx_plan_s* p, const pcx_tune_result& r) {
    if (r.form == PCX_FORM_FUSED || (r.form == PCX_FORM_DEFAULT && r.log_n1 > 0)) {
        const fs_variant v{r.log_n1, r.log_n2, r.blocks_per_sm, r.stages};
        if (fs_select(p, v) != PCX_OK) return false;
    }
    if (r.form == PCX_FORM_ONEPASS && !p->stw_one) return false;
    p->form        = r.form;
    p->fs_rounds   = r.rounds > 0 ? r.rounds : 3;
    p->chunk_bytes = r.chunk_bytes;
    return true;
}

std::once_flag g_cache_once;
}    // namespace

extern "C" int pcx_plan_tune(pcx_plan plan, size_t batch, void* stream, int* form_out) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        pcx_plan_s* p = plan;
        if (form_out) *form_out = p->form;
        if (!p->two_pass || batch == 0) return PCX_OK;
        const size_t eb    = p->elem_bytes();
        const size_t rows  = std::max<size_t>(1, std::min(batch, ((size_t)512 << 20) / (p->n * eb)));
        const char*  cpath = std::getenv("PCX_TUNE_CACHE");
        const bool   verbose = std::getenv("PCX_TUNE_VERBOSE") != nullptr;
        const std::string gpu = gpu_name();
        if (cpath && *cpath) {
            // a missing or unreadable file just means nothing is cached yet
            std::call_once(g_cache_once, [&]() { (void)pcx_tune_cache_load(cpath); });
            pcx_tune_result hit{};
            if (pcx_tune_cache_get(gpu.c_str(), p->n, p->dtype, rows, &hit) == PCX_OK && apply_choice(p, hit)) {
                if (form_out) *form_out = p->form;
                return PCX_OK;
            }
        }
        struct cand {
            int        form;
            int        rounds;
            size_t     chunk;
            fs_variant v;
        };
        std::vector<cand> cands;
        if (p->stw_one) cands.push_back({PCX_FORM_ONEPASS, 3, 0, {}});
        if (p->fs_tc > 0) {
            for (const fs_variant& v: fs_candidates(p)) {
                for (int r: {2, 3, 6}) cands.push_back({PCX_FORM_FUSED, r, 0, v});
            }
        }
        for (size_t mb: {24, 48}) cands.push_back({PCX_FORM_CHUNKED, 3, mb << 20, {}});
        const size_t bytes = rows * p->n * eb;
        cudaStream_t st    = static_cast<cudaStream_t>(stream);
        void *       x = nullptr, *y = nullptr;
        cudaEvent_t  e0 = nullptr, e1 = nullptr;
        auto         cleanup = [&]() {
            if (x) cudaFree(x);
            if (y) cudaFree(y);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        };
        const pcx_tune_result keep = plan_choice(p, 0.0);
        const fs_variant      keep_var = p->fs_var;
        auto restore = [&]() {
            if (keep_var.l1 > 0) fs_select(p, keep_var);
            p->form        = keep.form;
            p->fs_rounds   = keep.rounds;
            p->chunk_bytes = keep.chunk_bytes;
        };
        cudaError_t e = cudaMalloc(&x, bytes);
        if (e == cudaSuccess) e = cudaMalloc(&y, bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(x, 0, bytes, st);
        if (e == cudaSuccess) e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e != cudaSuccess) {
            cleanup();
            return pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e));
        }
        const size_t row    = 2 * p->n;
        const int    pk     = p->dtype == PCX_F64 ? 4 : 8;
        float        best_ms = 0.f;
        cand         best{keep.form, keep.rounds, keep.chunk_bytes, keep_var};
        for (const cand& c: cands) {
            if (c.form == PCX_FORM_FUSED && !(c.v == p->fs_var) && fs_select(p, c.v) != PCX_OK) continue;
            p->form        = c.form;
            p->fs_rounds   = c.rounds;
            p->chunk_bytes = c.chunk;
            int rc = PCX_OK;
            for (int w = 0; w < 2 && rc == PCX_OK; ++w) {
                rc = pcx_fft_run(p, y, x, p->n, pk, pk, PCX_FORWARD, 0, rows, row, row, nullptr, 0, st, 1.0);
            }
            if (rc == PCX_OK) e = cudaEventRecord(e0, st);
            for (int it = 0; it < 3 && rc == PCX_OK && e == cudaSuccess; ++it) {
                rc = pcx_fft_run(p, y, x, p->n, pk, pk, PCX_FORWARD, 0, rows, row, row, nullptr, 0, st, 1.0);
            }
            if (rc == PCX_OK && e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (rc == PCX_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (rc == PCX_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (rc != PCX_OK || e != cudaSuccess) {
                restore();
                cleanup();
                return rc != PCX_OK ? rc : pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e));
            }
            ms /= 3.f;
            if (verbose) {
                std::fprintf(stderr, "pcx_plan_tune n=%zu rows=%zu form=%d split=%dx%d blocks/SM=%d stages=%d rounds=%d "
                             "chunk=%zuMB: %.4f ms\n", p->n, rows, c.form, 1 << c.v.l1, 1 << c.v.l2, c.v.minb, c.v.st,
                             c.rounds, c.chunk >> 20, ms);
            }
            if (best_ms == 0.f || ms < best_ms) {
                best_ms = ms;
                best    = c;
            }
        }
        if (best.form == PCX_FORM_FUSED || (best.form == PCX_FORM_DEFAULT && best.v.l1 > 0)) {
            if (int rc = fs_select(p, best.v)) {
                restore();
                cleanup();
                return rc;
            }
        } else if (keep_var.l1 > 0 && !(p->fs_var == keep_var)) {
            fs_select(p, keep_var);
        }
        p->form        = best.form;
        p->fs_rounds   = best.rounds;
        p->chunk_bytes = best.chunk;
        cleanup();
        if (cpath && *cpath) {
            const pcx_tune_result r = plan_choice(p, best_ms);
            pcx_tune_cache_put(gpu.c_str(), p->n, p->dtype, rows, &r);
            pcx_tune_cache_save(cpath);
        }
        if (form_out) *form_out = p->form;
        return PCX_OK;
    });
}

extern "C" int pcx_plan_set_tuning(pcx_plan plan, const pcx_tune_result* r) {
    return pcx_guard([&]() -> int {
        if (!plan || !r) return pcx_fail(PCX_ERR_INVALID, "null argument");
        if (!plan->two_pass) {
            if (r->form != PCX_FORM_DEFAULT) return pcx_fail(PCX_ERR_UNSUPPORTED, "sizes up to 4096 have one form");
            return PCX_OK;
        }
        if (r->form < PCX_FORM_DEFAULT || r->form > PCX_FORM_CHUNKED) return pcx_fail(PCX_ERR_INVALID, "unknown form");
        if (!apply_choice(plan, *r)) {
            return pcx_fail(PCX_ERR_UNSUPPORTED, "this form or four-step variant is not built for the plan's size");
        }
        return PCX_OK;
    });
}

extern "C" int pcx_plan_tuning(pcx_plan plan, pcx_tune_result* out) {
    return pcx_guard([&]() -> int {
        if (!plan || !out) return pcx_fail(PCX_ERR_INVALID, "null argument");
        *out = plan_choice(plan, 0.0);
        if (out->chunk_bytes == 0) out->chunk_bytes = (size_t)24 << 20;
        return PCX_OK;
    });
}

extern "C" int pcx_plan_form(pcx_plan plan, int* form, int* rounds, size_t* chunk_bytes) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        if (form) *form = plan->form;
        if (rounds) *rounds = plan->fs_rounds;
        if (chunk_bytes) *chunk_bytes = plan->chunk_bytes ? plan->chunk_bytes : ((size_t)24 << 20);
        return PCX_OK;
    });
}

extern "C" size_t pcx_plan_workspace_size(pcx_plan plan, size_t batch) {
    if (!plan || !plan->two_pass) return 0;
    return 2 * plan->chunk_rows(batch) * plan->n * plan->elem_bytes();
}

// ------------------------------------------------------------------ exec
namespace {
int check_pack(int pack, const char* what) {
    if (pack < 1 || (pack & (pack - 1)) != 0) {
        return pcx_fail(PCX_ERR_INVALID, std::string(what) + " pack size (which is " + std::to_string(pack) +
                                             ") is not a power of two");
    }
    return PCX_OK;
}

// Pack width change of `rows` rows of 2 * n reals (packs of at most 16, the
// reference's widest; avx2_common.hpp:243-435 converts between its widths in
// the FFT's loads and stores).  Each warp moves 32 consecutive reals of a row:
// whole blocks of 2 * max(pack) reals, so the permutation stays inside the
// warp, and every lane reads before any lane writes (dst may be src).
template<class T>
__global__ void k_repack(T* dst, const T* src, int lp_to, int lp_from, long long chunks, long long rows,
                         long long dstride, long long sstride) {
    const long long w    = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int       lane = threadIdx.x & 31;
    if (w >= chunks * rows) return;    // uniform over the warp
    const long long r  = w / chunks;
    const long long o  = (w - r * chunks) * 32 + lane;    // offset of this real, source layout
    const T         v  = src[r * sstride + o];
    const long long e  = ((o >> (lp_from + 1)) << lp_from) | (o & ((1LL << lp_from) - 1));
    const long long im = (o >> lp_from) & 1;
    const long long d  = ((e >> lp_to) << (lp_to + 1)) + (e & ((1LL << lp_to) - 1)) + (im << lp_to);
    __syncwarp();
    dst[r * dstride + d] = v;
}

int repack(bool f64, void* dst, const void* src, int pack_to, int pack_from, size_t n, size_t rows,
           size_t dstride, size_t sstride, cudaStream_t st) {
    const long long chunks = (long long)(2 * n / 32);
    const long long warps  = chunks * (long long)rows;
    const unsigned  grid   = (unsigned)((warps * 32 + 255) / 256);
    const int       lt = __builtin_ctz(pack_to), lf = __builtin_ctz(pack_from);
    if (f64) {
        k_repack<double><<<grid, 256, 0, st>>>(static_cast<double*>(dst), static_cast<const double*>(src), lt, lf,
                                                chunks, (long long)rows, (long long)dstride, (long long)sstride);
    } else {
        k_repack<float><<<grid, 256, 0, st>>>(static_cast<float*>(dst), static_cast<const float*>(src), lt, lf,
                                               chunks, (long long)rows, (long long)dstride, (long long)sstride);
    }
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}
}    // namespace

int pcx_fft_run(pcx_plan_s* p, void* dst, const void* src, size_t src_len, int pd, int ps, int dir, int norm,
                size_t batch, size_t dstride, size_t sstride, void* ws, size_t ws_bytes, cudaStream_t st,
                double extra_scale, size_t chunk_cap) {
    if (!p) return pcx_fail(PCX_ERR_INVALID, "plan is null");
    if (int rc = check_pack(pd, "destination")) return rc;
    if (int rc = check_pack(ps, "source")) return rc;
    const size_t n = p->n;
    if (src_len == 0) src_len = n;
    if (src_len > n) {
        return pcx_fail(PCX_ERR_INVALID, "source size (which is " + std::to_string(src_len) +
                                             ") is bigger than fft size (which is " + std::to_string(n) + ")");
    }
    if (dir == PCX_INVERSE && src_len != n) {
        return pcx_fail(PCX_ERR_INVALID, "source size (which is " + std::to_string(src_len) +
                                             ") is not equal to fft size (which is " + std::to_string(n) + ")");
    }
    if (dir != PCX_FORWARD && dir != PCX_INVERSE) return pcx_fail(PCX_ERR_INVALID, "unknown direction");
    if ((size_t)pd > n || (size_t)ps > n) {
        return pcx_fail(PCX_ERR_UNSUPPORTED, "pack size larger than fft size is not supported");
    }
    const int cmin = p->dtype == PCX_F64 ? kcfg<double>::CMIN : kcfg<float>::CMIN;
    const bool wide = p->two_pass && (pd > cmin || ps > cmin);
    if (wide && (pd > 16 || ps > 16 || (ps > cmin && src_len != n))) {
        return pcx_fail(PCX_ERR_UNSUPPORTED, "pack sizes above " + std::to_string(ps > cmin && src_len != n ? cmin : 16) +
                                                 " are not supported for fft_size > 4096" +
                                                 (src_len != n ? " with a short source" : ""));
    }
    if (batch == 0) return PCX_OK;
    if (!dst || !src) return pcx_fail(PCX_ERR_INVALID, "null data pointer");
    const size_t vreals = 16 / (p->dtype == PCX_F64 ? sizeof(double) : sizeof(float));
    if (p->two_pass && batch > 1 && (dstride % vreals != 0 || sstride % vreals != 0)) {
        return pcx_fail(PCX_ERR_UNSUPPORTED, "row strides must be multiples of 16 bytes for fft_size > 4096");
    }
    if ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) % 16 != 0) {
        return pcx_fail(PCX_ERR_INVALID, "data pointers must be 16-byte aligned");
    }
    const size_t row_d = n * 2, row_s = n * 2;
    if (batch > 1 && (dstride < row_d || sstride < (src_len == n ? row_s : 0))) {
        return pcx_fail(PCX_ERR_INVALID, "row stride smaller than a row");
    }
    if (wide) {
        // the two-pass kernels read and write packs of up to `cmin`: a wider
        // source is repacked into dst first, a wider destination after
        const bool   f64 = p->dtype == PCX_F64;
        const size_t ds = batch > 1 ? dstride : row_d, ss = batch > 1 ? sstride : row_s;
        const void*  s2 = src;
        size_t       ss2 = ss;
        if (ps > cmin) {
            if (int rc = repack(f64, dst, src, cmin, ps, n, batch, ds, ss, st)) return rc;
            s2  = dst;
            ss2 = ds;
        }
        if (int rc = pcx_fft_run(p, dst, s2, src_len, std::min(pd, cmin), std::min(ps, cmin), dir, norm, batch, ds,
                                 ss2, ws, ws_bytes, st, extra_scale, chunk_cap)) {
            return rc;
        }
        if (pd > cmin) return repack(f64, dst, dst, pd, cmin, n, batch, ds, ds, st);
        return PCX_OK;
    }
    const bool   inv   = dir == PCX_INVERSE;
    const double scale = (inv && norm ? 1.0 / (double)n : 1.0) * extra_scale;

    io_args io{};
    io.src_stride = (long long)sstride;
    io.dst_stride = (long long)dstride;
    io.src_len    = (int)src_len;
    io.lp_src     = __builtin_ctz(ps);
    io.lp_dst     = __builtin_ctz(pd);
    io.order_in   = inv ? p->order : 0;
    io.order_out  = inv ? 0 : p->order;
    io.conj_in    = inv;
    io.conj_out   = inv;
    io.scale      = scale;
    const bool f64 = p->dtype == PCX_F64;
    const size_t eb = p->elem_bytes();
    const int    lp_def = f64 ? 2 : 3;    // default pack: 32 bytes of reals

    // hot-path argument block for the pcx_fft_v2.cuh kernels
    v2_args h{};
    h.conj_in  = io.conj_in;
    h.conj_out = io.conj_out;
    h.scale    = io.scale;

    if (!p->two_pass) {
        // TMA-fed kernel: any order, default pack, full-length rows on 16-byte strides
        const size_t vr = 16 / (f64 ? sizeof(double) : sizeof(float));
        const bool   tma = src_len == n && io.lp_src == lp_def && io.lp_dst == lp_def && p->log_n >= 5 &&
                         (batch == 1 || (sstride % vr == 0 && dstride % vr == 0));
        if (tma) {
            v3_args t3{};
            t3.src        = src;
            t3.dst        = dst;
            t3.src_stride = (long long)sstride;
            t3.dst_stride = (long long)dstride;
            t3.batch      = (long long)batch;
            t3.conj_in    = io.conj_in;
            t3.conj_out   = io.conj_out;
            t3.order_in   = io.order_in;
            t3.order_out  = io.order_out;
            t3.scale      = io.scale;
            t3.stw        = p->stwL;
            t3.error      = p->err;
            cudaError_t e = pcx_v3_single(f64, p->log_n, t3, st, p->sms, false);
            if (e != cudaErrorNotSupported) {
                PCX_CUDA_TRY(e);
                return PCX_OK;
            }
        }
        const bool hot = io.order_in == 0 && io.order_out == 0 && src_len == n && io.lp_src == lp_def &&
                         io.lp_dst == lp_def && p->log_n >= 7;
        if (hot) {
            h.src        = src;
            h.dst        = dst;
            h.src_stride = (long long)sstride;
            h.dst_stride = (long long)dstride;
            h.batch      = (long long)batch;
            h.stw        = p->stwL;
            cudaError_t e = pcx_v2_single(f64, p->log_n, h, st, false);
            if (e != cudaErrorNotSupported) {
                PCX_CUDA_TRY(e);
                return PCX_OK;
            }
        }
        io.src   = src;
        io.dst   = dst;
        io.batch = (long long)batch;
        PCX_CUDA_TRY(f64 ? dispatch_single<double>(p->log_n, io, p->twL, st, false)
                         : dispatch_single<float>(p->log_n, io, p->twL, st, false));
        return PCX_OK;
    }

    const bool tuned_one = ws || p->form == PCX_FORM_DEFAULT || p->form == PCX_FORM_ONEPASS;
    if (p->stw_one && tuned_one && src_len == n && io.lp_src == lp_def && io.lp_dst == lp_def &&
        (batch == 1 || (sstride % vreals == 0 && dstride % vreals == 0))) {
        // one-pass form of a two-pass size
        v3_args t3{};
        t3.src        = src;
        t3.dst        = dst;
        t3.src_stride = (long long)sstride;
        t3.dst_stride = (long long)dstride;
        t3.batch      = (long long)batch;
        t3.conj_in    = io.conj_in;
        t3.conj_out   = io.conj_out;
        t3.order_in   = io.order_in;
        t3.order_out  = io.order_out;
        t3.scale      = io.scale;
        t3.stw        = p->stw_one;
        t3.error      = p->err;
        cudaError_t e = pcx_v3_single(f64, p->log_n, t3, st, p->sms, false);
        if (e != cudaErrorNotSupported) {
            PCX_CUDA_TRY(e);
            return PCX_OK;
        }
    }

    // Four-step through L2-sized chunks of scratch.  With two scratch buffers
    // the passes are pipelined over two streams: the column pass of chunk c+1
    // (caller's stream) runs beside the row pass of chunk c (side stream).
    size_t       chunk = chunk_cap ? std::min(chunk_cap, p->chunk_rows(batch)) : p->chunk_rows(batch);
    const size_t per   = n * eb;
    if (!ws && p->chunk_bytes > 0) chunk = std::max<size_t>(1, std::min(batch, p->chunk_bytes / per));
    void*        scr   = ws;
    int          nbuf  = 2;
    if (!scr) {
        const size_t need = 2 * chunk * per;
        if (p->scratch_bytes < need) {
            if (p->scratch) cudaFree(p->scratch);
            p->scratch       = nullptr;
            p->scratch_bytes = 0;
            PCX_CUDA_TRY(cudaMalloc(&p->scratch, need));
            p->scratch_bytes = need;
        }
        scr = p->scratch;
    } else {
        if (ws_bytes < chunk * per) {
            if (chunk_cap == 0) return pcx_fail(PCX_ERR_INVALID, "workspace smaller than pcx_plan_workspace_size");
            chunk = std::max<size_t>(1, ws_bytes / per);
        }
        if (ws_bytes >= 2 * chunk * per) {
            nbuf = 2;
        } else if (ws_bytes >= 2 * per) {
            chunk = ws_bytes / (2 * per);
            nbuf  = 2;
        } else {
            nbuf = 1;
        }
    }
    const int nchunks = (int)((batch + chunk - 1) / chunk);
    if (nchunks <= 1) nbuf = 1;

    const size_t es     = f64 ? sizeof(double) : sizeof(float);
    const bool   direct = !(inv && p->order != 0);
    // hot-path eligibility of each pass
    const bool col_hot = direct && src_len == n && io.lp_src == lp_def;
    const bool use_tma = std::getenv("PCX_NO_TMA") == nullptr;
    const bool row_hot = direct && io.order_out == 0 && io.lp_dst == lp_def;

    // One launch over the whole batch (plan-owned scratch slots and counters);
    // PCX_FOURSTEP=chunked selects the two-launch chunk pipeline below.
    const char* fs_env = std::getenv("PCX_FOURSTEP");
    const bool tuned_fused = p->form == PCX_FORM_DEFAULT || p->form == PCX_FORM_FUSED;
    if (!ws && tuned_fused && col_hot && row_hot && use_tma && p->fs_tc > 0 &&
        !(fs_env && std::strcmp(fs_env, "chunked") == 0)) {
        const long long per_t = p->fs_tc + p->fs_tr;
        // a row tile runs about `rounds` rounds of items (one item per CTA)
        // after its transform's column tiles, and a slot is rewritten about as
        // long after its row tiles, so both dependencies have usually cleared
        // by the time the copy warp reaches them
        const char*     re     = std::getenv("PCX_FS_ROUNDS");
        const long long rounds = re && std::atol(re) > 0 ? std::atol(re) : p->fs_rounds;
        const long long ctas   = (long long)p->sms * std::max(1, p->fs_per_sm);
        long long       lag    = (rounds * ctas + per_t - 1) / per_t;
        lag                    = std::max<long long>(1, std::min<long long>(lag, (long long)batch));
        // slots in use at once: lag transforms between a column tile and its
        // row tiles, on both sides; rounded up to a power of two so that the
        // kernel finds a transform's slot with a mask
        long long nslot = 1;
        while (nslot < std::min<long long>((long long)batch, 2 * lag + 2)) nslot *= 2;
        std::lock_guard<std::mutex> g(p->mu);
        const size_t need = (size_t)nslot * per;
        if (p->scratch_bytes < need) {
            if (p->scratch) cudaFree(p->scratch);
            p->scratch       = nullptr;
            p->scratch_bytes = 0;
            PCX_CUDA_TRY(cudaMalloc(&p->scratch, need));
            p->scratch_bytes = need;
        }
        if (p->fs_ctr_n < 2 * batch) {
            if (p->fs_ctr) cudaFree(p->fs_ctr);
            p->fs_ctr   = nullptr;
            p->fs_ctr_n = 0;
            PCX_CUDA_TRY(cudaMalloc(&p->fs_ctr, 2 * batch * sizeof(int)));
            p->fs_ctr_n = 2 * batch;
        }
        PCX_CUDA_TRY(cudaMemsetAsync(p->fs_ctr, 0, 2 * batch * sizeof(int), st));
        fs_args a{};
        a.src        = src;
        a.dst        = dst;
        a.src_stride = (long long)sstride;
        a.dst_stride = (long long)dstride;
        a.batch      = (long long)batch;
        a.conj_in    = io.conj_in;
        a.conj_out   = io.conj_out;
        a.scale      = io.scale;
        a.stw1       = p->fs_st1;
        a.stw2       = p->fs_st2;
        a.tw_hi      = p->fs_thi;
        a.tw_lo      = p->fs_tlo;
        a.tw_b       = p->fs_tb;
        a.scratch    = p->scratch;
        a.nslot      = (int)nslot;
        a.lag        = (int)lag;
        a.col_done   = p->fs_ctr;
        a.row_done   = p->fs_ctr + batch;
        a.error      = p->err;
        PCX_CUDA_TRY(pcx_fourstep(f64, p->fs_var, a, st, p->sms, false, nullptr, nullptr, nullptr));
        return PCX_OK;
    }

    std::unique_lock<std::mutex> lock(p->mu, std::defer_lock);
    if (nbuf == 2) {
        lock.lock();
        PCX_CUDA_TRY(cudaEventRecord(p->ev_fork, st));
        PCX_CUDA_TRY(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    }
    for (int ci = 0; ci < nchunks; ++ci) {
        const size_t    r0   = (size_t)ci * chunk;
        const long long rows = (long long)std::min(chunk, batch - r0);
        const char*     s    = static_cast<const char*>(src) + r0 * sstride * es;
        char*           d    = static_cast<char*>(dst) + r0 * dstride * es;
        const int       b    = nbuf == 2 ? (ci & 1) : 0;
        void*           buf  = static_cast<char*>(scr) + (size_t)b * chunk * per;
        cudaStream_t    st2  = nbuf == 2 ? p->side : st;
        if (nbuf == 2 && ci >= 2) PCX_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_row[b], 0));

        pass_args a{};
        a.log_n1 = p->log_n1;
        a.log_n2 = p->log_n2;
        a.log_lo = p->log_n2;
        a.tw_hi  = p->tw_hi;
        a.tw_lo  = p->tw_lo;
        pass_args bb = a;
        if (direct) {
            // pass 1: columns src -> scratch (with twiddle); pass 2: rows scratch -> dst
            bool done = false;
            if (col_hot) {
                v2_args c = h;
                c.src        = src;
                c.dst        = buf;
                c.src_stride = (long long)sstride;
                c.dst_stride = (long long)(2 * n);
                c.batch      = rows;
                c.conj_out   = 0;
                c.scale      = 1.0;
                c.stw        = p->fst1;
                c.tw_hi      = p->tw_hi;
                c.tw_lo      = p->tw_lo;
                c.tw_b       = p->tw_b;
                cudaError_t e = use_tma ? pcx_v3_col(f64, p->log_n1, p->log_n2, c, (long long)batch, (long long)r0,
                                                     p->err, st, p->sms, false)
                                        : cudaErrorNotSupported;
                if (e != cudaErrorNotSupported) {
                    PCX_CUDA_TRY(e);
                    done = true;
                }
                c.src = s;
            }
            if (!done && col_hot) {
                v2_args c = h;
                c.src        = s;
                c.dst        = buf;
                c.src_stride = (long long)sstride;
                c.dst_stride = (long long)(2 * n);
                c.batch      = rows;
                c.conj_out   = 0;
                c.scale      = 1.0;
                c.stw        = p->stw1;
                c.tw_hi      = p->tw_hi;
                c.tw_lo      = p->tw_lo;
                c.tw_b       = p->tw_b;
                cudaError_t e = pcx_v2_col(f64, p->log_n1, p->log_n2, c, st, p->sms, false);
                if (e != cudaErrorNotSupported) {
                    PCX_CUDA_TRY(e);
                    done = true;
                }
            }
            if (!done) {
                a.io            = io;
                a.io.src        = s;
                a.io.dst        = buf;
                a.io.dst_stride = (long long)(2 * n);
                a.io.lp_dst     = 0;
                a.io.conj_out   = 0;
                a.io.scale      = 1.0;
                a.io.order_out  = 0;
                a.twiddle       = 1;
                PCX_CUDA_TRY(f64 ? dispatch_col<double>(p->log_n1, a, rows, p->twN1, st, false)
                                 : dispatch_col<float>(p->log_n1, a, rows, p->twN1, st, false));
            }
            if (nbuf == 2) {
                PCX_CUDA_TRY(cudaEventRecord(p->ev_col[b], st));
                PCX_CUDA_TRY(cudaStreamWaitEvent(st2, p->ev_col[b], 0));
            }
            done = false;
            if (row_hot && use_tma) {
                v2_args r = h;
                r.src        = buf;
                r.dst        = d;
                r.src_stride = (long long)(2 * n);
                r.dst_stride = (long long)dstride;
                r.batch      = rows;
                r.conj_in    = 0;
                r.stw        = p->fst2;
                cudaError_t e = pcx_v3_row(f64, p->log_n1, p->log_n2, r, p->err, st2, p->sms, false);
                if (e != cudaErrorNotSupported) {
                    PCX_CUDA_TRY(e);
                    done = true;
                }
            }
            if (!done && row_hot) {
                v2_args r = h;
                r.src        = buf;
                r.dst        = d;
                r.src_stride = (long long)(2 * n);
                r.dst_stride = (long long)dstride;
                r.batch      = rows;
                r.conj_in    = 0;
                r.stw        = p->stw2;
                cudaError_t e = pcx_v2_row(f64, p->log_n1, p->log_n2, r, st2, p->sms, false);
                if (e != cudaErrorNotSupported) {
                    PCX_CUDA_TRY(e);
                    done = true;
                }
            }
            if (!done) {
                bb.io             = io;
                bb.io.src         = buf;
                bb.io.src_stride  = (long long)(2 * n);
                bb.io.src_len     = (int)n;
                bb.io.lp_src      = 0;
                bb.io.conj_in     = 0;
                bb.io.order_in    = 0;
                bb.io.dst         = d;
                bb.twiddle        = 0;
                bb.transposed_out = io.order_out == 0;
                bb.row_map        = io.order_out != 0;
                PCX_CUDA_TRY(f64 ? dispatch_row<double>(p->log_n2, bb, rows, p->twN2, st2, false)
                                 : dispatch_row<float>(p->log_n2, bb, rows, p->twN2, st2, false));
            }
        } else {
            // inverse from a permuted order: rows first (input rows), then columns
            a.io             = io;
            a.io.src         = s;
            a.io.dst         = buf;
            a.io.dst_stride  = (long long)(2 * n);
            a.io.lp_dst      = 0;
            a.io.conj_out    = 0;
            a.io.scale       = 1.0;
            a.io.order_out   = 0;
            a.twiddle        = 1;
            a.row_map        = 1;
            a.transposed_out = 0;
            bb.io            = io;
            bb.io.src        = buf;
            bb.io.src_stride = (long long)(2 * n);
            bb.io.src_len    = (int)n;
            bb.io.lp_src     = 0;
            bb.io.conj_in    = 0;
            bb.io.order_in   = 0;
            bb.io.dst        = d;
            bb.twiddle       = 0;
            PCX_CUDA_TRY(f64 ? dispatch_row<double>(p->log_n2, a, rows, p->twN2, st, false)
                             : dispatch_row<float>(p->log_n2, a, rows, p->twN2, st, false));
            if (nbuf == 2) {
                PCX_CUDA_TRY(cudaEventRecord(p->ev_col[b], st));
                PCX_CUDA_TRY(cudaStreamWaitEvent(st2, p->ev_col[b], 0));
            }
            PCX_CUDA_TRY(f64 ? dispatch_col<double>(p->log_n1, bb, rows, p->twN1, st2, false)
                             : dispatch_col<float>(p->log_n1, bb, rows, p->twN1, st2, false));
        }
        if (nbuf == 2) PCX_CUDA_TRY(cudaEventRecord(p->ev_row[b], st2));
    }
    if (nbuf == 2) {
        // join: the caller's stream waits for the last row passes
        PCX_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_row[(nchunks - 1) & 1], 0));
        if (nchunks >= 2) PCX_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_row[(nchunks - 2) & 1], 0));
    }
    return PCX_OK;
}

extern "C" int pcx_fft_exec_ws(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst,
                               int pack_src, int direction, int normalize, size_t batch, size_t dst_stride,
                               size_t src_stride, void* workspace, size_t workspace_bytes, void* stream) {
    return pcx_guard([&]() -> int {
        return pcx_fft_run(plan, dst, src, src_len, pack_dst, pack_src, direction, normalize, batch, dst_stride,
                           src_stride, workspace, workspace_bytes, static_cast<cudaStream_t>(stream), 1.0);
    });
}

extern "C" int pcx_fft_exec(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst, int pack_src,
                            int direction, int normalize, size_t batch, size_t dst_stride, size_t src_stride,
                            void* stream) {
    return pcx_fft_exec_ws(plan, dst, src, src_len, pack_dst, pack_src, direction, normalize, batch, dst_stride,
                           src_stride, nullptr, 0, stream);
}

// Adjoint: y = F x  =>  x_bar = F^H y_bar, the unnormalised inverse read in
// the plan's order.  y = s * F^H x  =>  x_bar = s * F y_bar.
extern "C" int pcx_fft_vjp(pcx_plan plan, void* g_in, const void* g_out, int pack, int direction, int normalize,
                           size_t batch, size_t stride, void* stream) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (direction == PCX_FORWARD) {
            return pcx_fft_run(plan, g_in, g_out, 0, pack, pack, PCX_INVERSE, 0, batch, stride, stride, nullptr, 0,
                               st, 1.0);
        }
        const double s = normalize ? 1.0 / (double)plan->n : 1.0;
        return pcx_fft_run(plan, g_in, g_out, 0, pack, pack, PCX_FORWARD, 0, batch, stride, stride, nullptr, 0, st,
                           s);
    });
}
