// Ragged persistent batch: FFTs of uneven power-of-two sizes and overlap-save
// correlations, all in ONE persistent launch fed by a device work queue and
// replayed from a CUDA graph.
//
// Work items (built once on the host, executed in queue order; every CTA
// claims the next item with an atomic counter):
//   SINGLE  up to M whole transforms of one size N <= 4096
//   COL     one column tile of a four-step transform (N = 2^13..2^18): writes
//           the transform's scratch slot, then counts itself in col_done[t]
//   ROW     one row tile: waits until col_done[t] reaches the column-tile
//           count, reads the slot (through L2: slots are reused inside the
//           launch, so L1 must not serve them), counts itself in row_done[t]
//   XC      up to M consecutive overlap-save blocks of one correlation
// Scratch slots form a ring; a COL tile first waits until the transform that
// last used its slot has finished all its ROW tiles.  Every wait is on an item
// that sits earlier in the queue, so it was claimed earlier by a resident CTA
// that never waits on a later item: the waits always end.  They are still
// bounded (about one second); on timeout the CTA records an error and leaves.
#include "pcx_fft_v2.cuh"
#include "pcx_fxcorr_kernels.cuh"
#include "pcx_host.hpp"

#include <algorithm>
#include <map>
#include <vector>

namespace pcxg {
namespace rg {

constexpr int NT     = 512;
constexpr int LPK    = 3;    // pack 8 (complex64)
constexpr int MAXLG  = 32;

enum : int { K_SINGLE = 0, K_COL = 1, K_ROW = 2, K_XC = 3 };

struct item {
    int kind, lg, a, b, c;    // SINGLE: a first transform, b count; COL/ROW: a transform, b tile; XC: a request, b first block, c count
};
struct fft_req {
    const float* src;
    float*       dst;
    int          slot;        // four-step scratch slot
    int          prev;        // transform that used the slot before (-1 none)
    int          prev_rows;   // row tiles of that transform (its completion count)
};
struct xc_req {
    const float*      src;
    float*            dst;
    long long         len;
    int               step, nblk, lg;
    const cpx<float>* kspec;
};
struct tabs {
    const cpx<float>* stw[MAXLG];     // single-pass stage twiddles (lg <= 12)
    const cpx<float>* stw1[MAXLG];    // four-step: column stage twiddles (per total lg)
    const cpx<float>* stw2[MAXLG];
    const cpx<float>* thi[MAXLG];
    const cpx<float>* tlo[MAXLG];
    const cpx<float>* tb[MAXLG];
    const cpx<float>* xtw[MAXLG];     // correlator W_N table
};
struct args {
    const item*    items;
    int            nitems;
    const fft_req* req;
    const xc_req*  xreq;
    int*           col_done;
    int*           row_done;
    int            col_tiles[MAXLG];
    int            row_tiles[MAXLG];
    cpx<float>*    scratch;
    long long      slot_elems;
    unsigned*      counter;
    int*           error;
    int            conj;     // inverse: conjugate in and out
    float          scale;
    tabs           tb;
};

__device__ __forceinline__ bool wait_count(const int* p, int target) {
    if (*reinterpret_cast<const volatile int*>(p) >= target) return true;
    const unsigned long long t0 = timer_ns();
    while (true) {
        int v;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) return true;
        if (timer_ns() - t0 > 1000000000ull) return false;
        __nanosleep(128);
    }
}

template<int LOGL>
__device__ void single_items(const args& A, const item& it, cpx<float>* xch) {
    using P          = splan<LOGL>;
    constexpr int E  = P::E;
    constexpr int TT = P::TT;
    constexpr int M  = NT / TT;
    using X          = xch_blocked<P::L, M>;
    const int  tid  = threadIdx.x;
    const int  m    = tid / TT;
    const int  t    = tid - m * TT;
    const bool live = m < it.b;
    const fft_req& r = A.req[it.a + (live ? m : 0)];
    const float*   s = r.src;
    float*         d = r.dst;
    const auto*    stw = A.tb.stw[LOGL];
    cpx<float>     v[E];
    // element t + i*TT; its packed offset splits into base + constant only
    // when TT is a multiple of the pack width
    static_for<E>([&](auto ic) {
        constexpr int i  = decltype(ic)::value;
        const int     o  = pk<LPK>(t + i * TT);
        const float   re = s[o], im = s[o + 8];
        v[i]             = {re, A.conj ? -im : im};
    });
    stage_compute_tab<P, 0>(v, t, stw);
    run_stages_tab<P, X>(v, xch, m, t, stw);
    if (live) {
        const float sc = A.scale, sim = A.conj ? -A.scale : A.scale;
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const int     o = pk<LPK>(t + i * TT);
            d[o]            = v[i].re * sc;
            d[o + 8]        = v[i].im * sim;
        });
    }
}

template<int L1, int L2>
__device__ bool col_item(const args& A, const item& it, cpx<float>* xch, int* s_flag) {
    using P           = splan<L1>;
    constexpr int N2  = 1 << L2;
    constexpr int E   = P::E;
    constexpr int TT  = P::TT;
    constexpr int C   = (8192 >> L1) > 8 ? (8192 >> L1) : 8;
    static_assert(NT == C * TT, "threads");
    using X           = xch_interleaved<P::L, C>;
    const int       tid = threadIdx.x;
    const int       c   = tid % C;
    const int       t   = tid / C;
    const fft_req&  r   = A.req[it.a];
    if (tid == 0) {
        // the slot is free once the previous user finished all its row tiles
        *s_flag = r.prev < 0 || wait_count(A.row_done + r.prev, r.prev_rows);
    }
    __syncthreads();
    if (!*s_flag) return false;
    const int    c0  = it.b * C;
    const int    n2  = c0 + c;
    const float* src = r.src + pk<LPK>(t * N2 + n2);
    cpx<float>   v[E];
    static_for<E>([&](auto ic) {
        constexpr int i  = decltype(ic)::value;
        const float   re = src[2 * i * TT * N2], im = src[2 * i * TT * N2 + 8];
        v[i]            = {re, A.conj ? -im : im};
    });
    const auto* stw = A.tb.stw1[L1 + L2];
    stage_compute_tab<P, 0>(v, t, stw);
    run_stages_tab<P, X>(v, xch, c, t, stw);
    const uint32_t   e0   = (uint32_t)t * (uint32_t)n2;
    const cpx<float> base = cmul(ldg_cpx(A.tb.thi[L1 + L2] + (e0 >> L2)), ldg_cpx(A.tb.tlo[L1 + L2] + (e0 & (N2 - 1))));
    cpx<float>       bp[16];
    powers16(ldg_cpx(A.tb.tb[L1 + L2] + n2), bp);
    cpx<float>* dst = A.scratch + (long long)r.slot * A.slot_elems + (long long)t * N2 + n2;
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        cpx<float>    w = base;
        if constexpr (i > 0) w = cmul(base, bp[i]);
        const cpx<float> o = cmul(v[i], w);
        __stcg(reinterpret_cast<float2*>(dst + (long long)i * TT * N2), make_float2(o.re, o.im));
    });
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicAdd(A.col_done + it.a, 1);
    return true;
}

template<int L1, int L2>
__device__ bool row_item(const args& A, const item& it, cpx<float>* xch, int* s_flag) {
    using P           = splan<L2>;
    constexpr int N1  = 1 << L1;
    constexpr int N2  = P::L;
    constexpr int E   = P::E;
    constexpr int TT  = P::TT;
    constexpr int G8  = 8;
    constexpr int CR  = (8192 >> L2) > 8 ? (8192 >> L2) : 8;
    static_assert(NT == CR * TT, "threads");
    using X           = xch_grouped<N2, CR, G8>;
    const int      tid = threadIdx.x;
    const int      mlo = tid % G8;
    const int      t   = (tid / G8) % TT;
    const int      mhi = tid / (G8 * TT);
    const int      m   = mhi * G8 + mlo;
    const fft_req& r   = A.req[it.a];
    if (tid == 0) *s_flag = wait_count(A.col_done + it.a, A.col_tiles[L1 + L2]);
    __syncthreads();
    if (!*s_flag) return false;
    const int          k1  = it.b * CR + m;
    const cpx<float>*  src = A.scratch + (long long)r.slot * A.slot_elems + (long long)k1 * N2 + t;
    cpx<float>         v[E];
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const float2  x = __ldcg(reinterpret_cast<const float2*>(src + i * TT));
        v[i]            = {x.x, x.y};
    });
    const auto* stw = A.tb.stw2[L1 + L2];
    stage_compute_tab<P, 0>(v, t, stw);
    run_stages_tab<P, X>(v, xch, m, t, stw);
    float*      dst = r.dst + pk<LPK>(t * N1 + k1);
    const float sc = A.scale, sim = A.conj ? -A.scale : A.scale;
    static_for<E>([&](auto ic) {
        constexpr int i          = decltype(ic)::value;
        dst[2 * i * TT * N1]     = v[i].re * sc;
        dst[2 * i * TT * N1 + 8] = v[i].im * sim;
    });
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicAdd(A.row_done + it.a, 1);
    return true;
}

template<int LOGN>
__device__ void xc_items(const args& A, const item& it, cpx<float>* buf) {
    constexpr int EPT = LOGN >= 14 ? 32 : 16;
    using P           = splan<LOGN, EPT>;
    constexpr int L   = P::L;
    constexpr int E   = P::E;
    constexpr int TT  = P::TT;
    constexpr int M   = NT / TT;
    using X           = xch_blocked<L, M>;
    const xc_req& q   = A.xreq[it.a];
    const int     tid = threadIdx.x;
    const int     m   = tid / TT;
    const int     t   = tid - m * TT;
    // load M windows (blocks b .. b+count-1), zero outside the signal
    for (int e = tid; e < M * L; e += NT) {
        const int       mm  = e / L, l = e - mm * L;
        const long long pos = (long long)(it.b + mm) * q.step + l;
        cpx<float>      w   = {0.f, 0.f};
        if (mm < it.c && pos < q.len) {
            const long long o = ((pos >> 3) << 4) + (pos & 7);
            w                 = {q.src[o], q.src[o + 8]};
        }
        buf[e] = w;
    }
    __syncthreads();
    const cpx<float>* tw = A.tb.xtw[LOGN];
    cpx<float>        v[E];
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        v[i]            = buf[m * L + t + i * TT];
    });
    stage_compute<P, 0>(v, t, tw);
    run_stages<P, X>(v, buf, m, t, tw);
    static_for<E>([&](auto ic) {
        constexpr int    i = decltype(ic)::value;
        const cpx<float> k = ldg_cpx(q.kspec + t + i * TT);
        v[i]               = cmul(cpx<float>{v[i].re, -v[i].im}, k);
    });
    stage_compute<P, 0>(v, t, tw);
    run_stages<P, X>(v, buf, m, t, tw);
    if (m < it.c) {
        const long long b0 = (long long)(it.b + m) * q.step;
        static_for<E>([&](auto ic) {
            constexpr int   i  = decltype(ic)::value;
            const int       mo = t + i * TT;
            const long long e  = b0 + mo;
            if (mo < q.step && e < q.len) {
                const long long o = ((e >> 3) << 4) + (e & 7);
                q.dst[o]          = v[i].re;
                q.dst[o + 8]      = -v[i].im;
            }
        });
    }
    __syncthreads();
}

__global__ void __launch_bounds__(NT, 1) k_ragged(args A) {
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<float>*       buf = reinterpret_cast<cpx<float>*>(smem);
    __shared__ int    s_item;
    __shared__ int    s_flag;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(A.counter, 1u);
        __syncthreads();
        const int idx = s_item;
        if (idx >= A.nitems) break;
        const item it = A.items[idx];
        bool       ok = true;
        switch (it.kind * 64 + it.lg) {
        case K_SINGLE * 64 + 5: single_items<5>(A, it, buf); break;
        case K_SINGLE * 64 + 6: single_items<6>(A, it, buf); break;
        case K_SINGLE * 64 + 7: single_items<7>(A, it, buf); break;
        case K_SINGLE * 64 + 8: single_items<8>(A, it, buf); break;
        case K_SINGLE * 64 + 9: single_items<9>(A, it, buf); break;
        case K_SINGLE * 64 + 10: single_items<10>(A, it, buf); break;
        case K_SINGLE * 64 + 11: single_items<11>(A, it, buf); break;
        case K_SINGLE * 64 + 12: single_items<12>(A, it, buf); break;
        case K_COL * 64 + 13: ok = col_item<7, 6>(A, it, buf, &s_flag); break;
        case K_COL * 64 + 14: ok = col_item<7, 7>(A, it, buf, &s_flag); break;
        case K_COL * 64 + 15: ok = col_item<8, 7>(A, it, buf, &s_flag); break;
        case K_COL * 64 + 16: ok = col_item<8, 8>(A, it, buf, &s_flag); break;
        case K_COL * 64 + 17: ok = col_item<9, 8>(A, it, buf, &s_flag); break;
        case K_COL * 64 + 18: ok = col_item<9, 9>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 13: ok = row_item<7, 6>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 14: ok = row_item<7, 7>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 15: ok = row_item<8, 7>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 16: ok = row_item<8, 8>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 17: ok = row_item<9, 8>(A, it, buf, &s_flag); break;
        case K_ROW * 64 + 18: ok = row_item<9, 9>(A, it, buf, &s_flag); break;
        case K_XC * 64 + 7: xc_items<7>(A, it, buf); break;
        case K_XC * 64 + 8: xc_items<8>(A, it, buf); break;
        case K_XC * 64 + 9: xc_items<9>(A, it, buf); break;
        case K_XC * 64 + 10: xc_items<10>(A, it, buf); break;
        case K_XC * 64 + 11: xc_items<11>(A, it, buf); break;
        case K_XC * 64 + 12: xc_items<12>(A, it, buf); break;
        case K_XC * 64 + 13: xc_items<13>(A, it, buf); break;
        case K_XC * 64 + 14: xc_items<14>(A, it, buf); break;
        default: ok = false; break;
        }
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(A.error, 1);
            return;
        }
        __syncthreads();
    }
}

constexpr int SMEM = xch_blocked<16384, 1>::size * (int)sizeof(cpx<float>);    // largest user: 16384-point correlation

}    // namespace rg
}    // namespace pcxg

using namespace pcxg;

struct pcx_ragged_s {
    int                       dtype = PCX_F32;
    std::vector<void*>        allocs;
    rg::args                  A{};
    int                       grid    = 0;
    cudaGraph_t               graph   = nullptr;
    cudaGraphExec_t           gexec   = nullptr;
    size_t                    n_fft   = 0;
    size_t                    n_items = 0;
    std::vector<pcx_plan>     plans;
    void*                     ctl     = nullptr;    // counter, error, col_done[], row_done[]
    size_t                    ctl_bytes = 0;
};

namespace {

template<class V>
void* upload(pcx_ragged_s* h, const std::vector<V>& v, cudaError_t* e) {
    void* p = nullptr;
    *e      = cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(V));
    if (*e != cudaSuccess) return nullptr;
    h->allocs.push_back(p);
    if (!v.empty()) *e = cudaMemcpy(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice);
    return p;
}

int lg2(size_t n) { return n ? __builtin_ctzll(n) : -1; }

}    // namespace

extern "C" int pcx_ragged_destroy(pcx_ragged h) {
    if (!h) return PCX_OK;
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    for (void* p: h->allocs) cudaFree(p);
    for (auto p: h->plans) pcx_plan_destroy(p);
    delete h;
    return PCX_OK;
}

extern "C" int pcx_ragged_create(pcx_ragged* out, int dtype, size_t n_fft, const size_t* sizes, void* const* dst,
                                 const void* const* src, int direction, int normalize, size_t n_xc,
                                 const size_t* xc_len, const size_t* xc_k, const void* const* xc_g,
                                 const size_t* xc_nfft, void* const* xc_dst, const void* const* xc_src) {
    return pcx_guard([&]() -> int {
        if (!out) return pcx_fail(PCX_ERR_INVALID, "handle pointer is null");
        *out = nullptr;
        if (dtype != PCX_F32) return pcx_fail(PCX_ERR_UNSUPPORTED, "ragged batches are built for complex64");
        auto  h    = new pcx_ragged_s{};
        auto  fail = [&](int rc) {
            pcx_ragged_destroy(h);
            return rc;
        };
        cudaError_t e = cudaSuccess;
        // ---- requests and per-size tables
        std::vector<rg::fft_req> req(n_fft);
        std::map<int, std::vector<int>> by_lg;
        for (size_t i = 0; i < n_fft; ++i) {
            const int lg = lg2(sizes[i]);
            if (lg < 5 || lg > 18 || (sizes[i] & (sizes[i] - 1))) {
                return fail(pcx_fail(PCX_ERR_UNSUPPORTED, "ragged FFT sizes must be powers of two in 2^5..2^18"));
            }
            req[i] = {static_cast<const float*>(src[i]), static_cast<float*>(dst[i]), -1, -1, 0};
            by_lg[lg].push_back((int)i);
        }
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        h->A.conj  = direction == PCX_INVERSE;
        h->A.scale = 1.0f;
        std::map<int, pcx_plan> plan_of;
        auto get_plan = [&](int lg) -> pcx_plan {
            auto it = plan_of.find(lg);
            if (it != plan_of.end()) return it->second;
            pcx_plan p = nullptr;
            if (pcx_plan_create(&p, size_t(1) << lg, PCX_F32, PCX_ORDER_NORMAL, 2048) != PCX_OK) return nullptr;
            h->plans.push_back(p);
            plan_of[lg] = p;
            return p;
        };
        for (auto& [lg, idx]: by_lg) {
            pcx_plan p = get_plan(lg);
            if (!p) return fail(PCX_ERR_CUDA);
            if (lg <= 12) {
                h->A.tb.stw[lg] = static_cast<const cpx<float>*>(p->stwL);
            } else {
                h->A.tb.stw1[lg] = static_cast<const cpx<float>*>(p->stw1);
                h->A.tb.stw2[lg] = static_cast<const cpx<float>*>(p->stw2);
                h->A.tb.thi[lg]  = static_cast<const cpx<float>*>(p->tw_hi);
                h->A.tb.tlo[lg]  = static_cast<const cpx<float>*>(p->tw_lo);
                h->A.tb.tb[lg]   = static_cast<const cpx<float>*>(p->tw_b);
                const int l1 = (lg + 1) / 2, l2 = lg / 2;
                const int c  = std::max(8, 8192 >> l1), cr = std::max(8, 8192 >> l2);
                h->A.col_tiles[lg] = (1 << l2) / c;
                h->A.row_tiles[lg] = (1 << l1) / cr;
            }
            if (normalize && direction == PCX_INVERSE) {
                // one scale per launch: every transform of an inverse batch must share N
                if (by_lg.size() > 1) {
                    return fail(pcx_fail(PCX_ERR_UNSUPPORTED, "a normalised inverse ragged batch needs one size"));
                }
                h->A.scale = 1.0f / float(size_t(1) << lg);
            }
        }
        // correlation requests
        std::vector<rg::xc_req> xreq(n_xc);
        for (size_t j = 0; j < n_xc; ++j) {
            const int lg = lg2(xc_nfft[j]);
            if (lg < 7 || lg > 14 || (xc_nfft[j] & (xc_nfft[j] - 1)) || xc_k[j] == 0 || xc_k[j] + 7 > xc_nfft[j]) {
                return fail(pcx_fail(PCX_ERR_UNSUPPORTED, "ragged correlation: N_fft must be 2^7..2^14 and K <= N_fft-7"));
            }
            const size_t step = (xc_nfft[j] - (xc_k[j] - 1)) / 8 * 8;
            void*        ks   = nullptr;
            if ((e = cudaMalloc(&ks, xc_nfft[j] * 8)) != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
            h->allocs.push_back(ks);
            pcx_plan p = get_plan(lg);
            if (!p) return fail(PCX_ERR_CUDA);
            int rc = pcx_fft_run(p, ks, xc_g[j], xc_k[j], 1, 8, PCX_FORWARD, 0, 1, 2 * xc_nfft[j], 2 * xc_nfft[j], nullptr,
                                 0, 0, 1.0 / (double)xc_nfft[j]);
            if (rc) return fail(rc);
            if (!h->A.tb.xtw[lg]) {
                void* tw = nullptr;
                if ((e = cudaMalloc(&tw, xc_nfft[j] * 8)) != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
                h->allocs.push_back(tw);
                if ((e = pcx_gen_twiddles(tw, (int)xc_nfft[j], lg, 1, false, 0)) != cudaSuccess) {
                    return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
                }
                h->A.tb.xtw[lg] = static_cast<const cpx<float>*>(tw);
            }
            xreq[j] = {static_cast<const float*>(xc_src[j]), static_cast<float*>(xc_dst[j]), (long long)xc_len[j],
                       (int)step, (int)((xc_len[j] + step - 1) / step), lg, static_cast<const cpx<float>*>(ks)};
        }
        // ---- work queue
        std::vector<rg::item> items;
        std::vector<rg::item> fill;    // single-pass items and correlation blocks, spread between four-step work
        for (auto& [lg, idx]: by_lg) {
            if (lg > 12) continue;
            const int M = rg::NT / std::max(1, (1 << lg) / 16);    // rows per item: one thread row per 16 points
            for (size_t q = 0; q < idx.size(); q += M) {
                // requests of one size are consecutive in idx
                const int cnt = (int)std::min<size_t>(M, idx.size() - q);
                fill.push_back({rg::K_SINGLE, lg, idx[q], cnt, 0});
            }
        }
        for (size_t j = 0; j < n_xc; ++j) {
            const int lg = xreq[j].lg;
            const int tt = (1 << lg) / (lg >= 14 ? 32 : 16);
            const int M  = std::max(1, rg::NT / tt);
            for (int b = 0; b < xreq[j].nblk; b += M) fill.push_back({rg::K_XC, lg, (int)j, b, std::min(M, xreq[j].nblk - b)});
        }
        std::vector<int> four;
        for (auto& [lg, idx]: by_lg)
            if (lg > 12) four.insert(four.end(), idx.begin(), idx.end());
        // single-pass requests must be grouped by size with consecutive global indices
        {
            std::vector<rg::fft_req> sorted;
            std::vector<int>         order;
            for (auto& [lg, idx]: by_lg) order.insert(order.end(), idx.begin(), idx.end());
            std::vector<int> newpos(n_fft);
            for (size_t q = 0; q < order.size(); ++q) newpos[order[q]] = (int)q;
            for (int o: order) sorted.push_back(req[o]);
            req.swap(sorted);
            for (auto& it: fill)
                if (it.kind == rg::K_SINGLE) it.a = newpos[it.a];
            for (auto& f: four) f = newpos[f];
        }
        const int LAG = 2, NSLOT = 8;
        size_t    slot_elems = 0;
        for (auto& [lg, idx]: by_lg)
            if (lg > 12) slot_elems = std::max<size_t>(slot_elems, size_t(1) << lg);
        // four-step transforms in queue order with their sizes
        std::vector<int> four_lg;
        for (auto& [lg, idx]: by_lg)
            if (lg > 12) four_lg.insert(four_lg.end(), idx.size(), lg);
        for (size_t q = 0; q < four.size(); ++q) {
            req[four[q]].slot = (int)(q % NSLOT);
            req[four[q]].prev = q >= (size_t)NSLOT ? four[q - NSLOT] : -1;
            req[four[q]].prev_rows = q >= (size_t)NSLOT ? h->A.row_tiles[four_lg[q - NSLOT]] : 0;
        }
        const size_t nfill = fill.size(), nfour = four.size();
        size_t       fi    = 0;
        auto         push_fill = [&](size_t upto) {
            while (fi < std::min(upto, nfill)) items.push_back(fill[fi++]);
        };
        // column tiles of transform q, row tiles of transform q - LAG, then a
        // proportional share of the single-pass / correlation items
        for (size_t q = 0; q < nfour + LAG; ++q) {
            if (q < nfour) {
                const int lg = four_lg[q];
                for (int tile = 0; tile < h->A.col_tiles[lg]; ++tile) items.push_back({rg::K_COL, lg, four[q], tile, 0});
            }
            if (q >= (size_t)LAG && q - LAG < nfour) {
                const size_t p  = q - LAG;
                const int    lg = four_lg[p];
                for (int tile = 0; tile < h->A.row_tiles[lg]; ++tile) items.push_back({rg::K_ROW, lg, four[p], tile, 0});
            }
            push_fill(nfour ? (q + 1) * nfill / (nfour + LAG) : nfill);
        }
        push_fill(nfill);
        h->n_fft   = n_fft;
        h->n_items = items.size();
        // ---- device state
        h->A.items = static_cast<const rg::item*>(upload(h, items, &e));
        if (e == cudaSuccess) h->A.req = static_cast<const rg::fft_req*>(upload(h, req, &e));
        if (e == cudaSuccess) h->A.xreq = static_cast<const rg::xc_req*>(upload(h, xreq, &e));
        if (e != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        h->A.nitems     = (int)items.size();
        h->A.slot_elems = (long long)slot_elems;
        if (slot_elems) {
            void* s = nullptr;
            if ((e = cudaMalloc(&s, NSLOT * slot_elems * 8)) != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
            h->allocs.push_back(s);
            h->A.scratch = static_cast<cpx<float>*>(s);
        }
        h->ctl_bytes = (2 + 2 * std::max<size_t>(n_fft, 1)) * sizeof(int);
        if ((e = cudaMalloc(&h->ctl, h->ctl_bytes)) != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        h->allocs.push_back(h->ctl);
        int* c        = static_cast<int*>(h->ctl);
        h->A.counter  = reinterpret_cast<unsigned*>(c);
        h->A.error    = c + 1;
        h->A.col_done = c + 2;
        h->A.row_done = c + 2 + std::max<size_t>(n_fft, 1);
        if ((e = cudaFuncSetAttribute(rg::k_ragged, cudaFuncAttributeMaxDynamicSharedMemorySize, rg::SMEM)) != cudaSuccess) {
            return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        }
        h->grid = sms;
        if ((e = cudaMemset(h->ctl, 0, h->ctl_bytes)) != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        // ---- capture: reset counters, one persistent launch
        cudaStream_t cs = nullptr;
        if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) {
            return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(e)));
        }
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->ctl, 0, h->ctl_bytes, cs);
        if (e == cudaSuccess) {
            rg::k_ragged<<<h->grid, rg::NT, rg::SMEM, cs>>>(h->A);
            e = cudaGetLastError();
        }
        cudaError_t e2 = cudaStreamEndCapture(cs, &h->graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&h->gexec, h->graph, 0);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return fail(pcx_fail(PCX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)));
        *out = h;
        return PCX_OK;
    });
}

extern "C" int pcx_ragged_exec(pcx_ragged h, void* stream) {
    return pcx_guard([&]() -> int {
        if (!h) return pcx_fail(PCX_ERR_INVALID, "handle is null");
        PCX_CUDA_TRY(cudaGraphLaunch(h->gexec, static_cast<cudaStream_t>(stream)));
        return PCX_OK;
    });
}

extern "C" int pcx_ragged_status(pcx_ragged h) {
    return pcx_guard([&]() -> int {
        if (!h) return pcx_fail(PCX_ERR_INVALID, "handle is null");
        int err = 0;
        PCX_CUDA_TRY(cudaMemcpy(&err, h->A.error, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return pcx_fail(PCX_ERR_TIMEOUT, "a ragged work item gave up waiting for its dependency");
        return PCX_OK;
    });
}

extern "C" size_t pcx_ragged_items(pcx_ragged h) { return h ? h->n_items : 0; }
