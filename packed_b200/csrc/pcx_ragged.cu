// Ragged persistent batch: FFTs of uneven power-of-two sizes and overlap-save
// correlations, all in ONE persistent launch fed by a device work queue and
// replayed from a CUDA graph.
//
// Work items (built once on the host, each with its slot, destination, tensor
// map and dependency resolved, claimed in queue order from a device counter):
//   SINGLE  M whole transforms of one size N <= 4096 (M rows of 16 points per
//           thread fill the block)
//   COL     one column tile of a four-step transform (N = 2^13..2^18, split
//           split_l1): TMA copy of the tile (one tensor map per size when the
//           transforms lie at a uniform stride, else one per transform),
//           column FFTs, four-step twiddle, written to the transform's
//           scratch slot, then counted in col_done[t]
//   ROW     one row tile: waits until col_done[t] reaches the column-tile
//           count, bulk-copies the slot rows, row FFTs, natural-order output,
//           counted in row_done[t] once its rows have landed
//   XR      up to M consecutive overlap-save blocks of one correlation with
//           N_fft <= 2048: the producer bulk-copies the M packed windows into
//           the stage; forward FFT, times conj(K), inverse, in the stage.
//           With N_fft = 4096 (two windows per item) and 8192 (one) the
//           windows' rows are copied and each window runs as the in-CTA
//           four-step with in-place exchanges inside the window (one stage)
//   XC      one overlap-save window of a correlation with N_fft = 16384 on
//           the whole ring: the producer bulk-copies the window's rows, the
//           compute warps run the in-CTA four-step of the C3 correlator
// Each block has NT compute threads and, as the one-launch four-step kernel
// does, a producer warp and a publisher warp: the producer claims the next
// item, waits for its dependency (a scratch slot freed by an earlier
// transform's row tiles, or a transform's column tiles) and issues its
// copies into a three-stage shared-memory ring, so two items are in flight
// while one is computed; the publisher counts completions as soon as they
// happen and never waits on another block.  The compute warps run one loop
// per item kind and size (its own compile-time geometry and register
// allocation); the exchanges of the sub-transforms run in place in the item's
// stage.  16384-point correlation items (last in the queue) use the whole
// ring, so the producer drains the ring around them.  Every wait is on an
// item earlier in the queue, claimed by a resident block whose publisher
// never waits on a later item: the waits always end.  They are still bounded
// (about one second); on timeout the block records an error and leaves.
#include "pcx_fft_v2.cuh"
#include "pcx_fourstep.cuh"
#include "pcx_fxcorr2d.cuh"
#include "pcx_fxcorr_kernels.cuh"
#include "pcx_host.hpp"
#include "pcx_v2_launch.cuh"

#include <algorithm>
#include <map>
#include <string>
#include <vector>

namespace pcxg {
namespace rg {

constexpr int NT    = 512;    // compute threads; then the producer warp, then the publisher warp
constexpr int NW    = NT / 32;
constexpr int ST    = 3;      // ring stages
constexpr int LPK   = 3;      // pack 8 (complex64)
constexpr int MAXLG = 32;
// A stage holds a 64 KB tile (plus row padding) or the item's in-place
// exchange buffer (one padding slot per 16 elements): 68 KB at every size.
constexpr int STAGE = 69632;
constexpr int RING  = ST * STAGE;
constexpr int XRW   = 12;    // correlations of 2^XRW..2^13 points: in-place in-CTA four-step windows
// Behind the ring: the full stage tables of the 64..1024-point sub-transforms
// (the four-step passes of 2^13..2^18, the correlations of 128..1024 points
// and the sub-transforms of the 4096..16384-point correlation windows),
// copied from global memory once per launch.  The 1024-point table
// also serves 512 points (the same stages, a radix-4 last stage read at every
// other entry), so four tables are kept: 2^6, 2^7, 2^8 and 2^10.
constexpr int SUB_LO = 6, SUB_HI = 10;
template<int L>
using sub_plan = splan<(L == 9 ? 10 : L)>;    // the plan whose table serves 2^L points
template<int L>
__host__ __device__ constexpr bool sub_kept() {
    return L >= SUB_LO && L <= SUB_HI && L != 9;
}
template<int L>
__host__ __device__ constexpr int sub_off() {    // entries before the kept table of 2^L points
    int o = 0;
    if constexpr (L > SUB_LO) {
        o = sub_off<L - 1>();
        if constexpr (sub_kept<L - 1>()) o += fs_full_tw_size<splan<L - 1>>();
    }
    return o;
}
constexpr int SUBTAB = sub_off<SUB_HI + 1>() * 8;
constexpr int SMEM   = RING + SUBTAB;
static_assert(SUBTAB % 16 == 0 && SMEM <= 232448, "tables beside the ring");

extern __shared__ __align__(128) unsigned char rg_smem[];
__shared__ uint64_t s_full[ST];       // the item's copies landed (or, at the end, the producer arrived)
__shared__ uint64_t s_empty[ST];      // compute warps done with the stage, publisher past its item
__shared__ uint64_t s_slotok[ST];     // column tile: its scratch slot may be written
__shared__ uint64_t s_written[ST];    // column tile: compute warps wrote the slot
__shared__ int      s_item[ST];       // item index in the stage (-1: the queue is exhausted)

// Rows of a correlation window (N1 rows of N2 samples) that lie wholly inside
// the signal, given the samples left from the window's start.
template<int N1, int N2>
__host__ __device__ __forceinline__ int xc2_rows_inside(long long left) {
    const long long r = left > 0 ? left / N2 : 0;
    return (int)(r < N1 ? r : N1);
}

// The table (of plan sub_plan<L>) that serves 2^L points.
template<int L>
__device__ __forceinline__ const cpx<float>* sub_tab() {
    static_assert(L >= SUB_LO && L <= SUB_HI, "table kept in shared memory");
    static_assert(full_tab_serves<splan<L>, sub_plan<L>>(), "the kept table serves this size");
    return reinterpret_cast<const cpx<float>*>(rg_smem + RING) + sub_off<(L == 9 ? 10 : L)>();
}

enum : int { K_SINGLE = 0, K_COL = 1, K_ROW = 2, K_XC = 3, K_XR = 4 };

struct item {
    int kind, lg, a, b, c;    // SINGLE: a first transform, b count; COL/ROW: a transform, b tile; XC: a request, b first block, c count
    // resolved on the host, so that claiming an item is one read:
    int         tmap;         // COL: the transform's column-tile tensor map
    int         tz;           // COL: the transform's index in that map (0 for a map of its own)
    int         prev;         // COL: the transform that used the slot before (-1 none)
    int         prev_rows;    // COL: that transform's row tiles
    const void* p0;           // COL: the scratch slot; ROW: destination; SINGLE: stage tables
    const void* p1;           // COL: W_N^(i*N2); ROW: the scratch slot
    const void* p2;           // COL: W_N^i
    const void* p3;           // COL: W_{16*N2}^i
};
struct fft_req {
    const float* src;
    float*       dst;
    int          slot;        // four-step scratch slot (in the size's own ring)
    int          prev;        // transform that used the slot before (-1 none)
    int          prev_rows;   // row tiles of that transform (its completion count)
    int          tmap;        // its column-tile tensor map
    int          tz;          // its index in that map (four-step sizes)
};
struct xc_req {
    const float*      src;
    float*            dst;
    long long         len;
    int               step, nblk, lg;
    const cpx<float>* kspec;
};
struct tabs {
    const cpx<float>* stw[MAXLG];     // single pass: stage factor tables (lg <= 12)
    const cpx<float>* thi[MAXLG];     // W_N^(i*N2), i < N1
    const cpx<float>* tlo[MAXLG];     // W_N^i, i < N2
    const cpx<float>* tb[MAXLG];      // W_{16*N2}^i, i < N2
    cpx<float>*       scratch[MAXLG]; // the size's ring of scratch slots
    const cpx<float>* xft[MAXLG];     // correlator full stage tables
    const cpx<float>* x2tw[MAXLG];    // in-CTA four-step correlator: W_N^e (e < N/16), W_N^(TT1*n2), W_N^(TT2*k1)
    const void*       sub;            // SUBTAB bytes: full tables of 2^6, 2^7, 2^8, 2^10 points, in order
};
struct args {
    const item*        items;
    int                nitems;
    const fft_req*     req;
    const xc_req*      xreq;
    const CUtensorMap* tmaps;
    int*               col_done;
    int*               row_done;
    int                col_tiles[MAXLG];
    int                row_tiles[MAXLG];
    unsigned*          counter;
    int*               error;
    int                conj;     // inverse: conjugate in and out
    float              scale;
    tabs               tb;
};

// What the compute warps need of the item in each stage, filled by the
// producer while earlier items are computed, so that no chain of dependent
// global loads opens an item.
struct stage_meta {
    item   it;
    xc_req xq;    // XR, XC: the correlation request
};
__shared__ stage_meta s_meta[ST];
__shared__ int        s_conj;     // inverse: conjugate in and out
__shared__ float      s_scale;

// The four-step split N = 2^l1 * 2^(lg - l1) of a ragged transform of 2^lg
// points (host and device use this one table).
__host__ __device__ constexpr int split_l1(int lg) {
    return lg == 13 ? 6 : lg == 14 ? 6 : lg == 15 ? 6 : lg == 16 ? 6 : lg == 17 ? 7 : lg == 18 ? 8 : (lg + 1) / 2;
}

// Geometry of the four-step sizes: N = N1*N2, tiles of 8192 elements over NT
// threads of 16 points.
template<int L1, int L2>
struct fsg {
    static constexpr int N1 = 1 << L1, N2 = 1 << L2;
    using P1                = splan<L1>;
    using P2                = splan<L2>;
    static constexpr int C   = NT / P1::TT;    // columns per column tile
    static constexpr int CR  = NT / P2::TT;    // rows per row tile
    static constexpr int SEG = 2 * C;          // reals per tile row (packed, pack 8)
    static constexpr int RSI = N2 + 2;         // padded row of a row tile (complex)
    static constexpr int BOXY = N1 < 256 ? N1 : 256;
    using X1 = xch_interleaved<N1, C>;
    using X2 = xch_grouped<N2, CR, 8>;
    static_assert(C >= 8 && CR >= 8 && CR % 8 == 0, "tiles span whole 32-byte sectors");
    static_assert(N1 * SEG * 4 <= STAGE && CR * RSI * 8 <= STAGE, "tile fits a stage");
    static_assert(X1::size * 8 <= STAGE && X2::size * 8 <= STAGE, "exchange fits a stage");
    static_assert(2 * C <= 256, "TMA box width");
};
// Whole transforms of N = 2^LOGL <= 4096: M rows of RS reals.
template<int LOGL>
struct sgg {
    using P                 = splan<LOGL>;
    static constexpr int L  = P::L;
    static constexpr int TT = P::TT;
    static constexpr int M  = NT / TT;
    static constexpr int RS = 2 * L + single3_pad<TT>();
    using X                 = xch_blocked<L, M>;
    static_assert(M * RS * 4 <= STAGE && X::size * 8 <= STAGE, "rows and exchange fit a stage");
};

// Correlation blocks of N = 2^LOGN <= 8192 on the ring: M windows of WS reals.
template<int LOGN>
struct xrg {
    using P                 = splan<LOGN>;
    static constexpr int L  = P::L;
    static constexpr int TT = P::TT;
    static constexpr int M  = NT / TT;
    static constexpr int WS = 2 * L + single3_pad<TT>();
    using X                 = xch_blocked<L, M>;
    static_assert(M * WS * 4 <= STAGE && X::size * 8 <= STAGE, "windows and exchange fit a stage");
};

// Correlation windows of N = N1 x N2 = 2^LOGN points (4096, 8192) as the
// in-CTA four-step with in-place exchanges: W = 8192 / N windows per item,
// stacked as W*N1 rows of RS complex in one stage.  RS keeps a half-warp's
// column groups and row groups on distinct banks (2 mod 16 for 8-thread
// columns, 4 mod 16 for 4-thread ones).
template<int LOGN>
struct xrw_cfg {
    static constexpr int LOGN1 = (LOGN + 1) / 2;
    static constexpr int LOGN2 = LOGN / 2;
    static constexpr int N1    = 1 << LOGN1;
    static constexpr int N2    = 1 << LOGN2;
    static constexpr int N     = N1 * N2;
    using P1                   = splan<LOGN1>;
    using P2                   = splan<LOGN2>;
    static constexpr int TT1   = P1::TT;
    static constexpr int TT2   = P2::TT;
    static constexpr int W     = 8192 / N;
    static constexpr int RS    = N2 + (TT1 == 8 ? 2 : 4);
    static constexpr int NB    = N / 16;    // W_N^e, e < N/16 (= TT1*N2 = TT2*N1)
    static constexpr int WIN   = W * N1 * RS * 8;
    static_assert(P1::E == 16 && P2::E == 16 && TT1 <= 8 && TT2 <= 4, "groups inside a warp");
    static_assert(W * N2 * TT1 == NT && W * N1 * TT2 == NT, "one column and one row per group");
    static_assert(TT1 * N2 == NB && TT2 * N1 == NB, "twiddle split");
};

// ---------------------------------------------------------------- compute
// Each returns false when a give-up vote made every compute thread leave.
// They are inlined into the run loops below (one per kind and size).
template<int LOGL>
__device__ __forceinline__ bool single_items(const args& A, const stage_meta& mt, unsigned char* buf, bool bad, int tid,
                                          uint64_t* empty_bar) {
    const item&   it = mt.it;
    using G          = sgg<LOGL>;
    using P          = typename G::P;
    constexpr int E  = P::E;
    constexpr int TT = G::TT;
    constexpr int SW = TT >= 32 ? 16 : 0;
    const int     m  = tid / TT;
    const int     t  = tid - m * TT;
    const float*  in = reinterpret_cast<const float*>(buf);
    const auto*   stw  = static_cast<const cpx<float>*>(mt.it.p0);
    const bool    conj = s_conj != 0;
    cpx<float>    v[E];
    static_for<E>([&](auto ic) {
        constexpr int    i = decltype(ic)::value;
        const cpx<float> x = lds_swapped<float, SW>(in, m * G::RS + pk<LPK>(t + i * TT), 8);
        v[i]               = {x.re, conj ? -x.im : x.im};
    });
    stage_compute_tab<P, 0>(v, t, stw);
    // the exchanges run in place in the stage: the first (block-wide) barrier
    // also votes on `bad`
    if (bar1_any<NT>(bad)) return false;
    run_stages_tab<P, typename G::X, false, NT>(v, reinterpret_cast<cpx<float>*>(buf), m, t, stw);
    fence_proxy_async_smem();    // the stage is read: it may be refilled
    __syncwarp();
    if (tid % 32 == 0) mbar_arrive(empty_bar);
    if (m < it.b) {
        // element t + i*TT; its packed offset splits into a base and a
        // constant only when TT is a multiple of the pack width
        float*      d  = A.req[it.a + m].dst;
        const float sc = s_scale, sim = conj ? -sc : sc;
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const int     o = pk<LPK>(t + i * TT);
            d[o]            = v[i].re * sc;
            d[o + 8]        = v[i].im * sim;
        });
    }
    return true;
}

// The stage is free once this returns true (the caller releases it); the
// scratch stores wait for `slot_ready`.
template<int L1, int L2, class SlotWait>
__device__ __forceinline__ bool col_item(const stage_meta& mt, unsigned char* buf, bool& bad, int tid, SlotWait&& slot_ready,
                                         uint64_t* empty_bar) {
    using F          = fsg<L1, L2>;
    using P1         = typename F::P1;
    constexpr int E  = P1::E;
    constexpr int TT = P1::TT;
    constexpr int C  = F::C;
    constexpr int N2 = F::N2;
    const int     c  = tid % C;
    const int     t  = tid / C;
    const int     n2 = mt.it.b * C + c;
    // four-step twiddle inputs, used after the stages
    const uint32_t   e0 = (uint32_t)t * (uint32_t)n2;
    const cpx<float> th = ldg_cpx(static_cast<const cpx<float>*>(mt.it.p1) + (e0 >> L2));
    const cpx<float> tl = ldg_cpx(static_cast<const cpx<float>*>(mt.it.p2) + (e0 & (N2 - 1)));
    const cpx<float> tu = ldg_cpx(static_cast<const cpx<float>*>(mt.it.p3) + n2);
    const float*     in   = reinterpret_cast<const float*>(buf);
    const bool       conj = s_conj != 0;
    cpx<float>       v[E];
    static_for<E>([&](auto ic) {
        constexpr int    i = decltype(ic)::value;
        const cpx<float> x = lds_swapped<float, 16>(in, (t + i * TT) * F::SEG + pk<LPK>(c), 8);
        v[i]               = {x.re, conj ? -x.im : x.im};
    });
    const auto* fst = sub_tab<L1>();
    stage_compute_tab<P1, 0>(v, t, fst);
    if (run_stages_full<P1, typename F::X1, true, NT, sub_plan<L1>>(v, reinterpret_cast<cpx<float>*>(buf), c, t, fst,
                                                                   bad)) {
        return false;
    }
    // the stage is read: let the producer refill it while the tile is stored
    fence_proxy_async_smem();
    __syncwarp();
    if (tid % 32 == 0) mbar_arrive(empty_bar);
    if (!slot_ready()) bad = true;
    if (!bad) {
        cpx<float>* dst = const_cast<cpx<float>*>(static_cast<const cpx<float>*>(mt.it.p0)) + (long long)t * N2 + n2;
        apply_fourstep_tw(v, cmul(th, tl), tu, [&](auto ic, cpx<float> o) {
            constexpr int i             = decltype(ic)::value;
            dst[(long long)i * TT * N2] = o;
        });
    }
    return true;
}

template<int L1, int L2>
__device__ __forceinline__ bool row_item(const stage_meta& mt, unsigned char* buf, bool bad, int tid, uint64_t* empty_bar) {
    using F          = fsg<L1, L2>;
    using P2         = typename F::P2;
    constexpr int E  = P2::E;
    constexpr int TT = P2::TT;
    constexpr int N1 = F::N1;
    const int     mlo = tid % 8;
    const int     t   = (tid / 8) % TT;
    const int     mhi = tid / (8 * TT);
    const int     m   = mhi * 8 + mlo;
    const int     k1  = mt.it.b * F::CR + m;
    const cpx<float>* in = reinterpret_cast<const cpx<float>*>(buf) + m * F::RSI + t;
    cpx<float>        v[E];
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        v[i]            = in[i * TT];
    });
    const auto* fst = sub_tab<L2>();
    stage_compute_tab<P2, 0>(v, t, fst);
    if (run_stages_full<P2, typename F::X2, true, NT, sub_plan<L2>>(v, reinterpret_cast<cpx<float>*>(buf), m, t, fst,
                                                                   bad)) {
        return false;
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (tid % 32 == 0) mbar_arrive(empty_bar);
    float*      dst = const_cast<float*>(static_cast<const float*>(mt.it.p0)) + pk<LPK>(t * N1 + k1);
    const float sc = s_scale, sim = s_conj ? -sc : sc;
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        __stcs(dst + 2 * i * TT * N1, v[i].re * sc);
        __stcs(dst + 2 * i * TT * N1 + 8, v[i].im * sim);
    });
    return true;
}

// One overlap-save window of a 2^LOGN-point correlation (N_fft = 16384) on the
// whole ring: the in-CTA four-step of the C3 correlator, N = N1 x N2 with the
// window in shared memory as N1 rows of N2 samples.  The producer copied the
// rows that lie inside the signal (packed); the compute threads fill the
// others, convert to interleaved complex in place, and run
//   1. columns: N1-point FFTs, times W_N^(k1*n2);
//   2. rows: N2-point FFTs, times the request's spectrum (stored in the same
//      (k1, k2) order), inverse N2-point FFTs (as FFTs of the conjugate),
//      times W_N^(k1*n2) again;
//   3. columns: N1-point FFTs give conj(y), stored straight to the output.
// Block barriers are named barrier 1 over the NT compute threads; each sub-FFT
// belongs to TT threads of one warp and exchanges with warp barriers only.
template<int LOGN>
__device__ __noinline__ void xc2_window(const args& A, const stage_meta& mt, int tid, uint64_t* empty_bar) {
    using F            = xc2_cfg<LOGN>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int TT1  = F::TT1;
    constexpr int TT2  = F::TT2;
    constexpr int RS   = F::RS;
    constexpr int E    = 16;
    static_assert(F::NT == NT, "one compute thread per correlator thread");
    static_assert(F::WIN + F::XB <= RING, "window and exchange rows fit the ring");
    cpx<float>*       win  = reinterpret_cast<cpx<float>*>(rg_smem);
    cpx<float>*       xch  = reinterpret_cast<cpx<float>*>(rg_smem + F::WIN);
    const cpx<float>* tw1  = sub_tab<F::LOGN1>();
    const cpx<float>* tw2  = sub_tab<F::LOGN2>();
    const cpx<float>* fwb  = A.tb.x2tw[LOGN];
    const cpx<float>* fwu1 = fwb + F::NB;
    const cpx<float>* fwu2 = fwu1 + N2;
    const xc_req&     q    = mt.xq;
    const cpx<float>* kp   = q.kspec;    // K[k1 + N1*k2] / N at [k1*N2 + k2]
    const long long   b0   = (long long)mt.it.b * q.step;
    const int         rin  = xc2_rows_inside<N1, N2>(q.len - b0);
    // rows past the copied ones: packed samples, zeros past the signal
    for (int e = tid; e < (N1 - rin) * N2; e += NT) {
        const int       r   = rin + e / N2, c = e % N2;
        const long long pos = b0 + (long long)r * N2 + c;
        float           re = 0.f, im = 0.f;
        if (pos < q.len) {
            const long long o = ((pos >> 3) << 4) + (pos & 7);
            re                = q.src[o];
            im                = q.src[o + 8];
        }
        float* row                         = reinterpret_cast<float*>(win + r * RS);
        row[((c >> 3) << 4) + (c & 7)]     = re;
        row[((c >> 3) << 4) + (c & 7) + 8] = im;
    }
    xch_sync<NT>();
    // packed -> interleaved, in place, one 64-byte pack per thread and step
    // (consecutive threads take consecutive rows: distinct bank groups)
    for (int e = tid; e < N1 * N2 / 8; e += NT) {
        const int    r  = e % N1, p = e / N1;
        float4*      w  = reinterpret_cast<float4*>(win + r * RS + p * 8);
        const float4 r0 = w[0], r1 = w[1], i0 = w[2], i1 = w[3];
        w[0]            = make_float4(r0.x, i0.x, r0.y, i0.y);
        w[1]            = make_float4(r0.z, i0.z, r0.w, i0.w);
        w[2]            = make_float4(r1.x, i1.x, r1.y, i1.y);
        w[3]            = make_float4(r1.z, i1.z, r1.w, i1.w);
    }
    xch_sync<NT>();
    // ---- step 1: columns, forward, times W_N^(k1*n2)
    {
        const int g = tid / TT1, t = tid % TT1;
        for (int rd = 0; rd < F::R1; ++rd) {
            const int  n2 = rd * F::G1 + g;
            cpx<float> v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                v[i]            = win[(t + i * TT1) * RS + n2];
            });
            stage_compute_tab<P1, 0>(v, t, tw1);
            run_stages_full<P1, typename F::X1, true, -1>(v, xch, g, t, tw1);
            apply_fourstep_tw(v, ldg_cpx(fwb + t * n2), ldg_cpx(fwu1 + n2), [&](auto ic, cpx<float> o) {
                constexpr int i              = decltype(ic)::value;
                win[(t + i * TT1) * RS + n2] = o;
            });
        }
    }
    xch_sync<NT>();
    // ---- step 2: rows; spectrum times the kernel's; inverse rows
    {
        constexpr int S  = TT2 / 2;    // the U groups of a half-warp take rows S apart:
        constexpr int U  = 16 / TT2;   // their window rows fall in disjoint banks (RS = 2 mod 16)
        const int     g  = tid / TT2, t = tid % TT2;
        const int     bb = g / U, u = g % U;
        const int     r0 = (bb / S) * 8 + (bb % S) + u * S;
        for (int rd = 0; rd < F::R2; ++rd) {
            const int  k1 = rd * F::G2 + r0;
            cpx<float> v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                v[i]            = win[k1 * RS + t + i * TT2];
            });
            stage_compute_tab<P2, 0>(v, t, tw2);
            run_stages_full<P2, typename F::X2, true, -1>(v, xch, g, t, tw2);
            // v[i] = X[k1 + N1*k2], k2 = t + i*TT2: conj(X * conj(K)) = conj(X) * K
            static_for<E>([&](auto ic) {
                constexpr int    i = decltype(ic)::value;
                const cpx<float> k = ldg_cpx(kp + k1 * N2 + t + i * TT2);
                v[i]               = cmul(cpx<float>{v[i].re, -v[i].im}, k);
            });
            stage_compute_tab<P2, 0>(v, t, tw2);
            run_stages_full<P2, typename F::X2, true, -1>(v, xch, g, t, tw2);
            apply_fourstep_tw(v, ldg_cpx(fwb + k1 * t), ldg_cpx(fwu2 + k1), [&](auto ic, cpx<float> o) {
                constexpr int i            = decltype(ic)::value;
                win[k1 * RS + t + i * TT2] = o;
            });
        }
    }
    xch_sync<NT>();
    // ---- step 3: columns again; outputs y = conj(.) for window positions
    // n < step inside the signal (the window starts on a whole pack)
    {
        const int g  = tid / TT1, t = tid % TT1;
        const int hi = (int)min((long long)q.step, q.len - b0);
        float*    d  = q.dst + 2 * b0;
        for (int rd = 0; rd < F::R1; ++rd) {
            const int  n2 = rd * F::G1 + g;
            cpx<float> v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                v[i]            = win[(t + i * TT1) * RS + n2];
            });
            if (rd == F::R1 - 1) {
                // the window is read: the next window's rows may land while
                // this one finishes (its exchanges use the rows behind it)
                fence_proxy_async_smem();
                __syncwarp();
                if (tid % 32 == 0) mbar_arrive(empty_bar);
            }
            stage_compute_tab<P1, 0>(v, t, tw1);
            run_stages_full<P1, typename F::X1, true, -1>(v, xch, g, t, tw1);
            float* drow = d + 2 * t * N2 + ((n2 >> 3) << 4) + (n2 & 7);
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                if ((t + i * TT1) * N2 + n2 < hi) {
                    __stcs(drow + 2 * i * TT1 * N2, v[i].re);
                    __stcs(drow + 2 * i * TT1 * N2 + 8, -v[i].im);
                }
            });
        }
    }
}

// In-place exchange layouts inside a correlation window of rows of RS complex
// (RS = 2 mod 16): a sub-FFT exchanges through its own column (or row) of the
// window, logical slot l at position l ^ ((l / 16) & SW) -- a permutation
// inside each run of 16 slots.  A group of SW + 1 threads writes slots 16t + j
// and reads slots t + (SW + 1) i; the XOR keeps those on distinct banks (for
// the columns, position p of column m sits at bank 4p + 2m mod 32).
template<int RS, int SW>
struct xch_in_column {    // m: the column
    static_assert(SW < 16, "permutation inside runs of 16");
    __device__ static __forceinline__ int idx(int m, int l) { return (l ^ ((l >> 4) & SW)) * RS + m; }
};
template<int RS, int SW>
struct xch_in_row {       // m: the row
    static_assert(SW < 16, "permutation inside runs of 16");
    __device__ static __forceinline__ int idx(int m, int l) { return m * RS + (l ^ ((l >> 4) & SW)); }
};

// Overlap-save windows of a 4096- or 8192-point correlation in one ring stage
// (W = 8192 / N windows of the item, stacked): the in-CTA four-step of the C3
// correlator with its sub-FFTs exchanging in place in the window (no separate
// exchange rows), so the windows fit a stage and the ring keeps copying ahead.
// The producer copied the rows inside the signal (packed); the compute threads
// fill the others.  Windows past the request's last block (in its last item)
// are zeros and store nothing.
template<int LOGN>
__device__ __noinline__ bool xrw_window(const args& A, const stage_meta& mt, unsigned char* buf, bool bad, int tid,
                                        uint64_t* empty_bar) {
    using F            = xrw_cfg<LOGN>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int TT1  = F::TT1;
    constexpr int TT2  = F::TT2;
    constexpr int RS   = F::RS;
    constexpr int W    = F::W;
    constexpr int E    = 16;
    using XC           = xch_in_column<RS, TT1 - 1>;
    using XR           = xch_in_row<RS, TT2 - 1>;
    static_assert(F::WIN <= STAGE, "the windows fit a stage");
    cpx<float>*       win  = reinterpret_cast<cpx<float>*>(buf);
    const cpx<float>* tw1  = sub_tab<F::LOGN1>();
    const cpx<float>* tw2  = sub_tab<F::LOGN2>();
    const cpx<float>* fwb  = A.tb.x2tw[LOGN];
    const cpx<float>* fwu1 = fwb + F::NB;
    const cpx<float>* fwu2 = fwu1 + N2;
    const xc_req&     q    = mt.xq;
    const cpx<float>* kp   = q.kspec;    // K[k1 + N1*k2] / N at [k1*N2 + k2]
    // rows of each window past the copied ones: packed samples, zeros past the signal
    for (int w = 0; w < W; ++w) {
        const long long b0  = (long long)(mt.it.b + w) * q.step;
        const bool      in  = w < mt.it.c;
        const int       rin = in ? xc2_rows_inside<N1, N2>(q.len - b0) : 0;
        for (int e = tid; e < (N1 - rin) * N2; e += NT) {
            const int       r   = rin + e / N2, c = e % N2;
            const long long pos = b0 + (long long)r * N2 + c;
            float           re = 0.f, im = 0.f;
            if (in && pos < q.len) {
                const long long o = ((pos >> 3) << 4) + (pos & 7);
                re                = q.src[o];
                im                = q.src[o + 8];
            }
            float* row                         = reinterpret_cast<float*>(win + (w * N1 + r) * RS);
            row[((c >> 3) << 4) + (c & 7)]     = re;
            row[((c >> 3) << 4) + (c & 7) + 8] = im;
        }
    }
    // the first block barrier also votes on `bad`
    if (bar1_any<NT>(bad)) return false;
    for (int e = tid; e < W * N1 * N2 / 8; e += NT) {
        const int    r  = e % (W * N1), p = e / (W * N1);
        float4*      wp = reinterpret_cast<float4*>(win + r * RS + p * 8);
        const float4 r0 = wp[0], r1 = wp[1], i0 = wp[2], i1 = wp[3];
        wp[0]           = make_float4(r0.x, i0.x, r0.y, i0.y);
        wp[1]           = make_float4(r0.z, i0.z, r0.w, i0.w);
        wp[2]           = make_float4(r1.x, i1.x, r1.y, i1.y);
        wp[3]           = make_float4(r1.z, i1.z, r1.w, i1.w);
    }
    xch_sync<NT>();
    // ---- step 1: columns, forward, times W_N^(k1*n2); group g owns column g % N2 of window g / N2
    {
        const int   g   = tid / TT1, t = tid % TT1;
        const int   n2  = g % N2;
        cpx<float>* col = win + (g / N2) * N1 * RS;
        cpx<float>  v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = col[(t + i * TT1) * RS + n2];
        });
        stage_compute_tab<P1, 0>(v, t, tw1);
        run_stages_full<P1, XC, true, -1>(v, col, n2, t, tw1);
        __syncwarp();    // the column's exchange reads are done
        apply_fourstep_tw(v, ldg_cpx(fwb + t * n2), ldg_cpx(fwu1 + n2), [&](auto ic, cpx<float> o) {
            constexpr int i              = decltype(ic)::value;
            col[(t + i * TT1) * RS + n2] = o;
        });
    }
    xch_sync<NT>();
    // ---- step 2: rows; spectrum times the kernel's; inverse rows
    {
        const int g = tid / TT2, t = tid % TT2;
        int       R = g;    // the row: a half-warp's row groups take consecutive rows (RS = 4 mod 16) ...
        if constexpr (RS % 16 == 2) {
            // ... or rows S apart, S = TT2 / 2 (RS = 2 mod 16), to stay on distinct banks
            constexpr int S  = TT2 / 2;
            constexpr int U  = 16 / TT2;
            const int     bb = g / U, u = g % U;
            R                = (bb / S) * 8 + (bb % S) + u * S;
        }
        const int   k1  = R % N1;
        cpx<float>* row = win + (R / N1) * N1 * RS;
        cpx<float>  v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = row[k1 * RS + t + i * TT2];
        });
        stage_compute_tab<P2, 0>(v, t, tw2);
        run_stages_full<P2, XR, true, -1>(v, row, k1, t, tw2);
        static_for<E>([&](auto ic) {
            constexpr int    i = decltype(ic)::value;
            const cpx<float> k = ldg_cpx(kp + k1 * N2 + t + i * TT2);
            v[i]               = cmul(cpx<float>{v[i].re, -v[i].im}, k);
        });
        stage_compute_tab<P2, 0>(v, t, tw2);
        run_stages_full<P2, XR, true, -1>(v, row, k1, t, tw2);
        __syncwarp();
        apply_fourstep_tw(v, ldg_cpx(fwb + k1 * t), ldg_cpx(fwu2 + k1), [&](auto ic, cpx<float> o) {
            constexpr int i             = decltype(ic)::value;
            row[k1 * RS + t + i * TT2] = o;
        });
    }
    xch_sync<NT>();
    // ---- step 3: columns again; outputs y = conj(.) for window positions
    // n < step inside the signal
    {
        const int       g   = tid / TT1, t = tid % TT1;
        const int       w   = g / N2, n2 = g % N2;
        cpx<float>*     col = win + w * N1 * RS;
        const long long b0  = (long long)(mt.it.b + w) * q.step;
        const int       hi  = w < mt.it.c ? (int)min((long long)q.step, q.len - b0) : 0;
        cpx<float>      v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = col[(t + i * TT1) * RS + n2];
        });
        stage_compute_tab<P1, 0>(v, t, tw1);
        run_stages_full<P1, XC, true, -1>(v, col, n2, t, tw1);
        // the windows are read: the stage may be refilled while the outputs go out
        fence_proxy_async_smem();
        __syncwarp();
        if (tid % 32 == 0) mbar_arrive(empty_bar);
        float* drow = q.dst + 2 * b0 + 2 * t * N2 + ((n2 >> 3) << 4) + (n2 & 7);
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            if ((t + i * TT1) * N2 + n2 < hi) {
                __stcs(drow + 2 * i * TT1 * N2, v[i].re);
                __stcs(drow + 2 * i * TT1 * N2 + 8, -v[i].im);
            }
        });
    }
    return true;
}

// Up to M overlap-save blocks of one correlation (N_fft <= 8192) from their
// packed windows in the stage.
// Not inlined into its run loop: the correlation's two transforms need every
// register (inlined, the loop's state spilled).
template<int LOGN>
__device__ __noinline__ bool xr_items(const args& A, const stage_meta& mt, unsigned char* buf, bool bad, int tid,
                                      uint64_t* empty_bar) {
    const item&   it = mt.it;
    using G          = xrg<LOGN>;
    using P          = typename G::P;
    constexpr int E  = P::E;
    constexpr int TT = G::TT;
    constexpr int SW = TT >= 32 ? 16 : 0;
    static_assert(TT % 8 == 0, "whole packs per thread stride");
    const xc_req& q  = mt.xq;
    const int     m  = tid / TT;
    const int     t  = tid - m * TT;
    const long long b0 = (long long)(it.b + m) * q.step;
    // window samples left before the signal's end (0 for windows past the item)
    const long long left = m < it.c ? q.len - b0 : 0;
    const int       lim  = (int)(left < G::L ? (left > 0 ? left : 0) : G::L);
    const float*  in = reinterpret_cast<const float*>(buf);
    cpx<float>    v[E];
    static_for<E>([&](auto ic) {
        constexpr int    i = decltype(ic)::value;
        const cpx<float> x = lds_swapped<float, SW>(in, m * G::WS + pk<LPK>(t) + 2 * i * TT, 8);
        // the window is zero past the signal (the copy took whole packs)
        v[i] = t + i * TT < lim ? x : cpx<float>{0.f, 0.f};
    });
    constexpr bool TS  = LOGN <= SUB_HI;    // its table is in shared memory
    using PT           = std::conditional_t<TS, sub_plan<(TS ? LOGN : SUB_LO)>, P>;
    const auto*    fst = [&]() {
        if constexpr (TS) return sub_tab<(TS ? LOGN : SUB_LO)>();
        else return A.tb.xft[LOGN];
    }();
    auto* xch = reinterpret_cast<cpx<float>*>(buf);
    stage_compute_tab<P, 0>(v, t, fst);
    if (run_stages_full<P, typename G::X, TS, NT, PT>(v, xch, m, t, fst, bad)) return false;
    // v[i] = X[t + i*TT]: conj(X) * K, then the forward transform again
    static_for<E>([&](auto ic) {
        constexpr int    i = decltype(ic)::value;
        const cpx<float> k = ldg_cpx(q.kspec + t + i * TT);
        v[i]               = cmul(cpx<float>{v[i].re, -v[i].im}, k);
    });
    stage_compute_tab<P, 0>(v, t, fst);
    run_stages_full<P, typename G::X, TS, NT, PT>(v, xch, m, t, fst);
    fence_proxy_async_smem();    // the stage is read: it may be refilled
    __syncwarp();
    if (tid % 32 == 0) mbar_arrive(empty_bar);
    if (m < it.c) {
        // outputs t + i*TT < min(step, samples left); the window starts on a
        // whole pack, so the packed offset is a base plus a constant
        const int olim = lim < q.step ? lim : q.step;
        float*    d    = q.dst + 2 * b0 + pk<LPK>(t);
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            if (t + i * TT < olim) {
                d[2 * i * TT]     = v[i].re;
                d[2 * i * TT + 8] = -v[i].im;
            }
        });
    }
    return true;
}

// ---------------------------------------------------------------- producer
// Bytes and copies of an item into stage `buf` (lane 0 registers the bytes
// on `bar` first; the lanes issue the copies).  XC items copy nothing.
template<int L1, int L2>
__device__ void issue_col(const args& A, const item& it, unsigned char* buf, uint64_t* bar, int lane, uint64_t pol) {
    using F = fsg<L1, L2>;
    if (lane == 0) {
        mbar_arrive_expect_tx(bar, F::N1 * F::SEG * 4);
        const CUtensorMap* map = A.tmaps + it.tmap;
#pragma unroll
        for (int y = 0; y < F::N1; y += F::BOXY) {
            tma_load_3d_hint(buf + y * F::SEG * 4, map, 2 * it.b * F::C, y, it.tz, bar, pol);
        }
    }
}
template<int L1, int L2>
__device__ void issue_row(const args& A, const item& it, unsigned char* buf, uint64_t* bar, int lane) {
    using F = fsg<L1, L2>;
    if (lane == 0) {
        fence_proxy_async_global();    // other blocks' column stores -> TMA reads
        mbar_arrive_expect_tx(bar, F::CR * F::N2 * 8);
    }
    __syncwarp();
    const cpx<float>* g = static_cast<const cpx<float>*>(it.p1) + (long long)it.b * F::CR * F::N2;
    for (int q = lane; q < F::CR; q += 32) {
        bulk_g2s(reinterpret_cast<cpx<float>*>(buf) + q * F::RSI, g + (long long)q * F::N2, F::N2 * 8, bar);
    }
}
template<int LOGL>
__device__ void issue_single(const args& A, const item& it, unsigned char* buf, uint64_t* bar, int lane) {
    using G = sgg<LOGL>;
    if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)it.b * G::L * 8);
    __syncwarp();
    for (int q = lane; q < it.b; q += 32) {
        bulk_g2s(reinterpret_cast<float*>(buf) + q * G::RS, A.req[it.a + q].src, G::L * 8, bar);
    }
}

// The rows of a 4096- or 8192-point correlation item's windows that lie
// inside the signal (one bulk copy of N2 packed samples per row) into the
// stage, window w at rows [w*N1, (w+1)*N1).
template<int LOGN>
__device__ void issue_xrw(const args& A, const item& it, unsigned char* buf, uint64_t* bar, int lane) {
    using F            = xrw_cfg<LOGN>;
    const xc_req& q    = A.xreq[it.a];
    int           rin[F::W];
    uint32_t      rows = 0;
    for (int w = 0; w < F::W; ++w) {
        rin[w] = w < it.c ? xc2_rows_inside<F::N1, F::N2>(q.len - (long long)(it.b + w) * q.step) : 0;
        rows += (uint32_t)rin[w];
    }
    if (lane == 0) mbar_arrive_expect_tx(bar, rows * F::N2 * 8);
    __syncwarp();
    cpx<float>* win = reinterpret_cast<cpx<float>*>(buf);
    for (int w = 0; w < F::W; ++w) {
        const long long b0 = (long long)(it.b + w) * q.step;
        for (int r = lane; r < rin[w]; r += 32) {
            bulk_g2s(win + (w * F::N1 + r) * F::RS, q.src + 2 * (b0 + (long long)r * F::N2), F::N2 * 8, bar);
        }
    }
}

template<int LOGN>
__device__ void issue_xr(const args& A, const item& it, unsigned char* buf, uint64_t* bar, int lane) {
    if constexpr (LOGN >= XRW) {
        issue_xrw<LOGN>(A, it, buf, bar, lane);
        return;
    }
    using G          = xrg<LOGN>;
    const xc_req& q  = A.xreq[it.a];
    // window m: samples [(b+m)*step, +L) of the packed signal, whole packs
    // up to the signal's end
    uint32_t bytes = 0;
    for (int m = 0; m < it.c; ++m) {
        const long long pos   = (long long)(it.b + m) * q.step;
        const long long valid = q.len - pos < G::L ? q.len - pos : G::L;
        bytes += (uint32_t)((valid + 7) / 8) * 64;
    }
    if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
    __syncwarp();
    for (int m = lane; m < it.c; m += 32) {
        const long long pos   = (long long)(it.b + m) * q.step;
        const long long valid = q.len - pos < G::L ? q.len - pos : G::L;
        bulk_g2s(reinterpret_cast<float*>(buf) + m * G::WS, q.src + 2 * pos, (uint32_t)((valid + 7) / 8) * 64, bar);
    }
}

// The rows of a 16384-point correlation window that lie inside the signal,
// one bulk copy of N2 packed samples per row, to the window rows at the
// ring's start (the ring is drained first).
template<int LOGN>
__device__ void issue_xc2(const args& A, const item& it, uint64_t* bar, int lane) {
    using F          = xc2_cfg<LOGN>;
    const xc_req& q  = A.xreq[it.a];
    const long long b0 = (long long)it.b * q.step;
    const int     rin = xc2_rows_inside<F::N1, F::N2>(q.len - b0);
    if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)rin * F::N2 * 8);
    __syncwarp();
    cpx<float>* win = reinterpret_cast<cpx<float>*>(rg_smem);
    for (int r = lane; r < rin; r += 32) {
        bulk_g2s(win + r * F::RS, q.src + 2 * (b0 + (long long)r * F::N2), F::N2 * 8, bar);
    }
}

#define PCX_RG_FOURSTEP(X) X(13, 6, 7) X(14, 6, 8) X(15, 6, 9) X(16, 6, 10) X(17, 7, 10) X(18, 8, 10)
#define PCX_RG_CHECK_SPLIT(LG, A1, A2) static_assert(split_l1(LG) == A1 && LG == A1 + A2, "one split table");
PCX_RG_FOURSTEP(PCX_RG_CHECK_SPLIT)
#undef PCX_RG_CHECK_SPLIT
#define PCX_RG_SINGLE(X) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)
#define PCX_RG_XC(X) X(14)
#define PCX_RG_XR(X) X(7) X(8) X(9) X(10) X(11) X(12) X(13)

// ---------------------------------------------------------------- runs
// The compute warps take the items of the ring in order.  Consecutive items
// of one kind and size are worked by one run function, which loops until the
// next item is of another kind or size; the runs are not inlined into the
// dispatch, so each is allocated its registers on its own, and a call is made
// per run of items rather than per item.

// Compute-warp state carried from one run to the next.
struct cstate {
    int       s;         // stage of the next item in the block's ring sequence
    uint32_t  par;       // parity of that stage's current phase
    uint32_t  colpar;    // bit s: parity of the next slot hand-off wait on stage s
    bool      bad;       // a bounded wait of this thread gave up
};

enum : int { RUN_NEXT = 0, RUN_LEAVE = 1 };

// Waits (bounded) until the copies of the item in stage s (phase parity par)
// have landed and returns its index:
// -1 at the end of the queue, -2 when the wait gave up (the thread then votes
// at barrier 1, where every other compute thread meets it at the first
// barrier of its next item, and all of them leave).
__device__ __forceinline__ int next_item(const args& A, int s, uint32_t par) {
    if (!mbar_wait_bounded(&s_full[s], par)) {
        atomicExch(A.error, 1);
        return -2;
    }
    return s_item[s];
}


// Runs the items from stage cs.s on while Match(item) holds, with
// Work(stage_meta, s, stage buffer) returning false when the block leaves.
template<class Match, class Work>
__device__ __forceinline__ int run_loop(const args& A, cstate& cs, Match&& match, Work&& work) {
    int      s   = cs.s;
    uint32_t par = cs.par;
    int      r   = RUN_NEXT;
    for (;; s = s + 1 == ST ? 0 : s + 1, par ^= s == 0) {
        const int idx = next_item(A, s, par);
        if (idx == -2) {
            bar1_any<NT>(true);
            r = RUN_LEAVE;
            break;
        }
        if (idx < 0) break;    // the dispatch votes and leaves
        const stage_meta& mt = s_meta[s];
        if (!match(mt.it)) break;
        if (!work(mt, s, rg_smem + s * STAGE)) {
            r = RUN_LEAVE;
            break;
        }
    }
    cs.s   = s;
    cs.par = par;
    return r;
}

template<int L1, int L2>
__device__ __noinline__ int run_fourstep(const args& A, int tid, cstate& cs) {
    uint32_t colpar = cs.colpar;
    bool     bad    = cs.bad;
    const int r = run_loop(
        A, cs, [](const item& it) { return (it.kind == K_COL || it.kind == K_ROW) && it.lg == L1 + L2; },
        [&](const stage_meta& mt, int s, unsigned char* buf) -> bool {
            if (mt.it.kind == K_COL) {
                auto slot_ready = [&]() -> bool {
                    const bool ok = mbar_wait_bounded(&s_slotok[s], (colpar >> s) & 1u);
                    colpar ^= 1u << s;
                    if (!ok) atomicExch(A.error, 1);
                    return ok;
                };
                if (!col_item<L1, L2>(mt, buf, bad, tid, slot_ready, &s_empty[s])) return false;
                if (!bad) {
                    __syncwarp();
                    if (tid % 32 == 0) mbar_arrive(&s_written[s]);
                }
                return true;
            }
            return row_item<L1, L2>(mt, buf, bad, tid, &s_empty[s]);
        });
    cs.colpar = colpar;
    cs.bad    = bad;
    return r;
}

template<int LOGL>
__device__ __noinline__ int run_single(const args& A, int tid, cstate& cs) {
    bool      bad = cs.bad;
    const int r   = run_loop(
        A, cs, [](const item& it) { return it.kind == K_SINGLE && it.lg == LOGL; },
        [&](const stage_meta& mt, int s, unsigned char* buf) -> bool {
            return single_items<LOGL>(A, mt, buf, bad, tid, &s_empty[s]);
        });
    cs.bad = bad;
    return r;
}

template<int LOGN>
__device__ __noinline__ int run_xr(const args& A, int tid, cstate& cs) {
    bool      bad = cs.bad;
    const int r   = run_loop(
        A, cs, [](const item& it) { return it.kind == K_XR && it.lg == LOGN; },
        [&](const stage_meta& mt, int s, unsigned char* buf) -> bool {
            if constexpr (LOGN >= XRW) return xrw_window<LOGN>(A, mt, buf, bad, tid, &s_empty[s]);
            else return xr_items<LOGN>(A, mt, buf, bad, tid, &s_empty[s]);
        });
    cs.bad = bad;
    return r;
}

template<int LOGN>
__device__ __noinline__ int run_xc(const args& A, int tid, cstate& cs) {
    const bool bad = cs.bad;
    return run_loop(
        A, cs, [](const item& it) { return it.kind == K_XC && it.lg == LOGN; },
        [&](const stage_meta& mt, int s, unsigned char*) -> bool {
            if (bar1_any<NT>(bad)) return false;
            xc2_window<LOGN>(A, mt, tid, &s_empty[s]);    // releases the ring once the window is read
            return true;
        });
}

// The arguments sit in device memory (uploaded once at creation): the item
// functions take them by reference without a per-thread copy.
__global__ void __launch_bounds__(NT + 64, 1) k_ragged(const args* __restrict__ Ap) {
    const args& A   = *Ap;
    const int   tid = threadIdx.x;
    copy_table_to_smem<SUBTAB>(reinterpret_cast<cpx<float>*>(rg_smem + RING), A.tb.sub, tid, NT + 64);
    if (tid == 0) {
        s_conj  = A.conj;
        s_scale = A.scale;
        for (int s = 0; s < ST; ++s) {
            s_item[s] = -2;    // no item yet
            mbar_init(&s_full[s], 1);
            mbar_init(&s_empty[s], NW + 1);
            mbar_init(&s_slotok[s], 1);
            mbar_init(&s_written[s], NW);
        }
        fence_barrier_init();
    }
    __syncthreads();
    if (tid >= NT + 32) {
        // ======================= publisher warp
        const int lane   = tid - NT - 32;
        uint32_t  colpar = 0;    // bit s: parity of the next `written` wait on stage s
        for (int s = 0, par = 0;; s = s + 1 == ST ? 0 : s + 1, par ^= s == 0) {
            int ok = 1;
            if (lane == 0) ok = mbar_wait_bounded(&s_full[s], (uint32_t)par) ? 1 : 0;
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            const int idx = s_item[s];
            if (idx < 0) break;
            const item it = A.items[idx];
            if (it.kind == K_COL) {
                if (lane == 0) ok = mbar_wait_bounded(&s_written[s], (colpar >> s) & 1u) ? 1 : 0;
                colpar ^= 1u << s;
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    if (lane == 0) atomicExch(A.error, 1);
                    break;
                }
                if (lane == 0) {
                    fence_proxy_async_global();    // the slot is read back by TMA copies
                    red_release_add(A.col_done + it.a, 1);
                }
            } else if (it.kind == K_ROW) {
                // the rows are in shared memory: drop their L2 lines unwritten
                const int   l2   = it.lg - split_l1(it.lg);
                const int   cr   = NT / ((1 << l2) / 16);
                const char* g    = reinterpret_cast<const char*>(static_cast<const cpx<float>*>(it.p1) +
                                                                  (long long)it.b * cr * (1LL << l2));
                const int   lines = cr * (1 << l2) * 8 / 128;
                for (int q = lane; q < lines; q += 32) l2_discard(g + (size_t)q * 128);
                __syncwarp();
                if (lane == 0) red_release_add(A.row_done + it.a, 1);
            }
            if (lane == 0) mbar_arrive(&s_empty[s]);
        }
        __syncwarp();
        return;
    }

    if (tid >= NT) {
        // ======================= producer warp
        const int      lane   = tid - NT;
        const uint64_t pol    = l2_evict_first_policy();
        bool           fail   = false;
        long long      issued = 0;
        long long      drain_until = -1;    // after an XC item: wait for it before the next item
        auto           wait_empty = [&](long long q) -> bool {    // stage of item q released
            int ok = 1;
            if (lane == 0) ok = mbar_wait_bounded(&s_empty[(int)(q % ST)], (uint32_t)((q / ST) & 1)) ? 1 : 0;
            return __shfl_sync(0xffffffffu, ok, 0) != 0;
        };
        auto need = [&](const int* ctr, int target) -> bool {
            int ok = 1;
            if (lane == 0) ok = fs_wait(ctr, target) ? 1 : 0;
            return __shfl_sync(0xffffffffu, ok, 0) != 0;
        };
        for (long long k = 0; !fail; ++k) {
            const int s = (int)(k % ST);
            if (k >= ST && !wait_empty(k - ST)) {
                fail = true;
                break;
            }
            if (drain_until >= 0 && !wait_empty(drain_until)) {
                fail = true;
                break;
            }
            drain_until = -1;
            int idx = 0;
            if (lane == 0) idx = (int)atomicAdd(A.counter, 1u);
            idx = __shfl_sync(0xffffffffu, idx, 0);
            unsigned char* buf = rg_smem + s * STAGE;
            if (idx >= A.nitems) {
                if (lane == 0) {
                    s_item[s] = -1;
                    mbar_arrive(&s_full[s]);
                }
                issued = k + 1;
                break;
            }
            const item it = A.items[idx];
            if (lane == 0) {
                // published to the compute warps by this lane's arrival on full[s]
                stage_meta& mt = s_meta[s];
                mt.it          = it;
                if (it.kind == K_XR || it.kind == K_XC) mt.xq = A.xreq[it.a];
                s_item[s] = idx;
            }
            __syncwarp();
            if (it.kind == K_XC) {
                // the correlation uses the whole ring: the other stages' items
                // must be done first, and the next item waits for this one
                for (long long q = k - 1; q >= 0 && q > k - ST && !fail; --q) {
                    if (!wait_empty(q)) fail = true;
                }
                if (fail) break;
                switch (it.lg) {
#define PCX_RG_ISSUE_XC(LG) \
    case LG: issue_xc2<LG>(A, it, &s_full[s], lane); break;
                    PCX_RG_XC(PCX_RG_ISSUE_XC)
#undef PCX_RG_ISSUE_XC
                default:
                    if (lane == 0) mbar_arrive(&s_full[s]);
                    break;
                }
                drain_until = k;
                issued      = k + 1;
                continue;
            }
            if (it.kind == K_XR) {
                switch (it.lg) {
#define PCX_RG_ISSUE_X(LG) \
    case LG: issue_xr<LG>(A, it, buf, &s_full[s], lane); break;
                    PCX_RG_XR(PCX_RG_ISSUE_X)
#undef PCX_RG_ISSUE_X
                default: break;
                }
                issued = k + 1;
            } else if (it.kind == K_SINGLE) {
                switch (it.lg) {
#define PCX_RG_ISSUE_S(LG) \
    case LG: issue_single<LG>(A, it, buf, &s_full[s], lane); break;
                    PCX_RG_SINGLE(PCX_RG_ISSUE_S)
#undef PCX_RG_ISSUE_S
                default: break;
                }
                issued = k + 1;
            } else if (it.kind == K_COL) {
                switch (it.lg) {
#define PCX_RG_ISSUE_C(LG, A1, A2) \
    case LG: issue_col<A1, A2>(A, it, buf, &s_full[s], lane, pol); break;
                    PCX_RG_FOURSTEP(PCX_RG_ISSUE_C)
#undef PCX_RG_ISSUE_C
                default: break;
                }
                issued = k + 1;
                // the slot: free once the transform that used it before has
                // read all its rows
                if (it.prev >= 0 && !need(A.row_done + it.prev, it.prev_rows)) {
                    fail = true;
                    break;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&s_slotok[s]);
            } else {
                if (!need(A.col_done + it.a, A.col_tiles[it.lg])) {
                    fail = true;
                    break;
                }
                switch (it.lg) {
#define PCX_RG_ISSUE_R(LG, A1, A2) \
    case LG: issue_row<A1, A2>(A, it, buf, &s_full[s], lane); break;
                    PCX_RG_FOURSTEP(PCX_RG_ISSUE_R)
#undef PCX_RG_ISSUE_R
                default: break;
                }
                issued = k + 1;
            }
            __syncwarp();
        }
        if (fail && lane == 0) {
            atomicExch(A.error, 1);
            for (long long q = issued - 1; q >= 0 && q >= issued - ST; --q) {
                mbar_wait_bounded(&s_full[(int)(q % ST)], (uint32_t)((q / ST) & 1), 100000000ull);
            }
        }
        __syncwarp();
        return;
    }

    // ======================= compute warps
    cstate cs{0, 0u, 0u, false};
    for (;;) {
        const int idx = next_item(A, cs.s, cs.par);
        if (idx < 0) {
            // the end of the queue, or a wait that gave up: vote, so that
            // every compute thread leaves at the same barrier
            bar1_any<NT>(true);
            return;
        }
        const item it = A.items[idx];
        int        r  = RUN_LEAVE;
        if (it.kind == K_SINGLE) {
            switch (it.lg) {
#define PCX_RG_RUN_S(LG) \
    case LG: r = run_single<LG>(A, tid, cs); break;
                PCX_RG_SINGLE(PCX_RG_RUN_S)
#undef PCX_RG_RUN_S
            default: bar1_any<NT>(true); break;
            }
        } else if (it.kind == K_COL || it.kind == K_ROW) {
            switch (it.lg) {
#define PCX_RG_RUN_F(LG, A1, A2) \
    case LG: r = run_fourstep<A1, A2>(A, tid, cs); break;
                PCX_RG_FOURSTEP(PCX_RG_RUN_F)
#undef PCX_RG_RUN_F
            default: bar1_any<NT>(true); break;
            }
        } else if (it.kind == K_XR) {
            switch (it.lg) {
#define PCX_RG_RUN_XR(LG) \
    case LG: r = run_xr<LG>(A, tid, cs); break;
                PCX_RG_XR(PCX_RG_RUN_XR)
#undef PCX_RG_RUN_XR
            default: bar1_any<NT>(true); break;
            }
        } else {
            switch (it.lg) {
#define PCX_RG_RUN_X(LG) \
    case LG: r = run_xc<LG>(A, tid, cs); break;
                PCX_RG_XC(PCX_RG_RUN_X)
#undef PCX_RG_RUN_X
            default: bar1_any<NT>(true); break;
            }
        }
        if (r == RUN_LEAVE) return;
    }
}

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
void* upload(pcx_ragged_s* h, const std::vector<V>& v, cudaError_t* e, size_t align = 0) {
    void* p = nullptr;
    *e      = cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(V) + align);
    if (*e != cudaSuccess) return nullptr;
    h->allocs.push_back(p);
    if (align) p = reinterpret_cast<void*>((reinterpret_cast<uintptr_t>(p) + align - 1) / align * align);
    if (!v.empty()) *e = cudaMemcpy(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice);
    return p;
}

int lg2(size_t n) { return n ? __builtin_ctzll(n) : -1; }

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

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
    return pcx_ragged_create_tc(out, dtype, n_fft, sizes, dst, src, direction, normalize, n_xc, xc_len, xc_k, xc_g,
                                xc_nfft, xc_dst, xc_src, -1);
}

extern "C" int pcx_ragged_create_tc(pcx_ragged* out, int dtype, size_t n_fft, const size_t* sizes, void* const* dst,
                                    const void* const* src, int direction, int normalize, size_t n_xc,
                                    const size_t* xc_len, const size_t* xc_k, const void* const* xc_g,
                                    const size_t* xc_nfft, void* const* xc_dst, const void* const* xc_src,
                                    int tensor_core) {
    return pcx_guard([&]() -> int {
        if (!out) return pcx_fail(PCX_ERR_INVALID, "handle pointer is null");
        *out = nullptr;
        if (dtype != PCX_F32) return pcx_fail(PCX_ERR_UNSUPPORTED, "ragged batches are built for complex64");
        if (tensor_core < -1 || tensor_core > 2) {
            return pcx_fail(PCX_ERR_INVALID, "tensor_core: -1 off, 0 bf16x3, 1 tf32x3, 2 bf16x6");
        }
        auto  h    = new pcx_ragged_s{};
        auto  fail = [&](int rc) {
            pcx_ragged_destroy(h);
            return rc;
        };
        cudaError_t e = cudaSuccess;
        auto cuda_fail = [&](cudaError_t err) { return fail(pcx_fail(PCX_ERR_CUDA, cudaGetErrorString(err))); };
        // ---- requests and per-size tables
        std::vector<rg::fft_req> req(n_fft);
        std::map<int, std::vector<int>> by_lg;
        for (size_t i = 0; i < n_fft; ++i) {
            const int lg = lg2(sizes[i]);
            if (lg < 5 || lg > 18 || (sizes[i] & (sizes[i] - 1))) {
                return fail(pcx_fail(PCX_ERR_UNSUPPORTED, "ragged FFT sizes must be powers of two in 2^5..2^18"));
            }
            if (!aligned16(src[i]) || !aligned16(dst[i])) {
                return fail(pcx_fail(PCX_ERR_INVALID, "ragged FFT buffers must be 16-byte aligned"));
            }
            req[i] = {static_cast<const float*>(src[i]), static_cast<float*>(dst[i]), -1, -1, 0, -1, 0};
            by_lg[lg].push_back((int)i);
        }
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        h->A.conj  = direction == PCX_INVERSE;
        h->A.scale = 1.0f;
        // the tensor-core form takes the transforms of 2^8..2^12 points
        std::map<int, std::vector<int>> tc_by_lg;
        if (tensor_core >= 0) {
            for (int lg = 8; lg <= 12; ++lg) {
                auto it = by_lg.find(lg);
                if (it == by_lg.end()) continue;
                tc_by_lg[lg] = std::move(it->second);
                by_lg.erase(it);
            }
        }
        if (normalize && direction == PCX_INVERSE) {
            // one scale per launch: every transform of an inverse batch must share N
            if (by_lg.size() + tc_by_lg.size() > 1) {
                return fail(pcx_fail(PCX_ERR_UNSUPPORTED, "a normalised inverse ragged batch needs one size"));
            }
            const int lg = by_lg.empty() ? (tc_by_lg.empty() ? 0 : tc_by_lg.begin()->first) : by_lg.begin()->first;
            h->A.scale = 1.0f / float(size_t(1) << lg);
        }
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
        auto dev_alloc = [&](size_t bytes, void** p) -> cudaError_t {
            cudaError_t r = cudaMalloc(p, bytes);
            if (r == cudaSuccess) h->allocs.push_back(*p);
            return r;
        };
        for (auto& [lg, idx]: by_lg) {
            if (lg <= 12) {
                pcx_plan p = get_plan(lg);
                if (!p) return fail(PCX_ERR_CUDA);
                h->A.tb.stw[lg] = static_cast<const cpx<float>*>(p->stwL);
            } else {
                // the four-step split (split_l1) and its twiddles; the
                // sub-transforms' stage tables are the shared ones (SUBTAB)
                const int l1 = rg::split_l1(lg), l2 = lg - l1;
                const int n1 = 1 << l1, n2 = 1 << l2;
                void*     m  = nullptr;
                if ((e = dev_alloc(((size_t)n1 + 2 * (size_t)n2) * 8, &m)) != cudaSuccess) return cuda_fail(e);
                auto* b = static_cast<cpx<float>*>(m);
                h->A.tb.thi[lg]  = b;
                h->A.tb.tlo[lg]  = b + n1;
                h->A.tb.tb[lg]   = b + n1 + n2;
                if ((e = pcx_gen_twiddles(b, n1, lg, n2, false, 0)) != cudaSuccess) return cuda_fail(e);
                if ((e = pcx_gen_twiddles(b + n1, n2, lg, 1, false, 0)) != cudaSuccess) return cuda_fail(e);
                if ((e = pcx_gen_twiddles(b + n1 + n2, n2, l2 + 4, 1, false, 0)) != cudaSuccess) return cuda_fail(e);
                h->A.col_tiles[lg] = n2 / (rg::NT / std::max(1, n1 / 16));
                h->A.row_tiles[lg] = n1 / (rg::NT / std::max(1, n2 / 16));
            }
        }
        // full stage tables of 2^6, 2^7, 2^8 and 2^10 points, copied to shared memory by every block
        {
            void* sub = nullptr;
            if ((e = dev_alloc(rg::SUBTAB, &sub)) != cudaSuccess) return cuda_fail(e);
            auto*     sb   = static_cast<cpx<float>*>(sub);
            const int kept[4][2] = {{6, rg::sub_off<6>()}, {7, rg::sub_off<7>()}, {8, rg::sub_off<8>()},
                                    {10, rg::sub_off<10>()}};
            for (const auto& k: kept) {
                int fe = 0;
                if ((e = pcx_fourstep_tables(k[0], sb + k[1], false, 0, &fe)) != cudaSuccess) return cuda_fail(e);
            }
            h->A.tb.sub = sub;
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
            if ((e = dev_alloc(xc_nfft[j] * 8, &ks)) != cudaSuccess) return cuda_fail(e);
            pcx_plan p = get_plan(lg);
            if (!p) return fail(PCX_ERR_CUDA);
            int rc = pcx_fft_run(p, ks, xc_g[j], xc_k[j], 1, 8, PCX_FORWARD, 0, 1, 2 * xc_nfft[j], 2 * xc_nfft[j], nullptr,
                                 0, 0, 1.0 / (double)xc_nfft[j]);
            if (rc) return fail(rc);
            // the windows come by bulk copies of whole packs
            if (!aligned16(xc_src[j]) || !aligned16(xc_dst[j])) {
                return fail(pcx_fail(PCX_ERR_INVALID, "ragged correlation buffers must be 16-byte aligned"));
            }
            if (lg == 14 || lg >= rg::XRW) {
                // the in-CTA four-step windows: the spectrum in their (k1, k2)
                // order and the four-step twiddles (shared by the requests of a size)
                auto x2 = [&](auto cfg) -> int {
                    using C  = decltype(cfg);
                    void* kp = nullptr;
                    if ((e = dev_alloc(xc_nfft[j] * 8, &kp)) != cudaSuccess) return cuda_fail(e);
                    if ((e = pcx_xc2_perm_spectrum(ks, kp, C::LOGN1, C::LOGN2, 0)) != cudaSuccess) return cuda_fail(e);
                    ks = kp;
                    if (h->A.tb.x2tw[lg]) return PCX_OK;
                    void* tw = nullptr;
                    if ((e = dev_alloc(((size_t)C::NB + C::N2 + C::N1) * 8, &tw)) != cudaSuccess) return cuda_fail(e);
                    auto* t = static_cast<cpx<float>*>(tw);
                    if ((e = pcx_gen_twiddles(t, C::NB, lg, 1, false, 0)) != cudaSuccess) return cuda_fail(e);
                    if ((e = pcx_gen_twiddles(t + C::NB, C::N2, lg, C::TT1, false, 0)) != cudaSuccess) return cuda_fail(e);
                    if ((e = pcx_gen_twiddles(t + C::NB + C::N2, C::N1, lg, C::TT2, false, 0)) != cudaSuccess) {
                        return cuda_fail(e);
                    }
                    h->A.tb.x2tw[lg] = t;
                    return PCX_OK;
                };
                if (int rc2 = lg == 14 ? x2(xc2_cfg<14>{}) : lg == 13 ? x2(rg::xrw_cfg<13>{}) : x2(rg::xrw_cfg<12>{})) return rc2;
            } else if (!h->A.tb.xft[lg]) {
                int   fe = 0;
                void* ft = nullptr;
                if ((e = pcx_fourstep_tables(lg, nullptr, false, 0, &fe)) != cudaSuccess) return cuda_fail(e);
                if ((e = dev_alloc((size_t)fe * 8, &ft)) != cudaSuccess) return cuda_fail(e);
                if ((e = pcx_fourstep_tables(lg, ft, false, 0, &fe)) != cudaSuccess) return cuda_fail(e);
                h->A.tb.xft[lg] = static_cast<const cpx<float>*>(ft);
            }
            xreq[j] = {static_cast<const float*>(xc_src[j]), static_cast<float*>(xc_dst[j]), (long long)xc_len[j],
                       (int)step, (int)((xc_len[j] + step - 1) / step), lg, static_cast<const cpx<float>*>(ks)};
        }
        // ---- requests grouped by size (single-pass items take consecutive requests)
        {
            std::vector<rg::fft_req> sorted;
            for (auto& [lg, idx]: by_lg) {
                for (int& i: idx) {
                    sorted.push_back(req[i]);
                    i = (int)sorted.size() - 1;
                }
            }
            req.swap(sorted);
        }
        // ---- work queue
        // Single-pass items are spread between the four-step work; the
        // four-step transforms run in order of size, column tiles of transform
        // q beside the row tiles of transform q - lag, where the lag covers
        // about three items per block in flight; correlations come last.
        const long long in_flight = 3LL * sms * rg::ST / 2;
        std::vector<rg::item> fill;
        for (auto& [lg, idx]: by_lg) {
            if (lg > 12) continue;
            const int M = rg::NT / std::max(1, (1 << lg) / 16);
            for (size_t q = 0; q < idx.size(); q += M) {
                rg::item it{rg::K_SINGLE, lg, idx[q], (int)std::min<size_t>(M, idx.size() - q), 0};
                it.prev = -1;
                it.p0   = h->A.tb.stw[lg];
                fill.push_back(it);
            }
        }
        // correlations of up to 8192 points: M windows per item, on the ring
        for (size_t j = 0; j < n_xc; ++j) {
            const int lg = xreq[j].lg;
            if (lg > 13) continue;
            const int M = rg::NT / ((1 << lg) / 16);
            for (int b = 0; b < xreq[j].nblk; b += M) {
                rg::item it{rg::K_XR, lg, (int)j, b, std::min(M, xreq[j].nblk - b)};
                it.prev = -1;
                fill.push_back(it);
            }
        }
        std::vector<rg::item> items;
        std::vector<CUtensorMap> maps;
        size_t fi = 0, nfour_total = 0;
        for (auto& [lg, idx]: by_lg)
            if (lg > 12) nfour_total += idx.size();
        size_t four_seen = 0;
        auto push_fill = [&](size_t upto) {
            while (fi < std::min(upto, fill.size())) items.push_back(fill[fi++]);
        };
        for (auto& [lg, idx]: by_lg) {
            if (lg <= 12) continue;
            const int       l1 = rg::split_l1(lg), l2 = lg - l1;
            const int       tc = h->A.col_tiles[lg], tr = h->A.row_tiles[lg];
            const long long lag = std::max<long long>(1, (in_flight + tc + tr - 1) / (tc + tr));
            // this size's ring of scratch slots: 2*lag + 2 transforms
            const size_t nslot = std::min<size_t>(idx.size(), (size_t)(2 * lag + 2));
            void*        scr   = nullptr;
            if ((e = dev_alloc(nslot * ((size_t)8 << lg), &scr)) != cudaSuccess) return cuda_fail(e);
            h->A.tb.scratch[lg] = static_cast<cpx<float>*>(scr);
            // column tiles read the transforms through tensor maps [n1][2*N2
            // reals], box of 2*C reals x min(N1, 256) rows: one map over all of
            // them when they lie at a uniform stride (one descriptor for the
            // SMs' TMA units to cache), else a map per transform
            const int        c      = rg::NT / std::max(1, (1 << l1) / 16);
            const cuuint32_t box[3] = {(cuuint32_t)(2 * c), (cuuint32_t)std::min(1 << l1, 256), 1};
            const cuuint32_t estr[3] = {1, 1, 1};
            long long        ustride = idx.size() > 1 ? (long long)(req[idx[1]].src - req[idx[0]].src) : 0;
            bool             uniform = idx.size() > 1 && ustride >= (2LL << lg) && ustride % 4 == 0;
            for (size_t q = 0; uniform && q < idx.size(); ++q) uniform = req[idx[q]].src == req[idx[0]].src + q * ustride;
            int shared_map = -1;
            if (uniform) {
                CUtensorMap      map;
                const cuuint64_t dims[3] = {(cuuint64_t)2 << l2, (cuuint64_t)1 << l1, (cuuint64_t)idx.size()};
                const cuuint64_t strd[2] = {((cuuint64_t)2 << l2) * 4, (cuuint64_t)ustride * 4};
                if ((e = encode_tensor_map(&map, false, 3, const_cast<float*>(req[idx[0]].src), dims, strd, box, estr)) !=
                    cudaSuccess) {
                    return cuda_fail(e);
                }
                shared_map = (int)maps.size();
                maps.push_back(map);
            }
            for (size_t q = 0; q < idx.size(); ++q) {
                rg::fft_req& r = req[idx[q]];
                r.slot         = (int)(q % nslot);
                r.prev         = q >= nslot ? idx[q - nslot] : -1;
                r.prev_rows    = tr;
                if (shared_map >= 0) {
                    r.tmap = shared_map;
                    r.tz   = (int)q;
                    continue;
                }
                CUtensorMap      map;
                const cuuint64_t dims[3] = {(cuuint64_t)2 << l2, (cuuint64_t)1 << l1, 1};
                const cuuint64_t strd[2] = {((cuuint64_t)2 << l2) * 4, ((cuuint64_t)2 << lg) * 4};
                if ((e = encode_tensor_map(&map, false, 3, const_cast<float*>(r.src), dims, strd, box, estr)) !=
                    cudaSuccess) {
                    return cuda_fail(e);
                }
                r.tmap = (int)maps.size();
                r.tz   = 0;
                maps.push_back(map);
            }
            auto slot_of = [&](int t) -> const void* { return h->A.tb.scratch[lg] + (size_t)req[t].slot * ((size_t)1 << lg); };
            for (size_t q = 0; q < idx.size() + (size_t)lag; ++q) {
                if (q < idx.size()) {
                    const rg::fft_req& r = req[idx[q]];
                    for (int tile = 0; tile < tc; ++tile) {
                        rg::item it{rg::K_COL,  lg,         idx[q],      tile,           0,
                                    r.tmap,     r.tz,       r.prev,      r.prev_rows,    slot_of(idx[q]),
                                    h->A.tb.thi[lg], h->A.tb.tlo[lg], h->A.tb.tb[lg]};
                        items.push_back(it);
                    }
                }
                if (q >= (size_t)lag && q - lag < idx.size()) {
                    const int t = idx[q - lag];
                    for (int tile = 0; tile < tr; ++tile) {
                        rg::item it{rg::K_ROW, lg, t, tile, 0, 0, 0, -1, 0, req[t].dst, slot_of(t)};
                        items.push_back(it);
                    }
                }
                if (q < idx.size()) ++four_seen;
                push_fill(nfour_total ? four_seen * fill.size() / nfour_total : fill.size());
            }
        }
        push_fill(fill.size());
        // 16384-point correlations last, one window per item
        for (size_t j = 0; j < n_xc; ++j) {
            if (xreq[j].lg <= 13) continue;
            for (int b = 0; b < xreq[j].nblk; ++b) {
                rg::item it{rg::K_XC, xreq[j].lg, (int)j, b, 1};
                it.prev = -1;
                items.push_back(it);
            }
        }
        h->n_fft   = n_fft;
        // tensor-core items: 4096 points each (2^(12 - lg) transforms of one size)
        std::vector<tc_item> tc_items;
        for (auto& [lg, idx]: tc_by_lg) {
            const size_t per = size_t(1) << (12 - lg);
            for (size_t q = 0; q < idx.size(); q += per) {
                tc_item ti{};
                ti.lg   = lg;
                ti.rows = (int)std::min(per, idx.size() - q);
                for (int r = 0; r < ti.rows; ++r) {
                    ti.src[r] = static_cast<const float*>(src[idx[q + r]]);
                    ti.dst[r] = static_cast<float*>(dst[idx[q + r]]);
                }
                tc_items.push_back(ti);
            }
        }
        const tc_item* d_tc = nullptr;
        void*          tc_tw = nullptr;
        if (!tc_items.empty()) {
            d_tc = static_cast<const tc_item*>(upload(h, tc_items, &e));
            if (e != cudaSuccess) return cuda_fail(e);
            // W_4096^i, i < 4096: every item size reads it at a stride
            if ((e = dev_alloc(4096 * 8, &tc_tw)) != cudaSuccess) return cuda_fail(e);
            if ((e = pcx_gen_twiddles(tc_tw, 4096, 12, 1, false, 0)) != cudaSuccess) return cuda_fail(e);
        }
        h->n_items = items.size() + tc_items.size();
        // ---- device state
        h->A.items = static_cast<const rg::item*>(upload(h, items, &e));
        if (e == cudaSuccess) h->A.req = static_cast<const rg::fft_req*>(upload(h, req, &e));
        if (e == cudaSuccess) h->A.xreq = static_cast<const rg::xc_req*>(upload(h, xreq, &e));
        if (e == cudaSuccess) h->A.tmaps = static_cast<const CUtensorMap*>(upload(h, maps, &e, 128));
        if (e != cudaSuccess) return cuda_fail(e);
        h->A.nitems  = (int)items.size();
        h->ctl_bytes = (2 + 2 * std::max<size_t>(n_fft, 1)) * sizeof(int);
        void* ctl    = nullptr;
        if ((e = dev_alloc(h->ctl_bytes, &ctl)) != cudaSuccess) return cuda_fail(e);
        h->ctl        = ctl;
        int* c        = static_cast<int*>(h->ctl);
        h->A.counter  = reinterpret_cast<unsigned*>(c);
        h->A.error    = c + 1;
        h->A.col_done = c + 2;
        h->A.row_done = c + 2 + std::max<size_t>(n_fft, 1);
        if ((e = cudaFuncSetAttribute(rg::k_ragged, cudaFuncAttributeMaxDynamicSharedMemorySize, rg::SMEM)) !=
            cudaSuccess) {
            return cuda_fail(e);
        }
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rg::k_ragged, rg::NT + 64, rg::SMEM)) !=
            cudaSuccess) {
            return cuda_fail(e);
        }
        const rg::args* d_args = static_cast<const rg::args*>(upload(h, std::vector<rg::args>{h->A}, &e));
        if (e != cudaSuccess) return cuda_fail(e);
        if (per_sm < 1) {
            cudaFuncAttributes fa{};
            cudaFuncGetAttributes(&fa, rg::k_ragged);
            return fail(pcx_fail(PCX_ERR_CUDA, "ragged kernel does not fit an SM (registers " + std::to_string(fa.numRegs) +
                                                   ", max threads " + std::to_string(fa.maxThreadsPerBlock) +
                                                   ", static smem " + std::to_string(fa.sharedSizeBytes) + ")"));
        }
        h->grid = sms * per_sm;
        if ((e = cudaMemset(h->ctl, 0, h->ctl_bytes)) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(e);
        // ---- capture: reset counters, one persistent launch
        cudaStream_t cs = nullptr;
        if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e);
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->ctl, 0, h->ctl_bytes, cs);
        if (e == cudaSuccess) {
            rg::k_ragged<<<h->grid, rg::NT + 64, rg::SMEM, cs>>>(d_args);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && !tc_items.empty()) {
            e = pcx_tc_list_launch(tensor_core, d_tc, (int)tc_items.size(), h->A.conj, h->A.scale, tc_tw, 12,
                                   h->A.error, sms, cs);
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
