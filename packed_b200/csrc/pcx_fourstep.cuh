// One persistent launch for a whole batch of four-step transforms N = N1*N2.
//
// The column and row passes of every transform are work items of a single
// grid: for transform r there are TC = N2/C column tiles (C columns of N1
// points, TMA tensor copies of the source, twiddled, written to a scratch
// slot) and TR = N1/CR row tiles (CR rows of N2 points read back from the
// slot, written to the destination).  Items are ordered
//     col(0..lag-1), [col(r+lag), row(r)] for r = 0.., row(batch-lag..)
// and CTA b takes items b, b + grid, b + 2*grid, ...  A row tile waits until
// all column tiles of its transform are written (col_done[r] == TC); a column
// tile of transform r writes slot r & (nslot-1) only after every row tile of
// transform r - nslot has read it (row_done[r - nslot] == TR).  Every
// dependency points to an earlier item, so the smallest unfinished item can
// always run.
//
// Each CTA has NT compute threads and two helper warps, so that no wait sits
// on the compute warps' path except their own tile landing:
//  * the producer warp walks the CTA's items, waits for a ring stage to be
//    free and for the item's dependency on other CTAs, and issues the TMA
//    copies into the ST-stage ring (for a column tile it also tells the
//    compute warps when the slot may be written);
//  * the publisher warp walks the same items and publishes each completion as
//    soon as it happens (col_done once the compute warps wrote a column tile;
//    row_done once a row tile's scratch rows have landed in shared memory and
//    their L2 lines are dropped unwritten).  It never waits on another CTA, so
//    the completions other CTAs wait for are never held up behind this CTA's
//    own dependency waits.
// A stage is refilled after the compute warps are done with it and the
// publisher has passed its item (empty[s] counts both), so no barrier phase is
// ever overtaken.  With three stages the exchanges of the sub-transforms run
// in place in the item's own stage buffer (the tile is in registers by the
// first exchange barrier), which keeps the ring within the shared memory of
// two stages plus an exchange buffer while the producer runs two items ahead.
//
// Compared with one launch per pass per scratch chunk this removes the ramp
// and tail of every short launch (the SMs were idle ~30% of each chunk).
#pragma once

#include "pcx_fft_v2.cuh"

namespace pcxg {

struct fs_args {
    const void* src;
    void*       dst;
    long long   src_stride;    // reals between transforms
    long long   dst_stride;
    long long   batch;
    int         conj_in;
    int         conj_out;
    double      scale;
    const void* stw1;     // full stage tables of the N1 and N2 sub-transforms (fs_full_tw_*)
    const void* stw2;
    const void* tw_hi;    // W_N^(i*N2), i < N1
    const void* tw_lo;    // W_N^i, i < N2
    const void* tw_b;     // W_{16*N2}^m
    void*       scratch;  // nslot slots of N complex
    int         nslot;    // a power of two: transform r uses slot r & (nslot - 1)
    int         lag;      // transforms between a column pass and its row pass
    int*        col_done;
    int*        row_done;
    int*        error;
};

// Variant of the one-launch four-step: split N = 2^LOGN1 * 2^LOGN2, MINB
// resident blocks per SM (tiles of 64 KB / MINB: two blocks of 32 KB tiles
// let one block issue while the other waits at a barrier, and need both
// sub-transforms <= 512 points so that a tile still spans whole 32-byte
// sectors of its rows), and ST ring stages (3: the exchanges run in place in
// the item's stage; 2: a separate exchange buffer).  pcx_plan_tune times the
// variants that are built for a size and keeps the fastest.
template<class T, int LOGN1, int LOGN2, int MINB_ = (LOGN1 <= 9 ? 2 : 1), int ST_ = 3>
struct fs_cfg {
    static constexpr int N1   = 1 << LOGN1;
    static constexpr int N2   = 1 << LOGN2;
    static constexpr int MINB = MINB_;
    static constexpr int TILE = 65536 / MINB / (int)sizeof(cpx<T>);
    static constexpr int G8   = 64 / (2 * (int)sizeof(T));
    static constexpr int LP   = G8 == 8 ? 3 : 2;
    static constexpr int C    = (TILE >> LOGN1) > G8 ? (TILE >> LOGN1) : G8;    // columns per column tile
    static constexpr int CR   = (TILE >> LOGN2) > G8 ? (TILE >> LOGN2) : G8;    // rows per row tile
    using P1                  = splan<LOGN1>;
    using P2                  = splan<LOGN2>;
    static constexpr int NT   = C * P1::TT;
    static_assert(NT == CR * P2::TT, "both passes use the same block");
    static constexpr int TC   = N2 / C;
    static constexpr int TR   = N1 / CR;
    static constexpr int RSI  = N2 + 2;    // padded shared row of a row tile (complex)
    static constexpr int COLB = N1 * 2 * C * (int)sizeof(T);
    static constexpr int ROWB = CR * RSI * (int)sizeof(cpx<T>);
    using X1                  = xch_interleaved<N1, C>;
    using X2                  = xch_grouped<N2, CR, G8>;
    static constexpr int XB   = smem_align16((X1::size > X2::size ? X1::size : X2::size) * (int)sizeof(cpx<T>));
    static constexpr int ST   = ST_;
    static constexpr bool IP  = ST == 3;
    static_assert(ST == 2 || ST == 3, "two or three ring stages");
    static constexpr int TILEB = COLB > ROWB ? COLB : ROWB;
    static constexpr int STAGE = ((IP ? (TILEB > XB ? TILEB : XB) : TILEB) + 127) / 128 * 128;
    static constexpr int BASE = ST * STAGE + (IP ? 0 : XB);
    // one stage table for both passes when the larger sub-transform's serves
    // the smaller one (equal halves, or 512 with 1024 points): room for it
    // beside a three-stage ring of 64 KB tiles
    using PL                  = std::conditional_t<(LOGN1 >= LOGN2), P1, P2>;
    static constexpr bool ONE = full_tab_serves<P1, PL>() && full_tab_serves<P2, PL>();
    using PT1                 = std::conditional_t<ONE, PL, P1>;
    using PT2                 = std::conditional_t<ONE, PL, P2>;
    static constexpr int TB1  = fs_full_tw_size<PT1>() * (int)sizeof(cpx<T>);
    static constexpr int TB2  = ONE ? 0 : fs_full_tw_size<P2>() * (int)sizeof(cpx<T>);
    static constexpr bool SH  = stw_fits(BASE, TB1 + TB2, MINB);
    static constexpr int SMEM = SH ? BASE + TB1 + TB2 : BASE;
    static constexpr int BOXY = N1 < 256 ? N1 : 256;
};

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait for *p >= target (about one second); false on timeout.
__device__ __forceinline__ bool fs_wait(const int* p, int target) {
    if (ld_acquire(p) >= target) return true;
    const unsigned long long t0 = timer_ns();
    while (true) {
        if (ld_acquire(p) >= target) return true;
        if (timer_ns() - t0 > 1000000000ull) return false;
        __nanosleep(64);
    }
}

struct fs_item {
    int row;     // 0: column tile, 1: row tile
    int r;       // transform
    int tile;
};

// counter += 1 with release semantics at GPU scope: this thread's earlier
// writes, and those it has observed, are visible to whoever acquires the count
__device__ __forceinline__ void red_release_add(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Item j of the queue (32-bit: the launch holds fewer than 2^31 items).  TC
// and TR are powers of two, TC + TR a constant: no division is a real one.
template<int TC, int TR>
__device__ __forceinline__ fs_item fs_decode(uint32_t j, uint32_t batch, uint32_t lag) {
    const uint32_t A = lag * TC;
    if (j < A) return {0, (int)(j / TC), (int)(j % TC)};
    j -= A;
    constexpr uint32_t G      = TC + TR;
    const uint32_t     steady = (batch - lag) * G;
    if (j < steady) {
        const uint32_t q = j / G;
        const int      w = (int)(j - q * G);
        return w < TC ? fs_item{0, (int)(q + lag), w} : fs_item{1, (int)q, w - TC};
    }
    j -= steady;
    return {1, (int)(batch - lag + j / TR), (int)(j % TR)};
}

template<class T, int LOGN1, int LOGN2, int MINB, int ST_>
__global__ void __launch_bounds__(fs_cfg<T, LOGN1, LOGN2, MINB, ST_>::NT + 64, MINB)
    k_fourstep(const __grid_constant__ CUtensorMap tmap, fs_args a) {
    using F            = fs_cfg<T, LOGN1, LOGN2, MINB, ST_>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int NT   = F::NT;    // compute threads; then the producer warp, then the publisher warp
    constexpr int NW   = NT / 32;
    constexpr int ST   = F::ST;
    constexpr bool IP  = F::IP;
    constexpr int C    = F::C;
    constexpr int CR   = F::CR;
    constexpr int TC   = F::TC;
    constexpr int TR   = F::TR;
    constexpr int LP   = F::LP;
    constexpr int PK   = 1 << LP;
    constexpr int G8   = F::G8;
    constexpr int SEG  = 2 * C;
    constexpr int SW   = sizeof(T) == 8 ? 8 : 16;
    constexpr int RSI  = F::RSI;
    constexpr int RROW = N2 * (int)sizeof(cpx<T>);
    constexpr bool SH  = F::SH;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char*      ring = smem;
    cpx<T>*             tws1 = reinterpret_cast<cpx<T>*>(smem + F::BASE);
    cpx<T>*             tws2 = F::ONE ? tws1 : tws1 + F::TB1 / (int)sizeof(cpx<T>);
    // with one table it is the larger sub-transform's
    const void*         gtab1 = F::ONE && LOGN2 > LOGN1 ? a.stw2 : a.stw1;
    const void*         gtab2 = F::ONE && LOGN1 > LOGN2 ? a.stw1 : a.stw2;
    __shared__ uint64_t full[ST];      // TMA bytes landed
    __shared__ uint64_t empty[ST];     // compute warps done with the stage, publisher past its item
    __shared__ uint64_t slotok[ST];    // column tile: its scratch slot may be written
    __shared__ uint64_t written[ST];   // column tile: compute warps wrote the slot
    cpx<T>*             scr   = reinterpret_cast<cpx<T>*>(a.scratch);
    const int           tid   = threadIdx.x;
    const uint32_t      items = (uint32_t)a.batch * (uint32_t)(TC + TR);    // < 2^31 (host check)
    const uint32_t      batch = (uint32_t)a.batch;
    const uint32_t      lag   = (uint32_t)a.lag;
    const uint32_t      G     = gridDim.x;
    const long long     mask  = a.nslot - 1;

    if constexpr (SH) {
        copy_table_to_smem<F::TB1>(tws1, gtab1, tid, NT + 64);
        if constexpr (!F::ONE) copy_table_to_smem<F::TB2>(tws2, a.stw2, tid, NT + 64);
    }
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW + 1);
            mbar_init(&slotok[s], 1);
            mbar_init(&written[s], NW);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (tid >= NT + 32) {
        // ======================= publisher warp
        const int lane    = tid - NT - 32;
        uint32_t  colpar  = 0;    // bit s: parity of the next `written` wait on stage s
        bool      fail    = false;
        int       s       = 0;
        uint32_t  par     = 0;
        for (uint32_t j = blockIdx.x; j < items && !fail; j += G, s = s + 1 == ST ? 0 : s + 1, par ^= s == 0) {
            const fs_item  it  = fs_decode<TC, TR>(j, batch, lag);
            int            ok  = 1;
            if (!it.row) {
                // the compute warps' stores of the tile are done: make them
                // visible to other CTAs' TMA reads, then count the tile
                if (lane == 0) ok = mbar_wait_bounded(&written[s], (colpar >> s) & 1u) ? 1 : 0;
                ok = __shfl_sync(0xffffffffu, ok, 0);
                colpar ^= 1u << s;
                if (ok && lane == 0) {
                    fence_proxy_async_global();
                    red_release_add(a.col_done + it.r, 1);
                }
            } else {
                // the tile's scratch rows are in shared memory: drop their L2
                // lines unwritten and count the tile
                if (lane == 0) ok = mbar_wait_bounded(&full[s], par) ? 1 : 0;
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (ok) {
                    const char* g = reinterpret_cast<const char*>(scr + (it.r & mask) * (long long)(N1 * N2) +
                                                                  (long long)it.tile * CR * N2);
                    for (int q = lane; q < CR * RROW / 128; q += 32) l2_discard(g + (size_t)q * 128);
                    __syncwarp();
                    if (lane == 0) red_release_add(a.row_done + it.r, 1);
                }
            }
            if (!ok) {
                fail = true;
                if (lane == 0) atomicExch(a.error, 1);
            } else if (lane == 0) {
                mbar_arrive(&empty[s]);
            }
        }
        __syncwarp();
        return;
    }

    if (tid >= NT) {
        // ======================= producer warp
        const int      lane   = tid - NT;
        const uint64_t pol    = l2_evict_first_policy();    // column tiles are read once
        bool           fail   = false;
        long long      issued = 0;    // items whose copies were issued
        long long      k      = 0;
        // bounded wait for *ctr >= target by lane 0, the answer shared by the warp
        auto need = [&](const int* ctr, int target) -> bool {
            int ok = 1;
            if (lane == 0) ok = fs_wait(ctr, target) ? 1 : 0;
            return __shfl_sync(0xffffffffu, ok, 0) != 0;
        };
        int            s      = 0;
        uint32_t       par    = 0;
        for (uint32_t j = blockIdx.x; j < items && !fail; j += G, ++k, s = s + 1 == ST ? 0 : s + 1, par ^= s == 0) {
            if (k >= ST) {
                int ok = 1;
                if (lane == 0) ok = mbar_wait_bounded(&empty[s], par ^ 1u) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    fail = true;
                    break;
                }
            }
            const fs_item  it  = fs_decode<TC, TR>(j, batch, lag);
            unsigned char* buf = ring + s * F::STAGE;
            if (!it.row) {
                // the source tile does not depend on anything: copy it first
                if (lane == 0) {
                    mbar_arrive_expect_tx(&full[s], F::COLB);
#pragma unroll
                    for (int y = 0; y < N1; y += F::BOXY) {
                        tma_load_3d_hint(buf + y * SEG * (int)sizeof(T), &tmap, 2 * it.tile * C, y, (int)it.r,
                                         &full[s], pol);
                    }
                }
                issued = k + 1;
                // the acquire of the slot's counter (or a first use of the
                // slot) orders the compute warps' writes after the earlier
                // row tiles' reads, through this arrive and their wait
                if (!(it.r < a.nslot || need(a.row_done + (it.r - a.nslot), TR))) {
                    fail = true;
                    break;
                }
                if (lane == 0) mbar_arrive(&slotok[s]);
            } else {
                if (!need(a.col_done + it.r, TC)) {
                    fail = true;
                    break;
                }
                // one bulk copy per row, issued by as many lanes
                if (lane == 0) {
                    fence_proxy_async_global();    // column-pass writes -> TMA reads
                    mbar_arrive_expect_tx(&full[s], CR * RROW);
                }
                __syncwarp();
                const cpx<T>* g = scr + (it.r & mask) * (long long)(N1 * N2) + (long long)it.tile * CR * N2;
                for (int q = lane; q < CR; q += 32) {
                    bulk_g2s(reinterpret_cast<cpx<T>*>(buf) + q * RSI, g + (long long)q * N2, RROW, &full[s]);
                }
                issued = k + 1;
            }
            __syncwarp();
        }
        if (fail && lane == 0) {
            // no copy may still be landing when the block exits: wait
            // (bounded) for the last ST issued items' copies
            atomicExch(a.error, 1);
            for (long long q = issued - 1; q >= 0 && q >= issued - ST; --q) {
                mbar_wait_bounded(&full[(int)(q % ST)], (uint32_t)((q / ST) & 1), 100000000ull);
            }
        }
        __syncwarp();
        return;
    }

    // ======================= compute warps
    // A bounded wait that gives up (tile copy or slot hand-off) is recorded
    // in `bad`; the work of that item goes on with whatever the stage holds,
    // nothing is stored, and at the next exchange barrier, which doubles as
    // a vote, every compute thread leaves together (run_stages_full).
    const int lane   = tid % 32;
    uint32_t  colpar = 0;    // bit s: parity of the next slot hand-off on stage s
    bool      bad    = false;
    int       s      = 0;
    uint32_t  par    = 0;
    cpx<T>*   xsep   = reinterpret_cast<cpx<T>*>(smem + ST * F::STAGE);    // exchange buffer when !IP
    for (uint32_t j = blockIdx.x; j < items; j += G, s = s + 1 == ST ? 0 : s + 1, par ^= s == 0) {
        const fs_item it = fs_decode<TC, TR>(j, batch, lag);
        cpx<T>*        xch = IP ? reinterpret_cast<cpx<T>*>(ring + s * F::STAGE) : xsep;
        // the stage is no longer read: it may be refilled (the publisher adds
        // its own arrival once it has passed the item)
        auto release_stage = [&]() {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        };
        // column tile: the four-step twiddle inputs are requested before the
        // tile's data is waited for, and used after the stages
        cpx<T> th{}, tl{}, tu{};
        if (!it.row) {
            const int      n2 = it.tile * C + tid % C;
            const uint32_t e0 = (uint32_t)(tid / C) * (uint32_t)n2;
            th                = ldg_cpx(reinterpret_cast<const cpx<T>*>(a.tw_hi) + (e0 >> LOGN2));
            tl                = ldg_cpx(reinterpret_cast<const cpx<T>*>(a.tw_lo) + (e0 & (N2 - 1)));
            tu                = ldg_cpx(reinterpret_cast<const cpx<T>*>(a.tw_b) + n2);
        }
        if (!mbar_wait_bounded(&full[s], par)) {
            bad = true;
            atomicExch(a.error, 1);
        }
        if (!it.row) {
            // ---------------- column tile: N1-point DFTs down C columns
            constexpr int E    = P1::E;
            constexpr int TT   = P1::TT;
            const int     c    = tid % C;
            const int     t    = tid / C;
            const int     n2   = it.tile * C + c;
            const T*      in   = reinterpret_cast<const T*>(ring + s * F::STAGE);
            const auto*   stw1 = SH ? tws1 : reinterpret_cast<const cpx<T>*>(gtab1);
            cpx<T>        v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                cpx<T>        x = lds_swapped<T, SW>(in, (t + i * TT) * SEG + pk<LP>(c), PK);
                v[i]            = {x.re, a.conj_in ? -x.im : x.im};
            });
            if constexpr (!IP) release_stage();
            stage_compute_tab<P1, 0>(v, t, stw1);
            if (run_stages_full<P1, typename F::X1, SH, NT, typename F::PT1>(v, xch, c, t, stw1, bad)) return;
            if constexpr (IP) release_stage();
            if (!mbar_wait_bounded(&slotok[s], (colpar >> s) & 1u)) {
                // the producer gave up on this slot: nothing is written, and
                // the compute warps leave at the next item's vote
                bad = true;
                atomicExch(a.error, 1);
            }
            colpar ^= 1u << s;
            if (!bad) {
                cpx<T>* dst = scr + (it.r & mask) * (long long)(N1 * N2) + (long long)t * N2 + n2;
                apply_fourstep_tw(v, cmul(th, tl), tu, [&](auto ic, cpx<T> o) {
                    constexpr int i             = decltype(ic)::value;
                    dst[(long long)i * TT * N2] = o;
                });
                __syncwarp();
                if (lane == 0) mbar_arrive(&written[s]);
            }
        } else {
            // ---------------- row tile: N2-point DFTs along CR rows
            constexpr int E    = P2::E;
            constexpr int TT   = P2::TT;
            const int     mlo  = tid % G8;
            const int     t    = (tid / G8) % TT;
            const int     mhi  = tid / (G8 * TT);
            const int     m    = mhi * G8 + mlo;
            const int     k1   = it.tile * CR + m;
            const auto*   stw2 = SH ? tws2 : reinterpret_cast<const cpx<T>*>(gtab2);
            const cpx<T>* in   = reinterpret_cast<const cpx<T>*>(ring + s * F::STAGE) + m * RSI + t;
            cpx<T>        v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                v[i]            = in[i * TT];
            });
            if constexpr (!IP) release_stage();
            stage_compute_tab<P2, 0>(v, t, stw2);
            if (run_stages_full<P2, typename F::X2, SH, NT, typename F::PT2>(v, xch, m, t, stw2, bad)) return;
            if constexpr (IP) release_stage();
            T*      dst = reinterpret_cast<T*>(a.dst) + it.r * a.dst_stride + pk<LP>(t * N1 + k1);
            const T sc  = T(a.scale);
            const T sim = a.conj_out ? -sc : sc;
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                __stcs(dst + 2 * i * TT * N1, v[i].re * sc);
                __stcs(dst + 2 * i * TT * N1 + PK, v[i].im * sim);
            });
        }
    }
}

}    // namespace pcxg
