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
// tile of transform r writes slot r % nslot only after every row tile of
// transform r - nslot has read it (row_done[r - nslot] == TR).  Every
// dependency points to an earlier item, so the smallest unfinished item can
// always run.
//
// Each CTA has NT compute threads and one copy warp.  The copy warp owns
// everything that waits on other CTAs: it checks dependencies, issues the TMA
// copies into a two-stage ring, tells the compute warps when a column tile's
// slot is free, and publishes completions (col_done after the compute warps
// have written a column tile; row_done once a row tile's scratch rows have
// landed in shared memory and their L2 lines are dropped without write-back).
// Before it blocks on another CTA it first publishes its own pending
// completion, so it never waits while holding one.  The compute warps only
// wait on mbarriers of their own CTA and synchronise among themselves on a
// named barrier, so no dependency latency sits on their critical path.
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
    const void* stw1;     // stage tables of the N1 and N2 sub-transforms
    const void* stw2;
    const void* tw_hi;    // W_N^(i*N2), i < N1
    const void* tw_lo;    // W_N^i, i < N2
    const void* tw_b;     // W_{16*N2}^m
    void*       scratch;  // nslot slots of N complex
    int         nslot;
    int         lag;      // transforms between a column pass and its row pass
    int*        col_done;
    int*        row_done;
    int*        error;
};

template<class T, int LOGN1, int LOGN2>
struct fs_cfg {
    static constexpr int N1   = 1 << LOGN1;
    static constexpr int N2   = 1 << LOGN2;
    // Two blocks per SM with 32 KB tiles while a column tile still spans
    // whole 32-byte sectors of its rows (N1 <= 512): the two blocks' barrier
    // phases run independently, so one issues while the other waits.
    static constexpr int MINB = LOGN1 <= 9 ? 2 : 1;
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
    static constexpr int STAGE = ((COLB > ROWB ? COLB : ROWB) + 127) / 128 * 128;
    using X1                  = xch_interleaved<N1, C>;
    using X2                  = xch_grouped<N2, CR, G8>;
    static constexpr int XB   = smem_align16((X1::size > X2::size ? X1::size : X2::size) * (int)sizeof(cpx<T>));
    static constexpr int BASE = 2 * STAGE + XB;
    static constexpr int TB1  = stage_tw_smem_bytes<P1, T>();
    static constexpr int TB2  = stage_tw_smem_bytes<P2, T>();
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
    int       row;     // 0: column tile, 1: row tile
    long long r;       // transform
    int       tile;
};

// OR of `bad` over the NT compute threads (named barrier 2), the same answer
// in every one of them.
template<int NT>
__device__ __forceinline__ bool compute_any_failed(bool bad) {
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.or.pred q, 2, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((uint32_t)bad), "n"(NT)
                 : "memory");
    return r != 0;
}

// counter += 1 with release semantics at GPU scope: this thread's earlier
// writes, and those it has observed, are visible to whoever acquires the count
__device__ __forceinline__ void red_release_add(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ fs_item fs_decode(long long j, long long batch, int lag, int TC, int TR) {
    const long long A = (long long)lag * TC;
    if (j < A) return {0, j / TC, (int)(j % TC)};
    j -= A;
    const long long G      = TC + TR;
    const long long steady = (batch - lag) * G;
    if (j < steady) {
        const long long q = j / G;
        const int       w = (int)(j - q * G);
        return w < TC ? fs_item{0, q + lag, w} : fs_item{1, q, w - TC};
    }
    j -= steady;
    return {1, batch - lag + j / TR, (int)(j % TR)};
}

template<class T, int LOGN1, int LOGN2>
__global__ void __launch_bounds__(fs_cfg<T, LOGN1, LOGN2>::NT + 32, fs_cfg<T, LOGN1, LOGN2>::MINB)
    k_fourstep(const __grid_constant__ CUtensorMap tmap, fs_args a) {
    using F            = fs_cfg<T, LOGN1, LOGN2>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int NT   = F::NT;    // compute threads; warp NT/32 copies
    constexpr int NW   = NT / 32;
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
    cpx<T>*             xch  = reinterpret_cast<cpx<T>*>(smem + 2 * F::STAGE);
    cpx<T>*             tws1 = reinterpret_cast<cpx<T>*>(smem + F::BASE);
    cpx<T>*             tws2 = tws1 + F::TB1 / (int)sizeof(cpx<T>);
    __shared__ uint64_t full[2];     // TMA bytes landed
    __shared__ uint64_t empty[2];    // compute warps have read the stage
    __shared__ uint64_t slotok[2];   // column tile: its scratch slot may be written
    __shared__ uint64_t written[2];  // column tile: compute warps wrote the slot
    cpx<T>*             scr   = reinterpret_cast<cpx<T>*>(a.scratch);
    const int           tid   = threadIdx.x;
    const long long     items = a.batch * (TC + TR);
    const long long     G     = gridDim.x;

    if constexpr (SH) {
        stage_tw_to_smem<P1, T>(tws1, a.stw1, tid, NT + 32);
        stage_tw_to_smem<P2, T>(tws2, a.stw2, tid, NT + 32);
    }
    if (tid == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW);
            mbar_init(&slotok[s], 1);
            mbar_init(&written[s], NW);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (tid >= NT) {
        // ======================= copy warp
        const int      lane     = tid - NT;
        const uint64_t pol      = l2_evict_first_policy();    // column tiles are read once
        long long      pending  = -1;    // item whose completion is not yet published
        int            pend_s   = 0;
        uint32_t       pend_par = 0;
        long long      rowdef   = -1;    // row item published once its stage was read
        int            rd_s     = 0;
        uint32_t       rd_par   = 0;
        bool           fail     = false;
        int            ncol[2]  = {0, 0};    // column items seen per stage (slotok / written phases)
        int            pcol     = 0;         // written phase of the pending column item
        // bounded mbarrier wait by lane 0, the answer shared by the warp
        auto wwait = [&](uint64_t* bar, uint32_t parity) -> bool {
            int ok = 1;
            if (lane == 0) ok = mbar_wait_bounded(bar, parity) ? 1 : 0;
            return __shfl_sync(0xffffffffu, ok, 0) != 0;
        };
        // row item `jr` is done once its rows are in shared memory: drop their
        // L2 lines unwritten and count it
        auto publish_row = [&](long long jr) {
            const fs_item it = fs_decode(jr, a.batch, a.lag, TC, TR);
            const char*   g  = reinterpret_cast<const char*>(scr + (it.r % a.nslot) * (long long)(N1 * N2) +
                                                          (long long)it.tile * CR * N2);
            for (int q = lane; q < CR * RROW / 128; q += 32) l2_discard(g + (size_t)q * 128);
            __syncwarp();
            if (lane == 0) red_release_add(a.row_done + it.r, 1);
        };
        // the deferred row item, after waiting for its rows to land
        auto flush_rowdef = [&]() {
            if (rowdef < 0) return;
            if (!wwait(&full[rd_s], rd_par)) fail = true;
            if (!fail) publish_row(rowdef);
            rowdef = -1;
        };
        // publish the completion of `pending`; a row item may instead be
        // deferred until the compute warps have read its stage (so its copy
        // has landed without waiting for it here)
        auto complete = [&](bool defer_row) {
            if (pending < 0) return;
            const fs_item it = fs_decode(pending, a.batch, a.lag, TC, TR);
            if (!it.row) {
                if (!wwait(&written[pend_s], (uint32_t)(pcol & 1))) fail = true;
                if (lane == 0 && !fail) {
                    fence_proxy_async_global();    // the slot is read back by TMA copies
                    red_release_add(a.col_done + it.r, 1);
                }
            } else if (defer_row) {
                rowdef = pending;
                rd_s   = pend_s;
                rd_par = pend_par;
            } else {
                if (!wwait(&full[pend_s], pend_par)) fail = true;
                if (!fail) publish_row(pending);
            }
            pending = -1;
        };
        // wait for *ctr >= target, publishing every pending completion first
        auto need = [&](const int* ctr, int target) -> bool {
            int v = 0;
            if (lane == 0) v = ld_acquire(ctr);
            v = __shfl_sync(0xffffffffu, v, 0);
            if (v >= target) return true;
            flush_rowdef();
            complete(false);
            if (fail) return false;
            int ok = 1;
            if (lane == 0) ok = fs_wait(ctr, target) ? 1 : 0;
            return __shfl_sync(0xffffffffu, ok, 0) != 0;
        };
        long long k = 0;
        for (long long j = blockIdx.x; j < items && !fail; j += G, ++k) {
            const int      s   = (int)(k & 1);
            const uint32_t par = (uint32_t)((k >> 1) & 1);
            if (k >= 2 && !wwait(&empty[s], par ^ 1u)) {
                fail = true;
                break;
            }
            // the stage's previous item (k-2) has been read: a deferred row
            // item from it is done
            if (rowdef >= 0) {
                publish_row(rowdef);
                rowdef = -1;
            }
            const fs_item  it  = fs_decode(j, a.batch, a.lag, TC, TR);
            unsigned char* buf = ring + s * F::STAGE;
            if (!it.row) {
                if (lane == 0) {
                    mbar_arrive_expect_tx(&full[s], F::COLB);
#pragma unroll
                    for (int y = 0; y < N1; y += F::BOXY) {
                        tma_load_3d_hint(buf + y * SEG * (int)sizeof(T), &tmap, 2 * it.tile * C, y, (int)it.r,
                                         &full[s], pol);
                    }
                }
                const bool ok = it.r < a.nslot || need(a.row_done + (it.r - a.nslot), TR);
                if (!ok) {
                    fail     = true;
                    pending  = j;    // the copy is in flight: wait for it below
                    pend_s   = s;
                    pend_par = par;
                    break;
                }
                __syncwarp();
                // the acquire of the slot's counter (or a first use of the
                // slot) orders the compute warps' writes after the earlier
                // row tiles' reads, through this arrive and their wait
                if (lane == 0) mbar_arrive(&slotok[s]);
                complete(true);
                pending  = j;
                pend_s   = s;
                pend_par = par;
                pcol     = ncol[s]++;
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
                const cpx<T>* g = scr + (it.r % a.nslot) * (long long)(N1 * N2) + (long long)it.tile * CR * N2;
                for (int q = lane; q < CR; q += 32) {
                    bulk_g2s(reinterpret_cast<cpx<T>*>(buf) + q * RSI, g + (long long)q * N2, RROW, &full[s]);
                }
                __syncwarp();
                complete(true);
                pending  = j;
                pend_s   = s;
                pend_par = par;
            }
        }
        if (!fail) {
            flush_rowdef();
            complete(false);
        }
        if (fail && lane == 0) {
            // no copy may still be landing when the block exits
            atomicExch(a.error, 1);
            if (pending >= 0) mbar_wait_bounded(&full[pend_s], pend_par, 100000000ull);
            if (rowdef >= 0) mbar_wait_bounded(&full[rd_s], rd_par, 100000000ull);
        }
        __syncwarp();
        return;
    }

    // ======================= compute warps
    const int lane    = tid % 32;
    int       ncol[2] = {0, 0};
    long long k       = 0;
    for (long long j = blockIdx.x; j < items; j += G, ++k) {
        const int      s   = (int)(k & 1);
        const uint32_t par = (uint32_t)((k >> 1) & 1);
        const fs_item it = fs_decode(j, a.batch, a.lag, TC, TR);
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
        // all compute warps leave together when any of them gave up
        if (compute_any_failed<NT>(!mbar_wait_bounded(&full[s], par))) {
            if (tid == 0) atomicExch(a.error, 1);
            return;
        }
        if (!it.row) {
            // ---------------- column tile: N1-point DFTs down C columns
            constexpr int E    = P1::E;
            constexpr int TT   = P1::TT;
            const int     c    = tid % C;
            const int     t    = tid / C;
            const int     n2   = it.tile * C + c;
            const T*      in   = reinterpret_cast<const T*>(ring + s * F::STAGE);
            const auto*   stw1 = SH ? tws1 : reinterpret_cast<const cpx<T>*>(a.stw1);
            cpx<T>        v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                cpx<T>        x = lds_swapped<T, SW>(in, (t + i * TT) * SEG + pk<LP>(c), PK);
                v[i]            = {x.re, a.conj_in ? -x.im : x.im};
            });
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            stage_compute_tab<P1, 0>(v, t, stw1);
            run_stages_tab<P1, typename F::X1, SH, NT>(v, xch, c, t, stw1);
            const bool sok = mbar_wait_bounded(&slotok[s], (uint32_t)(ncol[s] & 1));
            ++ncol[s];
            if (compute_any_failed<NT>(!sok)) {
                // the copy warp gave up on this slot: nothing is written
                if (tid == 0) atomicExch(a.error, 1);
                return;
            }
            cpx<T>* dst = scr + (it.r % a.nslot) * (long long)(N1 * N2) + (long long)t * N2 + n2;
            apply_fourstep_tw(v, cmul(th, tl), tu, [&](auto ic, cpx<T> o) {
                constexpr int i             = decltype(ic)::value;
                dst[(long long)i * TT * N2] = o;
            });
            __syncwarp();
            if (lane == 0) mbar_arrive(&written[s]);
        } else {
            // ---------------- row tile: N2-point DFTs along CR rows
            constexpr int E    = P2::E;
            constexpr int TT   = P2::TT;
            const int     mlo  = tid % G8;
            const int     t    = (tid / G8) % TT;
            const int     mhi  = tid / (G8 * TT);
            const int     m    = mhi * G8 + mlo;
            const int     k1   = it.tile * CR + m;
            const auto*   stw2 = SH ? tws2 : reinterpret_cast<const cpx<T>*>(a.stw2);
            const cpx<T>* in   = reinterpret_cast<const cpx<T>*>(ring + s * F::STAGE) + m * RSI + t;
            cpx<T>        v[E];
            static_for<E>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                v[i]            = in[i * TT];
            });
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            stage_compute_tab<P2, 0>(v, t, stw2);
            run_stages_tab<P2, typename F::X2, SH, NT>(v, xch, m, t, stw2);
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
