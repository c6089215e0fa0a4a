// Overlap-save correlation for FP32 blocks of N = N1 * N2 = 2^13 or 2^14
// points (reference fxcorr.hpp:102-136), one block per CTA at a time.
//
// The N-point window sits in shared memory as N1 rows of N2 samples.  Its
// forward FFT is a four-step inside the CTA, and the inverse runs the same
// steps backwards, so no step needs the spectrum in natural order:
//   1. columns: N1-point FFT of every column n2, times W_N^(k1*n2);
//   2. rows:    N2-point FFT of every row k1 gives X[k1 + N1*k2] in
//               registers; times conj(K) (K = FFT(g)/N, stored row-major in
//               the same (k1, k2) order so the loads are coalesced); the
//               inverse N2-point FFT of the row (as FFT of the conjugate) and
//               times W_N^(k1*n2) again (the conjugate form of W_N^-(k1*n2));
//   3. columns: N1-point FFT of every column gives conj(y[n1*N2 + n2]),
//               written straight to the output.
// (y[n] = (1/N) sum_k Y[k] W_N^-(nk) with n = n1*N2 + n2, k = k1 + N1*k2
// splits as W_N1^-(n1*k1) * W_N^-(n2*k1) * W_N2^-(n2*k2).)
// Each sub-FFT belongs to a group of TT threads inside one warp, 16 points
// per thread, exchanging through a private padded buffer with warp barriers
// only; block barriers separate the steps.  The window rows arrive by 1-D
// bulk copies of the packed signal (one per row of 64-byte packs, converted
// in place to interleaved complex); rows that reach outside the signal are
// filled by the threads, with zeros outside.  Once step 3 has read the
// window, the copies of the CTA's next block start, so they land while step
// 3 finishes.
//
// In place, a block's outputs overwrite samples that the previous block's
// window reads, so every block publishes "window loaded" (the call's epoch in
// flags[item]) and waits for its predecessors before writing, as the general
// kernel does; the waits are bounded (about one second).
#pragma once

#include "pcx_fft_v2.cuh"
#include "pcx_fxcorr_kernels.cuh"
#include "pcx_tmem.cuh"

namespace pcxg {

template<int LOGN>
struct xc2_cfg {
    static constexpr int LOGN1 = (LOGN + 1) / 2;
    static constexpr int LOGN2 = LOGN / 2;
    static constexpr int N1    = 1 << LOGN1;
    static constexpr int N2    = 1 << LOGN2;
    static constexpr int N     = N1 * N2;
    using P1                   = splan<LOGN1>;
    using P2                   = splan<LOGN2>;
    static constexpr int NT    = 512;
    static constexpr int TT1   = P1::TT;
    static constexpr int TT2   = P2::TT;
    static constexpr int G1    = NT / TT1;    // column groups per round
    static constexpr int G2    = NT / TT2;    // row groups per round
    static constexpr int R1    = N2 / G1;     // column rounds
    static constexpr int R2    = N1 / G2;     // row rounds
    static constexpr int RS    = N2 + 2;      // window row stride (complex), 2 mod 16
    static constexpr int WIN   = N1 * RS * 8;
    using X1                   = xch_blocked<N1, G1>;
    using X2                   = xch_blocked<N2, G2>;
    static constexpr int XB    = (X1::size > X2::size ? X1::size : X2::size) * 8;
    static constexpr int TB1   = smem_align16(fs_full_tw_size<P1>() * 8);    // full stage tables
    static constexpr int TB2   = smem_align16(fs_full_tw_size<P2>() * 8);
    static constexpr int NB    = N / 16;      // W_N^e, e < N/16 (= TT1*N2 = TT2*N1)
    // in shared memory entry e sits at e + e/16: the threads of a warp read
    // e = t*n2 for eight t, which would share banks whenever n2 is a multiple of 16
    static constexpr int NBP   = NB + NB / 16;
    static constexpr int SMEM  = WIN + XB + TB1 + TB2 + (NBP + N2 + N1) * 8;
    static_assert(P1::E == 16 && P2::E == 16, "16 points per thread");
    static_assert(TT1 <= 32 && TT2 <= 32 && TT2 >= 2, "sub-FFT groups inside one warp");
    static_assert(R1 >= 1 && R2 >= 1 && G1 * R1 == N2 && G2 * R2 == N1, "rounds");
    static_assert(TT1 * N2 == NB && TT2 * N1 == NB, "twiddle split");
    static_assert(NBP % 2 == 0, "16-byte offset of the tables behind it");
    static_assert(WIN % 16 == 0 && XB % 16 == 0 && TB1 % 16 == 0 && TB2 % 16 == 0, "16-byte sections");
};

struct xc2_args {
    xc_args     base;
    const void* kperm;    // K[k1 + N1*k2] / N at [k1*N2 + k2]
    const void* stw1;     // stage tables of the N1- and N2-point FFTs
    const void* stw2;
    const void* tws;      // W_N^e (e < N/16), W_N^(TT1*n2) (n2 < N2), W_N^(TT2*k1) (k1 < N1)
};

template<int LOGN>
__global__ void __launch_bounds__(512, 1) k_fxcorr2d(xc2_args A) {
    using F            = xc2_cfg<LOGN>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int NT   = F::NT;
    constexpr int TT1  = F::TT1;
    constexpr int TT2  = F::TT2;
    constexpr int RS   = F::RS;
    constexpr int E    = 16;
    const xc_args& a   = A.base;
    extern __shared__ __align__(128) unsigned char smem[];
    cpx<float>*          win  = reinterpret_cast<cpx<float>*>(smem);
    cpx<float>*          xch  = reinterpret_cast<cpx<float>*>(smem + F::WIN);
    cpx<float>*          tw1  = reinterpret_cast<cpx<float>*>(smem + F::WIN + F::XB);
    cpx<float>*          tw2  = tw1 + F::TB1 / 8;
    cpx<float>*          fwb  = tw2 + F::TB2 / 8;    // W_N^e
    cpx<float>*          fwu1 = fwb + F::NBP;        // W_N^(TT1*n2)
    cpx<float>*          fwu2 = fwu1 + N2;           // W_N^(TT2*k1)
    __shared__ uint64_t  full;
    __shared__ long long s_item;
    __shared__ int       s_rlo;
    __shared__ int       s_rhi;
    __shared__ int       s_abort;
    __shared__ uint32_t  s_tmem;
    const int            tid  = threadIdx.x;
    const float*         src  = reinterpret_cast<const float*>(a.src);
    float*               dst  = reinterpret_cast<float*>(a.dst);
    const cpx<float>*    kp   = reinterpret_cast<const cpx<float>*>(A.kperm);

    // constant tables into shared memory
    copy_table_to_smem<F::TB1>(tw1, A.stw1, tid, NT);
    copy_table_to_smem<F::TB2>(tw2, A.stw2, tid, NT);
    const cpx<float>* tws = reinterpret_cast<const cpx<float>*>(A.tws);
    for (int e = tid; e < F::NB; e += NT) fwb[e + (e >> 4)] = ldg_cpx(tws + e);
    for (int i = tid; i < (N2 + N1) / 2; i += NT) {
        reinterpret_cast<uint4*>(fwu1)[i] = __ldg(reinterpret_cast<const uint4*>(tws + F::NB) + i);
    }
    if (tid == 0) {
        mbar_init(&full, 1);
        fence_barrier_init();
    }
    // step 2's row groups: the U groups of a half-warp take rows S apart, so
    // their window rows fall in disjoint banks (RS = 2 mod 16)
    constexpr int S2 = TT2 / 2;
    constexpr int U2 = 16 / TT2;
    const int     g2 = tid / TT2, t2 = tid % TT2;
    const int     r2 = ((g2 / U2) / S2) * 8 + ((g2 / U2) % S2) + (g2 % U2) * S2;
    // The kernel spectrum values a thread multiplies by are the same for every
    // block (its rows k1 = rd*G2 + r2, columns k2 = t2 + i*TT2): they are read
    // once into the thread's tensor-memory lane (otherwise idle in this kernel),
    // 32 columns per row round, instead of from global memory in every block.
    constexpr uint32_t TCOLS = 128 * F::R2;    // four warps share each lane quarter
    static_assert(TCOLS == 128 || TCOLS == 256, "a power-of-two TMEM allocation");
    if (tid < 32) {
        tmem_alloc(&s_tmem, TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = s_tmem;
    const uint32_t tcol  = tbase + ((uint32_t)(32 * ((tid / 32) % 4)) << 16) + (uint32_t)((tid / 128) * 32 * F::R2);
    for (int rd = 0; rd < F::R2; ++rd) {
        const int k1 = rd * F::G2 + r2;
        uint32_t  kr[32];
        static_for<E>([&](auto ic) {
            constexpr int    i = decltype(ic)::value;
            const cpx<float> k = ldg_cpx(kp + k1 * N2 + t2 + i * TT2);
            kr[2 * i]          = __float_as_uint(k.re);
            kr[2 * i + 1]      = __float_as_uint(k.im);
        });
        tmem_st32(tcol + 32 * rd, kr);
    }

    // channel and window start (samples) of an item
    auto item_pos = [&](long long item, long long& ch, long long& b0) {
        ch = item / a.nblk;
        b0 = (item - ch * a.nblk) * a.step - a.in_shift;
    };
    // warp 0: thread 0 claims the next item; the warp's lanes start the
    // copies of its rows that lie inside [0, len), a row each in turn; the
    // threads fill the others
    auto claim_and_copy = [&]() {
        if (tid == 0) {
            const long long item = (long long)atomicAdd(a.counter, 1u);
            s_item               = item;
            if (item < a.total) {
                long long ch, b0;
                item_pos(item, ch, b0);
                long long r_lo = b0 >= 0 ? 0 : (-b0 + N2 - 1) / N2;
                long long r_hi = b0 + (long long)N1 * N2 <= a.len ? N1 : (a.len - b0) / N2;
                r_lo           = r_lo > N1 ? N1 : r_lo;
                r_hi           = r_hi < r_lo ? r_lo : (r_hi > N1 ? N1 : r_hi);
                s_rlo          = (int)r_lo;
                s_rhi          = (int)r_hi;
                mbar_arrive_expect_tx(&full, (uint32_t)(r_hi - r_lo) * (N2 * 8));
            }
        }
        __syncwarp();
        const long long item = s_item;
        if (item >= a.total) return;
        long long ch, b0;
        item_pos(item, ch, b0);
        const float* base = src + ch * a.src_stride + 2 * b0;    // packed: 2 reals per sample
        for (int r = s_rlo + tid; r < s_rhi; r += 32) bulk_g2s(win + r * RS, base + 2LL * r * N2, N2 * 8, &full);
    };

    __syncthreads();
    if (tid < 32) claim_and_copy();
    uint32_t phase = 0;
    for (;;) {
        __syncthreads();
        const long long item = s_item;
        if (item >= a.total) break;
        const int r_lo = s_rlo, r_hi = s_rhi;
        long long ch, b0;
        item_pos(item, ch, b0);
        // rows outside the copied range: packed samples, zeros outside [0, len)
        if (r_hi - r_lo < N1) {
            for (int q = tid; q < N1 * N2; q += NT) {
                const int r = q / N2, c = q - r * N2;
                if (r >= r_lo && r < r_hi) continue;
                const long long pos = b0 + q;
                float           re = 0.f, im = 0.f;
                if (pos >= 0 && pos < a.len) {
                    const long long o = ch * a.src_stride + ((pos >> 3) << 4) + (pos & 7);
                    re                = src[o];
                    im                = src[o + 8];
                }
                float* row                         = reinterpret_cast<float*>(win + r * RS);
                row[((c >> 3) << 4) + (c & 7)]     = re;
                row[((c >> 3) << 4) + (c & 7) + 8] = im;
            }
        }
        const bool ok = mbar_wait_bounded(&full, phase);
        if (__syncthreads_or(!ok)) {
            // give up: record it and let the copies in flight land first
            if (tid == 0) {
                atomicExch(a.error, 1);
                mbar_wait_bounded(&full, phase, 100000000ull);
            }
            __syncthreads();
            break;    // every thread leaves the loop together; TMEM is freed below
        }
        phase ^= 1;
        if (a.inplace && tid == 0) {
            __threadfence();
            st_release(a.flags + item, a.epoch);    // this window is loaded
        }
        // packed -> interleaved, in place, one 64-byte pack per thread and step;
        // consecutive threads take consecutive rows (row stride 65 x 16 bytes),
        // so each quarter-warp's 16-byte accesses hit eight distinct bank groups
        for (int q = tid; q < N1 * N2 / 8; q += NT) {
            const int    r  = q % N1, p = q / N1;
            float4*      w  = reinterpret_cast<float4*>(win + r * RS + p * 8);
            const float4 r0 = w[0], r1 = w[1], i0 = w[2], i1 = w[3];
            w[0]            = make_float4(r0.x, i0.x, r0.y, i0.y);
            w[1]            = make_float4(r0.z, i0.z, r0.w, i0.w);
            w[2]            = make_float4(r1.x, i1.x, r1.y, i1.y);
            w[3]            = make_float4(r1.z, i1.z, r1.w, i1.w);
        }
        __syncthreads();

        // ---------------- step 1: columns, forward, times W_N^(k1*n2)
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
                const int e = t * n2;
                apply_fourstep_tw(v, fwb[e + (e >> 4)], fwu1[n2], [&](auto ic, cpx<float> o) {
                    constexpr int i              = decltype(ic)::value;
                    win[(t + i * TT1) * RS + n2] = o;
                });
            }
        }
        __syncthreads();

        // in place: thread 0 reads the load flags of the first previous windows
        // now, so that step 3 rarely has to wait for them
        unsigned pflag[4] = {0u, 0u, 0u, 0u};
        if (a.inplace && tid == 0) {
            const long long blk = item % a.nblk;
            static_for<4>([&](auto dc) {
                constexpr int d = decltype(dc)::value + 1;
                if (d <= a.hwait && d <= blk) pflag[d - 1] = ld_acquire(a.flags + (item - d));
            });
        }
        // ---------------- step 2: rows; spectrum times conj(K) or K; inverse rows
        {
            const int g = g2, t = t2;
            for (int rd = 0; rd < F::R2; ++rd) {
                const int  k1 = rd * F::G2 + r2;
                cpx<float> v[E];
                static_for<E>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    v[i]            = win[k1 * RS + t + i * TT2];
                });
                stage_compute_tab<P2, 0>(v, t, tw2);
                run_stages_full<P2, typename F::X2, true, -1>(v, xch, g, t, tw2);
                // v[i] = X[k1 + N1*k2], k2 = t + i*TT2: conj(X * conj(K)) or conj(X * K),
                // K from tensor memory eight values at a time
                static_for<2>([&](auto hc) {
                    constexpr int h = decltype(hc)::value;
                    uint32_t      kq[16];
                    tmem_ld16(tcol + 32 * rd + 16 * h, kq);
                    static_for<8>([&](auto jc) {
                        constexpr int    i = 8 * h + decltype(jc)::value;
                        const cpx<float> k = {__uint_as_float(kq[2 * (i - 8 * h)]), __uint_as_float(kq[2 * (i - 8 * h) + 1])};
                        const cpx<float> c = {v[i].re, -v[i].im};
                        v[i]               = a.conj_kernel ? cmul(c, k) : cmulc(c, k);
                    });
                });
                stage_compute_tab<P2, 0>(v, t, tw2);
                run_stages_full<P2, typename F::X2, true, -1>(v, xch, g, t, tw2);
                // v[i] at n2 = t + i*TT2, times W_N^(k1*n2) = W_N^(k1*t) * W_N^(TT2*k1)^i
                const int e = k1 * t;
                apply_fourstep_tw(v, fwb[e + (e >> 4)], fwu2[k1], [&](auto ic, cpx<float> o) {
                    constexpr int i           = decltype(ic)::value;
                    win[k1 * RS + t + i * TT2] = o;
                });
            }
        }
        __syncthreads();

        // ---------------- step 3: columns again; outputs y = conj(.)
        if (a.inplace) {
            // the outputs overwrite samples of the windows of the hwait
            // previous blocks of this channel: wait until those are loaded
            if (tid == 0) {
                s_abort              = 0;
                const long long blk  = item % a.nblk;
                for (int d = 1; d <= a.hwait && d <= blk && !s_abort; ++d) {
                    const unsigned* f = a.flags + (item - d);
                    if (d <= 4) {
                        unsigned pv = 0u;
                        static_for<4>([&](auto ic) {
                            if (decltype(ic)::value == d - 1) pv = pflag[decltype(ic)::value];
                        });
                        if (pv == a.epoch) continue;
                    }
                    if (ld_acquire(f) == a.epoch) continue;
                    const unsigned long long t0 = globaltimer_ns();
                    while (ld_acquire(f) != a.epoch) {
                        if (globaltimer_ns() - t0 > XC_WAIT_NS) {
                            atomicExch(a.error, 1);
                            s_abort = 1;
                            break;
                        }
                        __nanosleep(256);
                    }
                }
            }
            __syncthreads();
            if (s_abort) break;    // every thread leaves together; no copy is in flight
        }
        {
            const int       g    = tid / TT1, t = tid % TT1;
            // window index n is output position e0 + n; it is written when
            // out_shift <= n < out_shift + step and e0 + n < len.  e0 and every
            // row start are whole packs, so the packed offset of e0 + row*N2 + n2
            // is 2*(e0 + row*N2) + pk(n2).
            const long long e0 = b0 + a.in_shift - a.out_shift;
            const int       lo = a.out_shift;
            const long long hl = min((long long)a.out_shift + a.step, a.len - e0);
            const int       hi = (int)max(0LL, min(hl, (long long)N1 * N2));
            float*          d  = dst + ch * a.dst_stride + 2 * e0;
            for (int rd = 0; rd < F::R1; ++rd) {
                const int  n2 = rd * F::G1 + g;
                cpx<float> v[E];
                static_for<E>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    v[i]            = win[(t + i * TT1) * RS + n2];
                });
                if (rd == F::R1 - 1) {
                    // the window is read: start the next block's copies
                    fence_proxy_async_smem();
                    __syncthreads();
                    if (tid < 32) claim_and_copy();
                }
                stage_compute_tab<P1, 0>(v, t, tw1);
                run_stages_full<P1, typename F::X1, true, -1>(v, xch, g, t, tw1);
                float* drow = d + 2 * t * N2 + ((n2 >> 3) << 4) + (n2 & 7);
                static_for<E>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    const int     n = (t + i * TT1) * N2 + n2;    // window index
                    if (n >= lo && n < hi) {
                        __stcs(drow + 2 * i * TT1 * N2, v[i].re);
                        __stcs(drow + 2 * i * TT1 * N2 + 8, -v[i].im);
                    }
                });
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid < 32) tmem_dealloc(tbase, TCOLS);
}

// ---------------------------------------------------------------------------
// Kernel-gradient pass in the same form (the counterpart of k_fxcorr_kgrad for
// FP32 N = 2^13 / 2^14, pack 8): per block, the gy block (zero-padded to N)
// and then the x window land in the window rows, and steps 1-2 of the forward
// four-step leave each thread the spectrum values of its rows k1 at columns
// k2 = t + i*TT2 -- the same (k1, k2) every block.  So each thread keeps its
// share of FFT(gy block) and of the running sum of FFT(x window) *
// conj(FFT(gy block)) in tensor memory: per row round 32 columns of each (at
// 16384 points the SM's 512 TMEM columns hold the spectrum twice; the four
// warps that share a lane quarter take a quarter of the columns each).  At the end every CTA
// writes its sum in natural order (k = k1 + N1*k2) to acc[blockIdx.x]; the
// reduction over CTAs and the inverse FFT follow as for the general kernel.
struct xc2_kg_args {
    kg_args     base;
    const void* stw1;    // as xc2_args
    const void* stw2;
    const void* tws;
};

template<int LOGN>
__global__ void __launch_bounds__(512, 1) k_fxcorr2d_kgrad(xc2_kg_args A) {
    using F            = xc2_cfg<LOGN>;
    using P1           = typename F::P1;
    using P2           = typename F::P2;
    constexpr int N1   = F::N1;
    constexpr int N2   = F::N2;
    constexpr int NT   = F::NT;
    constexpr int TT1  = F::TT1;
    constexpr int TT2  = F::TT2;
    constexpr int RS   = F::RS;
    constexpr int E    = 16;
    // per thread, 32 TMEM columns per row round for FFT(gy) and as many for the sum;
    // the four warps that share a lane quarter take CPT columns each
    constexpr uint32_t CPT   = 64 * F::R2;
    constexpr uint32_t TCOLS = 4 * CPT;
    static_assert(TCOLS == 256 || TCOLS == 512, "a power-of-two TMEM allocation");
    const kg_args& a   = A.base;
    extern __shared__ __align__(128) unsigned char smem[];
    cpx<float>*          win  = reinterpret_cast<cpx<float>*>(smem);
    cpx<float>*          xch  = reinterpret_cast<cpx<float>*>(smem + F::WIN);
    cpx<float>*          tw1  = reinterpret_cast<cpx<float>*>(smem + F::WIN + F::XB);
    cpx<float>*          tw2  = tw1 + F::TB1 / 8;
    cpx<float>*          fwb  = tw2 + F::TB2 / 8;
    cpx<float>*          fwu1 = fwb + F::NBP;
    __shared__ uint64_t  full;
    __shared__ long long s_item;
    __shared__ int       s_rhi;
    __shared__ uint32_t  s_tmem;
    const int            tid  = threadIdx.x;
    const int            warp = tid / 32;

    copy_table_to_smem<F::TB1>(tw1, A.stw1, tid, NT);
    copy_table_to_smem<F::TB2>(tw2, A.stw2, tid, NT);
    const cpx<float>* tws = reinterpret_cast<const cpx<float>*>(A.tws);
    for (int e = tid; e < F::NB; e += NT) fwb[e + (e >> 4)] = ldg_cpx(tws + e);
    for (int i = tid; i < (N2 + N1) / 2; i += NT) {
        reinterpret_cast<uint4*>(fwu1)[i] = __ldg(reinterpret_cast<const uint4*>(tws + F::NB) + i);
    }
    if (warp == 0) {
        tmem_alloc(&s_tmem, TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&full, 1);
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = s_tmem;
    // this thread's columns: FFT(gy) of round rd at 32*rd, the sum at SUM + 32*rd
    constexpr uint32_t SUM  = 32 * F::R2;
    const uint32_t     tcol = tbase + ((uint32_t)(32 * (warp % 4)) << 16) + (uint32_t)(warp / 4) * CPT;
    {
        uint32_t z[32];
        static_for<32>([&](auto jc) { z[decltype(jc)::value] = 0u; });
        for (int rd = 0; rd < F::R2; ++rd) tmem_st32(tcol + SUM + 32 * rd, z);
    }

    // window `ph` of an item: 0 the gy block [b*step, b*step + step), 1 the x
    // window [b*step, b*step + N); samples past the block or the signal are zero
    auto item_pos = [&](long long item, long long& ch, long long& b0) {
        ch = item / a.nblk;
        b0 = (item - ch * a.nblk) * a.step;
    };
    auto valid_of = [&](int ph, long long b0) -> long long {
        const long long v = a.len - b0;
        return ph == 0 ? (v < a.step ? v : (long long)a.step) : v;
    };
    // warp 0: the bulk copies of the whole rows that lie inside the valid
    // samples (thread 0 first claims the next item when ph == 0)
    // rows [lo, hi) of the window (the part of them inside the valid samples);
    // `claim` first sets the window up (the whole window's bytes expected on
    // `full`), so a window may arrive in two batches of rows
    auto copy_window = [&](int ph, bool claim, int lo, int hi) {
        if (claim && tid == 0) {
            if (ph == 0) s_item = (long long)atomicAdd(a.counter, 1u);
            const long long item = s_item;
            if (item < a.total) {
                long long ch, b0;
                item_pos(item, ch, b0);
                long long r_hi = valid_of(ph, b0) / N2;
                r_hi           = r_hi < 0 ? 0 : (r_hi > N1 ? N1 : r_hi);
                s_rhi          = (int)r_hi;
                mbar_arrive_expect_tx(&full, (uint32_t)r_hi * (N2 * 8));
            }
        }
        __syncwarp();
        const long long item = s_item;
        if (item >= a.total) return;
        long long ch, b0;
        item_pos(item, ch, b0);
        const float* base = reinterpret_cast<const float*>(ph == 0 ? a.gy : a.x) + ch * a.stride + 2 * b0;
        const int    rhi  = s_rhi < hi ? s_rhi : hi;
        for (int r = lo + tid; r < rhi; r += 32) bulk_g2s(win + r * RS, base + 2LL * r * N2, N2 * 8, &full);
    };

    __syncthreads();
    if (tid < 32) copy_window(0, true, 0, N1);
    uint32_t phase   = 0;
    bool     aborted = false;
    // step 2's row groups (as k_fxcorr2d): the U groups of a half-warp take
    // rows S apart
    constexpr int S  = TT2 / 2;
    constexpr int U  = 16 / TT2;
    const int     g2 = tid / TT2, t2 = tid % TT2;
    const int     r0 = ((g2 / U) / S) * 8 + ((g2 / U) % S) + (g2 % U) * S;
    for (;;) {
        __syncthreads();
        const long long item = s_item;
        if (item >= a.total) break;
        long long ch, b0;
        item_pos(item, ch, b0);
        for (int ph = 0; ph < 2; ++ph) {
            if (ph == 1) __syncthreads();    // warp 0 has set this window's copies going
            const int       r_hi  = s_rhi;
            const long long valid = valid_of(ph, b0);
            const float*    sp    = reinterpret_cast<const float*>(ph == 0 ? a.gy : a.x) + ch * a.stride;
            // rows past the copied ones: the samples of a partial row, zeros after
            for (int q = r_hi * N2 + tid; q < N1 * N2; q += NT) {
                const int r = q / N2, c = q - r * N2;
                float     re = 0.f, im = 0.f;
                if (q < valid) {
                    const long long pos = b0 + q;
                    const long long o   = ((pos >> 3) << 4) + (pos & 7);
                    re                  = sp[o];
                    im                  = sp[o + 8];
                }
                float* row                         = reinterpret_cast<float*>(win + r * RS);
                row[((c >> 3) << 4) + (c & 7)]     = re;
                row[((c >> 3) << 4) + (c & 7) + 8] = im;
            }
            const bool ok = mbar_wait_bounded(&full, phase);
            if (__syncthreads_or(!ok)) {
                // give up: record it and let the copies in flight land first
                if (tid == 0) {
                    atomicExch(a.error, 1);
                    mbar_wait_bounded(&full, phase, 100000000ull);
                }
                aborted = true;
                break;
            }
            phase ^= 1;
            for (int q = tid; q < N1 * N2 / 8; q += NT) {
                const int    r  = q % N1, p = q / N1;
                float4*      w  = reinterpret_cast<float4*>(win + r * RS + p * 8);
                const float4 r0v = w[0], r1v = w[1], i0v = w[2], i1v = w[3];
                w[0]             = make_float4(r0v.x, i0v.x, r0v.y, i0v.y);
                w[1]             = make_float4(r0v.z, i0v.z, r0v.w, i0v.w);
                w[2]             = make_float4(r1v.x, i1v.x, r1v.y, i1v.y);
                w[3]             = make_float4(r1v.z, i1v.z, r1v.w, i1v.w);
            }
            __syncthreads();
            // ---------------- step 1: columns, forward, times W_N^(k1*n2)
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
                    const int e = t * n2;
                    apply_fourstep_tw(v, fwb[e + (e >> 4)], fwu1[n2], [&](auto ic, cpx<float> o) {
                        constexpr int i              = decltype(ic)::value;
                        win[(t + i * TT1) * RS + n2] = o;
                    });
                }
            }
            __syncthreads();
            // ---------------- step 2: rows; the spectrum to tensor memory
            for (int rd = 0; rd < F::R2; ++rd) {
                const int  k1 = rd * F::G2 + r0;
                cpx<float> v[E];
                static_for<E>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    v[i]            = win[k1 * RS + t2 + i * TT2];
                });
                // round rd has read rows [rd*G2, (rd+1)*G2): the next window's
                // copies into them (the x window of this block, or the next
                // block's gy block) start now, the rest after the last round
                if (F::R2 == 1 || rd == 0 || rd == F::R2 - 1) {
                    fence_proxy_async_smem();
                    __syncthreads();
                    if (tid < 32) {
                        const int lo = F::R2 == 1 || rd == 0 ? 0 : F::G2;
                        const int hi = F::R2 == 1 || rd == F::R2 - 1 ? N1 : F::G2;
                        copy_window(ph ^ 1, rd == 0, lo, hi);
                    }
                }
                stage_compute_tab<P2, 0>(v, t2, tw2);
                run_stages_full<P2, typename F::X2, true, -1>(v, xch, g2, t2, tw2);
                // v[i] = spectrum at k1 + N1*k2, k2 = t2 + i*TT2
                if (ph == 0) {
                    uint32_t r[32];
                    static_for<E>([&](auto ic) {
                        constexpr int i = decltype(ic)::value;
                        r[2 * i]        = __float_as_uint(v[i].re);
                        r[2 * i + 1]    = __float_as_uint(v[i].im);
                    });
                    tmem_st32(tcol + 32 * rd, r);
                } else {
                    // sum += X * conj(GY), eight values at a time
                    static_for<2>([&](auto hc) {
                        constexpr int h = decltype(hc)::value;
                        uint32_t      gq[16], sq[16];
                        tmem_ld16(tcol + 32 * rd + 16 * h, gq);
                        tmem_ld16(tcol + SUM + 32 * rd + 16 * h, sq);
                        static_for<8>([&](auto jc) {
                            constexpr int    j = decltype(jc)::value;
                            const cpx<float> p = cmulc(v[8 * h + j], cpx<float>{__uint_as_float(gq[2 * j]),
                                                                                 __uint_as_float(gq[2 * j + 1])});
                            sq[2 * j]          = __float_as_uint(__uint_as_float(sq[2 * j]) + p.re);
                            sq[2 * j + 1]      = __float_as_uint(__uint_as_float(sq[2 * j + 1]) + p.im);
                        });
                        tmem_st16(tcol + SUM + 32 * rd + 16 * h, sq);
                    });
                }
            }
        }
        if (aborted) break;
    }
    if (!aborted) {
        // this CTA's sum, natural order
        cpx<float>* acc = reinterpret_cast<cpx<float>*>(a.acc) + (long long)blockIdx.x * (N1 * N2);
        for (int rd = 0; rd < F::R2; ++rd) {
            const int k1 = rd * F::G2 + r0;
            uint32_t  sq[32];
            tmem_ld32(tcol + SUM + 32 * rd, sq);
            static_for<E>([&](auto ic) {
                constexpr int i                = decltype(ic)::value;
                acc[k1 + N1 * (t2 + i * TT2)] = {__uint_as_float(sq[2 * i]), __uint_as_float(sq[2 * i + 1])};
            });
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, TCOLS);
}

}    // namespace pcxg
