// Hot-path FFT kernels: natural order, pack width known at compile time.
//
// Differences from the general kernels in pcx_fft_kernels.cuh:
//  * data go straight between global memory and registers — stage 0 reads
//    element t + i*TT of its row, and the Stockham last stage leaves
//    frequency t + i*TT in v[i], so both ends are coalesced without a
//    shared-memory staging copy; shared memory only carries the exchanges
//    between stages;
//  * every address is a per-thread base plus compile-time offsets (sizes and
//    pack width are template parameters);
//  * stage twiddles come from per-stage tables laid out [k][j] so that one
//    butterfly's R twiddles are R contiguous entries (vector loads);
//  * the four-step twiddle W_N^(k1*n2), k1 = t + i*TT, is W_N^(t*n2) (one
//    two-level lookup per thread) times W_{16*N2}^(i*n2) (one table entry).
#pragma once

#include "pcx_fft_kernels.cuh"
#include "pcx_tma.cuh"

namespace pcxg {

// ---- per-stage twiddle tables ------------------------------------------------
// Stage S >= 1 of splan P has Ns = 2^nsbits(S) butterfly positions k and radix
// R.  Its twiddles are W^(j*k), W = W_{Ns*R}, j = 1..R-1.  Writing j = 4m + i
// (i, m < 4), W^(jk) = W^(ik) * W^(4mk), so the table keeps, per position k,
// only the factors (generated in FP64, rounded once):
//   R = 16: W^k, W^2k, W^3k, W^4k, W^8k, W^12k
//   R = 8:  W^k, W^2k, W^3k, W^4k
//   R = 4:  W^k, W^2k, W^3k, 1
//   R = 2:  W^k, 1
// and a butterfly forms each twiddle as one entry or the product of two.  That
// is 48 bytes per radix-16 butterfly instead of 120, and the entries of
// consecutive positions are contiguous (16-byte vector loads).
__host__ __device__ constexpr int stw_q(int rb) { return rb == 4 ? 6 : (rb == 1 ? 2 : 4); }
__host__ __device__ constexpr int stw_mult(int rb, int q) {
    return q < 3 ? ((q + 1) < (1 << rb) ? q + 1 : 0) : (rb == 4 ? 4 * (q - 2) : (rb == 3 && q == 3 ? 4 : 0));
}
template<class P>
__host__ __device__ constexpr int stage_tw_offset(int S) {
    int off = 0;
    for (int s = 1; s < S; ++s) off += (1 << P::nsbits(s)) * stw_q(P::rbits(s));
    return off;
}
template<class P>
__host__ __device__ constexpr int stage_tw_size() {
    return stage_tw_offset<P>(P::NST);
}

template<class T>
__global__ void k_stage_twiddles(cpx<T>* out, int ns, int rb, int log_nsr) {
    const int q  = blockIdx.x * blockDim.x + threadIdx.x;
    const int nq = stw_q(rb);
    if (q >= ns * nq) return;
    const int       k = q / nq, slot = q - k * nq;
    const long long e = (long long)stw_mult(rb, slot) * k;
    double          s, c;
    sincospi(2.0 * (double)e / (double)(1LL << log_nsr), &s, &c);
    out[q] = {T(c), T(-s)};
}

// Two consecutive table entries; SH: the table is in shared memory.
template<bool SH, class T>
__device__ __forceinline__ void ld2(const cpx<T>* p, cpx<T>& a, cpx<T>& b) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = SH ? *reinterpret_cast<const float4*>(p) : __ldg(reinterpret_cast<const float4*>(p));
        a              = {v.x, v.y};
        b              = {v.z, v.w};
    } else {
        if constexpr (SH) {
            a = p[0];
            b = p[1];
        } else {
            a = ldg_cpx(p);
            b = ldg_cpx(p + 1);
        }
    }
}
template<class T>
__device__ __forceinline__ void ldg2(const cpx<T>* p, cpx<T>& a, cpx<T>& b) {
    ld2<false>(p, a, b);
}

// Twiddle j of a radix-R butterfly from its table factors f[0..Q-1].
template<int RB, int J, class T>
__device__ __forceinline__ cpx<T> stw_factor(const cpx<T>* f) {
    constexpr int i = J & 3, m = J >> 2;
    if constexpr (RB <= 2) {
        return f[J - 1];
    } else if constexpr (RB == 3) {
        if constexpr (m == 0) return f[i - 1];
        else if constexpr (i == 0) return f[3];
        else return cmul(f[3], f[i - 1]);
    } else {
        if constexpr (m == 0) return f[i - 1];
        else if constexpr (i == 0) return f[2 + m];
        else return cmul(f[2 + m], f[i - 1]);
    }
}

// Stage-S table factors of thread t (G butterflies): f[g*Q + q].
template<class P, int S, bool SH = false, class T>
__device__ __forceinline__ void load_stage_tw(cpx<T>* f, int t, const cpx<T>* __restrict__ stw) {
    constexpr int RB  = P::rbits(S);
    constexpr int Q   = stw_q(RB);
    constexpr int NSB = P::nsbits(S);
    constexpr int G   = P::E / (1 << RB);
    static_for<G>([&](auto gc) {
        constexpr int g  = decltype(gc)::value;
        const int     k  = (t + g * P::TT) & ((1 << NSB) - 1);
        const cpx<T>* tw = stw + stage_tw_offset<P>(S) + k * Q;
        static_for<Q / 2>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            ld2<SH>(tw + 2 * q, f[g * Q + 2 * q], f[g * Q + 2 * q + 1]);
        });
    });
}

// Butterflies of stage S >= 1 with preloaded table factors.
template<class P, int S, class T, int E>
__device__ __forceinline__ void stage_apply_tw(cpx<T> (&v)[E], const cpx<T>* f) {
    constexpr int RB = P::rbits(S);
    constexpr int R  = 1 << RB;
    constexpr int Q  = stw_q(RB);
    constexpr int G  = E / R;
    static_for<G>([&](auto gc) {
        constexpr int g = decltype(gc)::value;
        cpx<T>        a[R];
        a[0] = v[g];
        static_for<R - 1>([&](auto jc) {
            constexpr int j = decltype(jc)::value + 1;
            a[j]            = cmul(v[g + j * G], stw_factor<RB, j>(f + g * Q));
        });
        dft<R, 1, 0>(a);
        static_for<R>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            v[g + j * G]    = a[j];
        });
    });
}

template<class P, int S, class T, int E>
__device__ __forceinline__ void stage_compute_tab(cpx<T> (&v)[E], int t, const cpx<T>* __restrict__ stw) {
    constexpr int NSB = P::nsbits(S);
    if constexpr (NSB > 0) {
        cpx<T> f[(E >> P::rbits(S)) * stw_q(P::rbits(S))];
        load_stage_tw<P, S>(f, t, stw);
        stage_apply_tw<P, S>(v, f);
    } else {
        constexpr int R = 1 << P::rbits(S);
        constexpr int G = E / R;
        static_for<G>([&](auto gc) {
            constexpr int g = decltype(gc)::value;
            cpx<T>        a[R];
            static_for<R>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                a[j]            = v[g + j * G];
            });
            dft<R, 1, 0>(a);
            static_for<R>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                v[g + j * G]    = a[j];
            });
        });
    }
}

// Exchange-buffer index with the padding (one slot per 16) split into a
// per-thread base and compile-time offsets.  Valid when the low four bits of
// base plus those of the offset do not carry (true for every Stockham access
// pattern here: offsets are multiples of 16, or the base is).
__device__ __forceinline__ int pad16(int l) { return l + (l >> 4); }

// Barrier of the threads that share the exchange buffer: the whole block
// (BARN = 0), the warp (BARN < 0: each transform's threads and exchange rows
// stay inside one warp) or named barrier 1 over the first BARN threads (the
// compute warps of a block that also has a copy warp).
template<int BARN>
__device__ __forceinline__ void xch_sync() {
    if constexpr (BARN == 0) {
        __syncthreads();
    } else if constexpr (BARN < 0) {
        __syncwarp();
    } else {
        asm volatile("bar.sync 1, %0;" ::"n"(BARN) : "memory");
    }
}

// Stages 1..NST-1 through the exchange buffer.  SH: the stage tables are in
// shared memory, and each stage's factors are loaded after the exchange
// (short latency, registers stay free); global tables are requested before
// the exchange barriers so their latency overlaps them.
template<class P, class X, bool SH = false, int BARN = 0, class T, int E>
__device__ __forceinline__ void run_stages_tab(cpx<T> (&v)[E], cpx<T>* xch, int m, int t,
                                               const cpx<T>* __restrict__ stw) {
    static_for<P::NST - 1>([&](auto sc) {
        constexpr int S  = decltype(sc)::value;
        constexpr int G  = E / (1 << P::rbits(S));
        constexpr int RB = P::rbits(S + 1);
        cpx<T>        f[(E >> RB) * stw_q(RB)];
        if constexpr (!SH) load_stage_tw<P, S + 1, SH>(f, t, stw);
        xch_sync<BARN>();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int g = i % G, j = i / G;
            xch[X::idx(m, stage_out_index<P, S>(t, g, j))] = v[i];
        });
        xch_sync<BARN>();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = xch[X::idx(m, t + i * P::TT)];
        });
        if constexpr (SH) load_stage_tw<P, S + 1, SH>(f, t, stw);
        stage_apply_tw<P, S + 1>(v, f);
    });
}

// Copy a stage table into shared memory (16-byte units; the caller syncs).
template<class P, class T>
__device__ __forceinline__ void stage_tw_to_smem(cpx<T>* dst, const void* src, int tid, int nt) {
    constexpr int U = stage_tw_size<P>() * (int)sizeof(cpx<T>) / 16;
    static_assert((stage_tw_size<P>() * (int)sizeof(cpx<T>)) % 16 == 0, "table in 16-byte units");
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4*       d = reinterpret_cast<uint4*>(dst);
    for (int i = tid; i < U; i += nt) d[i] = __ldg(s + i);
}
template<class P, class T>
__host__ __device__ constexpr int stage_tw_smem_bytes() {
    return stage_tw_size<P>() * (int)sizeof(cpx<T>);
}

// Whether a kernel whose own shared memory is `base` bytes (MINB resident CTAs
// per SM wanted) can also hold a `tab`-byte stage table without losing
// residency: 228 KB per SM, 227 KB per CTA, 1 KB reserved per CTA.
__host__ __device__ constexpr int smem_align16(int b) { return (b + 15) & ~15; }
__host__ __device__ constexpr bool stw_fits(int base, int tab, int minb) {
    const int per   = smem_align16(base) + 1024 + 256;
    int       ctas  = 233472 / per;
    ctas            = ctas < minb ? ctas : minb;
    ctas            = ctas < 1 ? 1 : ctas;
    const int total = smem_align16(base) + tab;
    return total <= 232448 && ctas * (total + 1024 + 256) <= 233472;
}

// b^i for i = 0..15 by repeated squaring (at most five products deep).
template<class T>
__device__ __forceinline__ void powers16(cpx<T> b, cpx<T> (&p)[16]) {
    p[0] = {T(1), T(0)};
    p[1] = b;
    p[2] = cmul(b, b);
    p[3] = cmul(p[2], b);
    p[4] = cmul(p[2], p[2]);
    p[5] = cmul(p[4], b);
    p[6] = cmul(p[4], p[2]);
    p[7] = cmul(p[4], p[3]);
    p[8] = cmul(p[4], p[4]);
    static_for<7>([&](auto ic) {
        constexpr int i = decltype(ic)::value + 1;
        p[8 + i]        = cmul(p[8], p[i]);
    });
}

// out(i, v[i] * base * u^i) for i < E (E a multiple of 4), with u^i formed as
// u^(4a) * u^b from short product chains (u^4a: a products of u^4; then at
// most two more), so only a few complex values are live at a time.
template<int E, class T, class F>
__device__ __forceinline__ void apply_fourstep_tw(const cpx<T> (&v)[E], cpx<T> base, cpx<T> u, F&& out) {
    static_assert(E % 4 == 0, "groups of four");
    const cpx<T> u2 = cmul(u, u);
    const cpx<T> u4 = cmul(u2, u2);
    cpx<T>       wa = base;
    static_for<E / 4>([&](auto ac) {
        constexpr int a  = decltype(ac)::value * 4;
        const cpx<T>  w1 = cmul(wa, u);
        out(std::integral_constant<int, a>{}, cmul(v[a], wa));
        out(std::integral_constant<int, a + 1>{}, cmul(v[a + 1], w1));
        out(std::integral_constant<int, a + 2>{}, cmul(v[a + 2], cmul(wa, u2)));
        out(std::integral_constant<int, a + 3>{}, cmul(v[a + 3], cmul(w1, u2)));
        if constexpr (a + 4 < E) wa = cmul(wa, u4);
    });
}

// Exchange layout for groups of G8 transforms side by side (element-major
// inside a group), groups one after another.
template<int L, int M, int G8>
struct xch_grouped {
    static constexpr int LP   = L + (L >= 16 ? L / 16 : 0);
    static constexpr int size = M * LP;
    __device__ static __forceinline__ int idx(int m, int l) {
        const int pl = l + (L >= 16 ? (l >> 4) : 0);
        return ((m / G8) * LP + pl) * G8 + (m % G8);
    }
};

template<int LP>
__device__ __forceinline__ int pk(int i) {
    return ((i >> LP) << (LP + 1)) | (i & ((1 << LP) - 1));
}

struct v2_args {
    const void* src;
    void*       dst;
    long long   src_stride;    // reals between rows (transforms)
    long long   dst_stride;
    long long   batch;         // rows (transforms) in this launch
    int         conj_in;
    int         conj_out;
    double      scale;
    const void* stw;           // stage twiddles of the sub-transform
    const void* tw_hi;         // four-step twiddle, two-level W_N^e
    const void* tw_lo;
    const void* tw_b;          // W_{16*N2}^m, m < 16*N2
};

// ---------------------------------------------------------------------------
// Single-pass, natural order, N = 2^LOGL (128 <= N <= 4096), pack 2^LP.
template<class T, int LOGL, int LP, int NT>
__global__ void __launch_bounds__(NT) k_single2(v2_args a) {
    using P          = splan<LOGL>;
    constexpr int L  = P::L;
    constexpr int E  = P::E;
    constexpr int TT = P::TT;
    constexpr int M  = NT / TT;
    constexpr int PK = 1 << LP;
    static_assert(TT % PK == 0, "pack must divide threads per row");
    using X = xch_blocked<L, M>;
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<T>*       xch = reinterpret_cast<cpx<T>*>(smem);
    const auto*   stw = reinterpret_cast<const cpx<T>*>(a.stw);
    const int     tid = threadIdx.x;
    const int     m   = tid / TT;
    const int     t   = tid - m * TT;
    const long long row = (long long)blockIdx.x * M + m;
    const bool    live  = row < a.batch;
    const T*      src = reinterpret_cast<const T*>(a.src) + (live ? row : 0) * a.src_stride + pk<LP>(t);
    T*            dst = reinterpret_cast<T*>(a.dst) + row * a.dst_stride + pk<LP>(t);

    cpx<T> v[E];
    static_for<E>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const T       re = src[2 * i * TT], im = src[2 * i * TT + PK];
        v[i]           = {re, a.conj_in ? -im : im};
    });
    stage_compute_tab<P, 0>(v, t, stw);
    run_stages_tab<P, X>(v, xch, m, t, stw);
    if (live) {
        const T sc  = T(a.scale);
        const T sim = a.conj_out ? -sc : sc;
        static_for<E>([&](auto ic) {
            constexpr int i   = decltype(ic)::value;
            dst[2 * i * TT]      = v[i].re * sc;
            dst[2 * i * TT + PK] = v[i].im * sim;
        });
    }
}

// ---------------------------------------------------------------------------
// Four-step column pass: C columns n2 = c0..c0+C-1 of N1 = 2^LOGN1 rows,
// packed natural input (pack 2^LP) -> interleaved scratch rows [k1][n2],
// with the twiddle W_N^(k1*n2).  Persistent over the launch's tiles.
template<class T, int LOGN1, int LOGN2, int LP, int C, int NT>
__global__ void __launch_bounds__(NT, 2) k_col2(v2_args a) {
    using P           = splan<LOGN1>;
    constexpr int N1  = P::L;
    constexpr int N2  = 1 << LOGN2;
    constexpr int E   = P::E;
    constexpr int TT  = P::TT;
    constexpr int PK  = 1 << LP;
    constexpr int TPR = N2 / C;    // tiles per transform
    static_assert(NT == C * TT, "threads");
    static_assert(C % PK == 0, "pack must divide the column group");
    using X = xch_interleaved<N1, C>;
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<T>*     xch = reinterpret_cast<cpx<T>*>(smem);
    const auto* stw = reinterpret_cast<const cpx<T>*>(a.stw);
    const auto* thi = reinterpret_cast<const cpx<T>*>(a.tw_hi);
    const auto* tlo = reinterpret_cast<const cpx<T>*>(a.tw_lo);
    const auto* tb  = reinterpret_cast<const cpx<T>*>(a.tw_b);
    const int   tid = threadIdx.x;
    const int   c   = tid % C;
    const int   t   = tid / C;
    const long long tiles = a.batch * TPR;

    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long row = tile / TPR;
        const int       c0  = (int)(tile - row * TPR) * C;
        const int       n2  = c0 + c;
        const T* src = reinterpret_cast<const T*>(a.src) + row * a.src_stride + pk<LP>(t * N2 + n2);
        cpx<T>   v[E];
        static_for<E>([&](auto ic) {
            constexpr int i  = decltype(ic)::value;
            const T       re = src[2 * i * TT * N2], im = src[2 * i * TT * N2 + PK];
            v[i]            = {re, a.conj_in ? -im : im};
        });
        stage_compute_tab<P, 0>(v, t, stw);
        run_stages_tab<P, X>(v, xch, c, t, stw);
        // v[i] = column spectrum at k1 = t + i*TT; twiddle W_N^(k1*n2)
        const uint32_t e0   = (uint32_t)t * (uint32_t)n2;
        const cpx<T>   base = cmul(ldg_cpx(thi + (e0 >> LOGN2)), ldg_cpx(tlo + (e0 & (N2 - 1))));
        cpx<T>         bp[16];
        powers16(ldg_cpx(tb + n2), bp);
        cpx<T>*        dst  = reinterpret_cast<cpx<T>*>(a.dst) + row * (a.dst_stride / 2) + (long long)t * N2 + n2;
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            cpx<T>        w = base;
            if constexpr (i > 0) w = cmul(base, bp[i]);
            dst[(long long)i * TT * N2] = cmul(v[i], w);
        });
    }
}

// ---------------------------------------------------------------------------
// Four-step row pass: CR rows k1 = r0..r0+CR-1 of N2 = 2^LOGN2 interleaved
// scratch elements -> natural packed output X[k2*N1 + k1] (pack 2^LP).
// Threads: G8 rows fastest (one 64-byte output segment per k2), then t.
template<class T, int LOGN1, int LOGN2, int LP, int CR, int G8, int NT>
__global__ void __launch_bounds__(NT, 2) k_row2(v2_args a) {
    using P           = splan<LOGN2>;
    constexpr int N1  = 1 << LOGN1;
    constexpr int N2  = P::L;
    constexpr int E   = P::E;
    constexpr int TT  = P::TT;
    constexpr int PK  = 1 << LP;
    constexpr int TPR = N1 / CR;
    static_assert(NT == CR * TT, "threads");
    static_assert(CR % G8 == 0 && G8 % PK == 0, "row grouping");
    using X = xch_grouped<N2, CR, G8>;
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<T>*     xch = reinterpret_cast<cpx<T>*>(smem);
    const auto* stw = reinterpret_cast<const cpx<T>*>(a.stw);
    const int   tid = threadIdx.x;
    const int   mlo = tid % G8;
    const int   t   = (tid / G8) % TT;
    const int   mhi = tid / (G8 * TT);
    const int   m   = mhi * G8 + mlo;
    const long long tiles = a.batch * TPR;

    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long row = tile / TPR;
        const int       r0  = (int)(tile - row * TPR) * CR;
        const int       k1  = r0 + m;
        const cpx<T>*   src = reinterpret_cast<const cpx<T>*>(a.src) + row * (a.src_stride / 2) + (long long)k1 * N2 + t;
        cpx<T>          v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = src[i * TT];
        });
        stage_compute_tab<P, 0>(v, t, stw);
        run_stages_tab<P, X>(v, xch, m, t, stw);
        // v[i] = X[k2*N1 + k1], k2 = t + i*TT
        T*      dst = reinterpret_cast<T*>(a.dst) + row * a.dst_stride + pk<LP>(t * N1 + k1);
        const T sc  = T(a.scale);
        const T sim = a.conj_out ? -sc : sc;
        static_for<E>([&](auto ic) {
            constexpr int i              = decltype(ic)::value;
            dst[2 * i * TT * N1]         = v[i].re * sc;
            dst[2 * i * TT * N1 + PK]    = v[i].im * sim;
        });
    }
}

}    // namespace pcxg

// ===========================================================================
// TMA-fed single pass.  Persistent CTAs; each tile (M rows) is brought into
// shared memory by one-dimensional bulk copies through a two-stage ring, so
// the next tiles are in flight while this one is transformed.  Stage 0 reads
// the packed rows from shared memory (any input order), the last stage
// writes packed rows into a staging area (any output order) that the threads
// copy out with 16-byte stores.  Rows are padded in shared memory so that
// the rows of one warp fall into different banks.
namespace pcxg {

struct v3_args {
    const void* src;
    void*       dst;
    long long   src_stride;
    long long   dst_stride;
    long long   batch;
    int         conj_in;
    int         conj_out;
    int         order_in;
    int         order_out;
    double      scale;
    const void* stw;
    int*        error;    // set when a bounded wait gives up
};

// Read (re, im) stored `pk_off` reals apart at `o`; lanes with bit SW set
// fetch the imaginary part first, so the two halves of each shared-memory
// wavefront hit disjoint banks.
template<class T, int SW>
__device__ __forceinline__ cpx<T> lds_swapped(const T* base, int o, int pk_off) {
    const bool sw = (threadIdx.x & SW) != 0;
    const T    x0 = base[o + (sw ? pk_off : 0)];
    const T    x1 = base[o + (sw ? 0 : pk_off)];
    return {sw ? x1 : x0, sw ? x0 : x1};
}
// The matching store.
template<class T, int SW>
__device__ __forceinline__ void sts_swapped(T* base, int o, int pk_off, T re, T im) {
    const bool sw        = (threadIdx.x & SW) != 0;
    base[o + (sw ? pk_off : 0)] = sw ? im : re;
    base[o + (sw ? 0 : pk_off)] = sw ? re : im;
}

template<int TT>
__host__ __device__ constexpr int single3_pad() {
    return TT >= 32 ? 0 : (TT >= 8 ? 8 : 4);
}
// Resident CTAs per SM a single-pass launch is built for (registers: 128 per
// thread either way).
__host__ __device__ constexpr int single3_minb(int nt) { return nt >= 512 ? 1 : 2; }
template<class T, int LOGL, int NT>
__host__ __device__ constexpr int single3_base_smem() {
    using P          = splan<LOGL>;
    constexpr int M  = NT / P::TT;
    constexpr int RS = 2 * P::L + single3_pad<P::TT>();
    return 2 * M * RS * (int)sizeof(T) + xch_blocked<P::L, M>::size * (int)sizeof(cpx<T>);
}
template<class T, int LOGL, int NT>
__host__ __device__ constexpr bool single3_tws() {
    return stw_fits(single3_base_smem<T, LOGL, NT>(), stage_tw_smem_bytes<splan<LOGL>, T>(), single3_minb(NT));
}
template<class T, int LOGL, int NT>
__host__ __device__ constexpr int single3_smem() {
    return single3_tws<T, LOGL, NT>()
               ? smem_align16(single3_base_smem<T, LOGL, NT>()) + stage_tw_smem_bytes<splan<LOGL>, T>()
               : single3_base_smem<T, LOGL, NT>();
}

template<class T, int LOGL, int LP, int NT>
__global__ void __launch_bounds__(NT, single3_minb(NT)) k_single3(v3_args a) {
    using P             = splan<LOGL>;
    constexpr int L     = P::L;
    constexpr int E     = P::E;
    constexpr int TT    = P::TT;
    constexpr int M     = NT / TT;
    constexpr int PK    = 1 << LP;
    constexpr int PADR  = single3_pad<TT>();
    constexpr int RS    = 2 * L + PADR;    // shared-memory row stride (reals)
    constexpr int TILE  = M * RS;
    constexpr int ROWB  = 2 * L * (int)sizeof(T);
    constexpr int V     = 16 / (int)sizeof(T);
    // a warp inside one row: its two halves read reals / imaginaries on
    // disjoint banks by swapping the order in half of the lanes (rows of fewer
    // than 32 threads keep the plain order: their rows are padded instead)
    constexpr int SW    = TT >= 32 ? (sizeof(T) == 8 ? 8 : 16) : 0;
    using X             = xch_blocked<L, M>;
    static_assert(X::size * 2 >= TILE, "staging fits the exchange buffer");
    static_assert((RS * (int)sizeof(T)) % 16 == 0, "rows stay 16-byte aligned");
    extern __shared__ __align__(128) unsigned char smem[];
    T*               in0 = reinterpret_cast<T*>(smem);
    cpx<T>*          xch = reinterpret_cast<cpx<T>*>(in0 + 2 * TILE);
    T*               stg = reinterpret_cast<T*>(xch);
    __shared__ uint64_t full[2];
    constexpr bool   SH  = single3_tws<T, LOGL, NT>();
    cpx<T>*          tws = reinterpret_cast<cpx<T>*>(smem + smem_align16(single3_base_smem<T, LOGL, NT>()));
    const auto*      stw = SH ? tws : reinterpret_cast<const cpx<T>*>(a.stw);
    const T*         src = reinterpret_cast<const T*>(a.src);
    T*               dst = reinterpret_cast<T*>(a.dst);
    const int        tid = threadIdx.x;
    const int        m   = tid / TT;
    const int        t   = tid - m * TT;
    const long long  ntile = (a.batch + M - 1) / M;
    const bool       contig_in  = PADR == 0 && a.src_stride == 2 * L;
    const bool       contig_out = PADR == 0 && a.dst_stride == 2 * L;

    if constexpr (SH) stage_tw_to_smem<P, T>(tws, a.stw, tid, NT);
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](long long tile, int s) {    // thread 0 only
        const int  rows = (int)min((long long)M, a.batch - tile * M);
        T*         buf  = in0 + s * TILE;
        const T*   g    = src + tile * M * a.src_stride;
        mbar_arrive_expect_tx(&full[s], (uint32_t)rows * ROWB);
        if (contig_in) {
            bulk_g2s(buf, g, (uint32_t)rows * ROWB, &full[s]);
        } else {
            for (int r = 0; r < rows; ++r) bulk_g2s(buf + r * RS, g + r * a.src_stride, ROWB, &full[s]);
        }
    };
    if (tid == 0) {
        if ((long long)blockIdx.x < ntile) issue(blockIdx.x, 0);
        if ((long long)blockIdx.x + gridDim.x < ntile) issue(blockIdx.x + gridDim.x, 1);
    }

    long long k = 0;
    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x, ++k) {
        const int      s   = (int)(k & 1);
        const uint32_t par = (uint32_t)((k >> 1) & 1);
        const bool     ok  = mbar_wait_bounded(&full[s], par);
        if (__syncthreads_or(!ok)) {
            // give up: record it, let the other stage's copy land, leave together
            if (tid == 0) {
                atomicExch(a.error, 1);
                mbar_wait_bounded(&full[s], par, 100000000ull);
                mbar_wait_bounded(&full[s ^ 1], par ^ (s ? 1u : 0u), 100000000ull);
            }
            __syncthreads();
            return;
        }
        const T* in = in0 + s * TILE;
        cpx<T>   v[E];
        static_for<E>([&](auto ic) {
            constexpr int  i  = decltype(ic)::value;
            const uint32_t p  = order_pos(t + i * TT, a.order_in, LOGL);
            const int      o  = m * RS + pk<LP>((int)p);
            const cpx<T>   x  = lds_swapped<T, SW>(in, o, PK);    // halves of a warp on disjoint banks
            v[i]              = {x.re, a.conj_in ? -x.im : x.im};
        });
        fence_proxy_async_smem();
        __syncthreads();    // stage s consumed: refill it with the tile after next
        if (tid == 0 && tile + 2 * (long long)gridDim.x < ntile) issue(tile + 2 * (long long)gridDim.x, s);
        stage_compute_tab<P, 0>(v, t, stw);
        // a transform's TT <= 32 threads share one warp and its own exchange
        // block: its exchanges need only that warp's barrier (the block-wide
        // barriers before and after them order the stage and staging reuse)
        run_stages_tab<P, X, SH, (TT <= 32 ? -1 : 0)>(v, xch, m, t, stw);
        __syncthreads();    // exchange reads done: reuse the buffer as staging
        {
            constexpr int S   = P::NST - 1;
            constexpr int G   = E / (1 << P::rbits(S));
            const T       sc  = T(a.scale);
            const T       sim = a.conj_out ? -sc : sc;
            static_for<E>([&](auto ic) {
                constexpr int  i = decltype(ic)::value;
                constexpr int  g = i % G, j = i / G;
                const uint32_t kf = stage_out_index<P, S>(t, g, j);
                const int      o  = m * RS + pk<LP>((int)order_pos(kf, a.order_out, LOGL));
                sts_swapped<T, SW>(stg, o, PK, v[i].re * sc, v[i].im * sim);
            });
        }
        __syncthreads();
        const int rows = (int)min((long long)M, a.batch - tile * M);
        T*        d    = dst + tile * M * a.dst_stride;
        if (contig_out) {
            for (int q = tid; q < rows * (2 * L / V); q += NT) {
                *reinterpret_cast<float4*>(d + q * V) = *reinterpret_cast<const float4*>(stg + q * V);
            }
        } else {
            for (int q = tid; q < rows * (2 * L / V); q += NT) {
                const int r = q / (2 * L / V), c = (q - r * (2 * L / V)) * V;
                *reinterpret_cast<float4*>(d + r * a.dst_stride + c) = *reinterpret_cast<const float4*>(stg + r * RS + c);
            }
        }
    }
}

}    // namespace pcxg

namespace pcxg {

// Copy a table of BYTES bytes into shared memory (16-byte units; the caller syncs).
template<int BYTES, class T>
__device__ __forceinline__ void copy_table_to_smem(cpx<T>* dst, const void* src, int tid, int nt) {
    static_assert(BYTES % 16 == 0, "table in 16-byte units");
    const uint4* sp = reinterpret_cast<const uint4*>(src);
    uint4*       dp = reinterpret_cast<uint4*>(dst);
    for (int i = tid; i < BYTES / 16; i += nt) dp[i] = __ldg(sp + i);
}

// ---- full stage tables of the sub-transforms -------------------------------
// For stage S >= 1 of splan P (Ns = 2^nsbits(S) butterfly positions, radix R)
// position k keeps all R entries W^(j*k), j = 0..R-1, W = W_{Ns*R} (entry 0 is
// 1), generated in FP64 and rounded once.  A butterfly then multiplies each
// input by its table entry, where the factor tables of pcx_fft_v2.cuh form
// nine of the fifteen radix-16 twiddles as products of two entries (36 more
// FP32 instructions per butterfly).  For the sub-transforms of the four-step
// (64..1024 points) a full table is 1-15 KB.  Each position's row of 4 or more
// entries is padded by 16 bytes: the threads of a warp read up to eight
// positions at once, and with power-of-two rows of 32 bytes or more those
// would share banks.  Radix-2 rows (16 bytes in FP32) are not padded: eight
// neighbouring positions fill 128 contiguous bytes.
__host__ __device__ constexpr int full_tw_row(int rb) { return (1 << rb) + (rb == 1 ? 0 : 2); }
template<class P>
__host__ __device__ constexpr int fs_full_tw_offset(int S) {
    int off = 0;
    for (int s = 1; s < S; ++s) off += (1 << P::nsbits(s)) * full_tw_row(P::rbits(s));
    return off;
}
template<class P>
__host__ __device__ constexpr int fs_full_tw_size() {
    return fs_full_tw_offset<P>(P::NST);
}

template<class T>
__global__ void k_full_twiddles(cpx<T>* out, int ns, int rb, int log_nsr) {
    const int row = full_tw_row(rb);
    const int q   = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns * row) return;
    const int k = q / row, j = q - k * row;
    if (j >= (1 << rb)) {
        out[q] = {T(0), T(0)};    // padding
        return;
    }
    const long long e = (long long)k * j;
    double          sn, cs;
    sincospi(2.0 * (double)e / (double)(1LL << log_nsr), &sn, &cs);
    out[q] = {T(cs), T(-sn)};
}

// Whether the full table of splan PL serves splan P as well: the same stages
// with the same butterfly positions, only the last stage's radix of PL may be
// larger.  Position k of P's last stage (radix R) then needs W_{Ns*R}^(j*k) =
// entry j*D of PL's row k, D = R_PL / R.
template<class P, class PL>
__host__ __device__ constexpr bool full_tab_serves() {
    if (P::NST != PL::NST) return false;
    for (int s = 0; s < P::NST; ++s) {
        if (P::nsbits(s) != PL::nsbits(s)) return false;
        if (s + 1 < P::NST ? P::rbits(s) != PL::rbits(s) : P::rbits(s) > PL::rbits(s)) return false;
    }
    return true;
}

// Butterflies of stage S >= 1 with the full table `tab` of splan PT (P's own,
// or a larger sub-transform's that serves P: full_tab_serves).
template<class P, int S, bool SH, class PT = P, class T, int E>
__device__ __forceinline__ void stage_apply_full(cpx<T> (&v)[E], int t, const cpx<T>* __restrict__ tab) {
    static_assert(full_tab_serves<P, PT>(), "table of another stage structure");
    constexpr int RB  = P::rbits(S);
    constexpr int R   = 1 << RB;
    constexpr int NSB = P::nsbits(S);
    constexpr int G   = E / R;
    constexpr int D   = 1 << (PT::rbits(S) - RB);    // column step in PT's rows
    static_for<G>([&](auto gc) {
        constexpr int g  = decltype(gc)::value;
        const int     k  = (t + g * P::TT) & ((1 << NSB) - 1);
        const cpx<T>* tw = tab + fs_full_tw_offset<PT>(S) + k * full_tw_row(PT::rbits(S));
        cpx<T>        a[R];
        static_for<R / 2>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            cpx<T>        w0, w1;
            if constexpr (D == 1) {
                ld2<SH>(tw + 2 * q, w0, w1);
            } else {
                if constexpr (q > 0) w0 = SH ? tw[2 * q * D] : ldg_cpx(tw + 2 * q * D);
                w1 = SH ? tw[(2 * q + 1) * D] : ldg_cpx(tw + (2 * q + 1) * D);
            }
            a[2 * q]     = q == 0 ? v[g] : cmul(v[g + 2 * q * G], w0);
            a[2 * q + 1] = cmul(v[g + (2 * q + 1) * G], w1);
        });
        dft<R, 1, 0>(a);
        static_for<R>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            v[g + j * G]    = a[j];
        });
    });
}

// Barrier 1 over the NT compute threads that also ORs `bad` across them.
template<int NT>
__device__ __forceinline__ bool bar1_any(bool bad) {
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((uint32_t)bad), "n"(NT)
                 : "memory");
    return r != 0;
}

// Stages 1..NST-1 through the exchange buffer with the full tables; the
// barriers are xch_sync<BARN>.  With a named barrier (BARN > 0: the NT = BARN
// compute threads of a block that also has a copy warp) the first exchange's
// opening barrier doubles as the give-up vote: it returns true, before
// anything is written, when any of those threads passes `bad`, so all of them
// leave at the same point without a barrier of its own.  With BARN <= 0 `bad`
// is ignored and the result is false.
template<class P, class X, bool SH, int BARN, class PT = P, class T, int E>
__device__ __forceinline__ bool run_stages_full(cpx<T> (&v)[E], cpx<T>* xch, int m, int t,
                                                const cpx<T>* __restrict__ tab, bool bad = false) {
    bool abort = false;
    static_for<P::NST - 1>([&](auto sc) {
        constexpr int S = decltype(sc)::value;
        constexpr int G = E / (1 << P::rbits(S));
        if (abort) return;
        if constexpr (S == 0 && BARN > 0) {
            if (bar1_any<BARN>(bad)) {
                abort = true;
                return;
            }
        } else {
            xch_sync<BARN>();
        }
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int g = i % G, j = i / G;
            xch[X::idx(m, stage_out_index<P, S>(t, g, j))] = v[i];
        });
        xch_sync<BARN>();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = xch[X::idx(m, t + i * P::TT)];
        });
        stage_apply_full<P, S + 1, SH, PT>(v, t, tab);
    });
    return abort;
}

// ===========================================================================
// TMA-fed four-step passes.  Same arithmetic as k_col2 / k_row2; the input
// tiles arrive in shared memory through a two-stage bulk-copy ring
// (column pass: 3-D tensor copies of N1 x 64-byte row segments; row pass:
// one bulk copy per scratch row into padded rows), outputs are written from
// registers as in the direct kernels.

__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// The same copy with an L2 eviction-priority hint (an L2::evict_first policy
// for data read once, so it does not push the four-step scratch out of L2).
__device__ __forceinline__ void tma_load_3d_hint(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar,
                                                 uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(
            smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Drop a 128-byte line from L2 without writing it back (its data are dead).
__device__ __forceinline__ void l2_discard(const void* p) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

struct v3_pass_args {
    v2_args   base;
    long long row0;    // first batch row of this launch in the tensor map (column pass)
    int*      error;
};

template<class T, int LOGN1>
__host__ __device__ constexpr int col3_boxy() {
    return (1 << LOGN1) < 256 ? (1 << LOGN1) : 256;
}

template<class T, int LOGN1, int C>
__host__ __device__ constexpr int col3_base_smem() {
    return 2 * (1 << LOGN1) * 2 * C * (int)sizeof(T) + xch_interleaved<(1 << LOGN1), C>::size * (int)sizeof(cpx<T>);
}
// Full stage table bytes of an L = 2^LOGL point sub-transform.
template<class T, int LOGL>
__host__ __device__ constexpr int full_tw_bytes() {
    return fs_full_tw_size<splan<LOGL>>() * (int)sizeof(cpx<T>);
}
template<class T, int LOGN1, int C>
__host__ __device__ constexpr bool col3_tws() {
    return stw_fits(col3_base_smem<T, LOGN1, C>(), full_tw_bytes<T, LOGN1>(), 1);
}
template<class T, int LOGN1, int C>
__host__ __device__ constexpr int col3_smem() {
    return col3_tws<T, LOGN1, C>() ? smem_align16(col3_base_smem<T, LOGN1, C>()) + full_tw_bytes<T, LOGN1>()
                                   : col3_base_smem<T, LOGN1, C>();
}

template<class T, int LOGN1, int LOGN2, int LP, int C, int NT>
__global__ void __launch_bounds__(NT, 1) k_col3(const __grid_constant__ CUtensorMap tmap, v3_pass_args pa) {
    using P            = splan<LOGN1>;
    constexpr int N1   = P::L;
    constexpr int N2   = 1 << LOGN2;
    constexpr int E    = P::E;
    constexpr int TT   = P::TT;
    constexpr int PK   = 1 << LP;
    constexpr int TPR  = N2 / C;
    constexpr int SEG  = 2 * C;                // reals per row segment
    constexpr int TILE = N1 * SEG;             // reals per stage
    constexpr int BOXY = col3_boxy<T, LOGN1>();
    constexpr int SW   = sizeof(T) == 8 ? 8 : 16;
    static_assert(NT == C * TT, "threads");
    using X = xch_interleaved<N1, C>;
    extern __shared__ __align__(128) unsigned char smem[];
    T*                  in0 = reinterpret_cast<T*>(smem);
    cpx<T>*             xch = reinterpret_cast<cpx<T>*>(in0 + 2 * TILE);
    __shared__ uint64_t full[2];
    const v2_args&      a   = pa.base;
    constexpr bool      SH  = col3_tws<T, LOGN1, C>();
    cpx<T>*             tws = reinterpret_cast<cpx<T>*>(smem + smem_align16(col3_base_smem<T, LOGN1, C>()));
    const auto*         stw = SH ? tws : reinterpret_cast<const cpx<T>*>(a.stw);
    const auto*         thi = reinterpret_cast<const cpx<T>*>(a.tw_hi);
    const auto*         tlo = reinterpret_cast<const cpx<T>*>(a.tw_lo);
    const auto*         tb  = reinterpret_cast<const cpx<T>*>(a.tw_b);
    const int           tid = threadIdx.x;
    const int           c   = tid % C;
    const int           t   = tid / C;
    const long long     tiles = a.batch * TPR;

    if constexpr (SH) copy_table_to_smem<full_tw_bytes<T, LOGN1>()>(tws, a.stw, tid, NT);
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    auto issue = [&](long long tile, int s) {
        const long long row = tile / TPR;
        const int       c0  = (int)(tile - row * TPR) * C;
        T*              buf = in0 + s * TILE;
        mbar_arrive_expect_tx(&full[s], TILE * (int)sizeof(T));
        const uint64_t pol = l2_evict_first_policy();
#pragma unroll
        for (int y = 0; y < N1; y += BOXY) {
            tma_load_3d_hint(buf + y * SEG, &tmap, 2 * c0, y, (int)(pa.row0 + row), &full[s], pol);
        }
    };
    if (tid == 0) {
        if ((long long)blockIdx.x < tiles) issue(blockIdx.x, 0);
        if ((long long)blockIdx.x + gridDim.x < tiles) issue(blockIdx.x + gridDim.x, 1);
    }
    long long k = 0;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
        const int      s   = (int)(k & 1);
        const uint32_t par = (uint32_t)((k >> 1) & 1);
        const bool     ok  = mbar_wait_bounded(&full[s], par);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(pa.error, 1);
                mbar_wait_bounded(&full[s], par, 100000000ull);
                mbar_wait_bounded(&full[s ^ 1], par ^ (s ? 1u : 0u), 100000000ull);
            }
            __syncthreads();
            return;
        }
        const long long row = tile / TPR;
        const int       c0  = (int)(tile - row * TPR) * C;
        const int       n2  = c0 + c;
        const T*        in  = in0 + s * TILE;
        cpx<T>          v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            cpx<T>        x = lds_swapped<T, SW>(in, (t + i * TT) * SEG + pk<LP>(c), PK);
            v[i]            = {x.re, a.conj_in ? -x.im : x.im};
        });
        fence_proxy_async_smem();
        __syncthreads();    // stage s consumed: refill it with the tile after next
        if (tid == 0 && tile + 2 * (long long)gridDim.x < tiles) issue(tile + 2 * (long long)gridDim.x, s);
        // four-step twiddle inputs: requested now, used after the stages
        const uint32_t e0 = (uint32_t)t * (uint32_t)n2;
        const cpx<T>   th = ldg_cpx(thi + (e0 >> LOGN2));
        const cpx<T>   tl = ldg_cpx(tlo + (e0 & (N2 - 1)));
        const cpx<T>   tu = ldg_cpx(tb + n2);
        stage_compute_tab<P, 0>(v, t, stw);
        run_stages_full<P, X, SH, 0>(v, xch, c, t, stw);
        cpx<T>* dst = reinterpret_cast<cpx<T>*>(a.dst) + row * (a.dst_stride / 2) + (long long)t * N2 + n2;
        apply_fourstep_tw(v, cmul(th, tl), tu, [&](auto ic, cpx<T> o) {
            constexpr int i             = decltype(ic)::value;
            dst[(long long)i * TT * N2] = o;
        });
    }
}



template<class T, int LOGN2, int CR, int G8>
__host__ __device__ constexpr int row3_base_smem() {
    return 2 * CR * ((1 << LOGN2) + 2) * (int)sizeof(cpx<T>) +
           xch_grouped<(1 << LOGN2), CR, G8>::size * (int)sizeof(cpx<T>);
}
template<class T, int LOGN2, int CR, int G8>
__host__ __device__ constexpr bool row3_tws() {
    return stw_fits(row3_base_smem<T, LOGN2, CR, G8>(), full_tw_bytes<T, LOGN2>(), 1);
}
template<class T, int LOGN2, int CR, int G8>
__host__ __device__ constexpr int row3_smem() {
    return row3_tws<T, LOGN2, CR, G8>() ? smem_align16(row3_base_smem<T, LOGN2, CR, G8>()) + full_tw_bytes<T, LOGN2>()
                                        : row3_base_smem<T, LOGN2, CR, G8>();
}

template<class T, int LOGN1, int LOGN2, int LP, int CR, int G8, int NT>
__global__ void __launch_bounds__(NT, 1) k_row3(v3_pass_args pa) {
    using P            = splan<LOGN2>;
    constexpr int N1   = 1 << LOGN1;
    constexpr int N2   = P::L;
    constexpr int E    = P::E;
    constexpr int TT   = P::TT;
    constexpr int PK   = 1 << LP;
    constexpr int TPR  = N1 / CR;
    constexpr int RSI  = N2 + 2;               // padded shared row (complex)
    constexpr int TILE = CR * RSI;             // complex per stage
    constexpr int ROWB = N2 * (int)sizeof(cpx<T>);
    static_assert(NT == CR * TT, "threads");
    using X = xch_grouped<N2, CR, G8>;
    extern __shared__ __align__(128) unsigned char smem[];
    cpx<T>*             in0 = reinterpret_cast<cpx<T>*>(smem);
    cpx<T>*             xch = in0 + 2 * TILE;
    __shared__ uint64_t full[2];
    const v2_args&      a   = pa.base;
    constexpr bool      SH  = row3_tws<T, LOGN2, CR, G8>();
    cpx<T>*             tws = reinterpret_cast<cpx<T>*>(smem + smem_align16(row3_base_smem<T, LOGN2, CR, G8>()));
    const auto*         stw = SH ? tws : reinterpret_cast<const cpx<T>*>(a.stw);
    const int           tid = threadIdx.x;
    const int           mlo = tid % G8;
    const int           t   = (tid / G8) % TT;
    const int           mhi = tid / (G8 * TT);
    const int           m   = mhi * G8 + mlo;
    const long long     tiles = a.batch * TPR;
    const cpx<T>*       src = reinterpret_cast<const cpx<T>*>(a.src);

    if constexpr (SH) copy_table_to_smem<full_tw_bytes<T, LOGN2>()>(tws, a.stw, tid, NT);
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    auto issue = [&](long long tile, int s) {
        const long long row = tile / TPR;
        const int       r0  = (int)(tile - row * TPR) * CR;
        cpx<T>*         buf = in0 + s * TILE;
        const cpx<T>*   g   = src + row * (a.src_stride / 2) + (long long)r0 * N2;
        mbar_arrive_expect_tx(&full[s], CR * ROWB);
        for (int r = 0; r < CR; ++r) bulk_g2s(buf + r * RSI, g + (long long)r * N2, ROWB, &full[s]);
    };
    if (tid == 0) {
        if ((long long)blockIdx.x < tiles) issue(blockIdx.x, 0);
        if ((long long)blockIdx.x + gridDim.x < tiles) issue(blockIdx.x + gridDim.x, 1);
    }
    long long k = 0;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
        const int      s   = (int)(k & 1);
        const uint32_t par = (uint32_t)((k >> 1) & 1);
        const bool     ok  = mbar_wait_bounded(&full[s], par);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(pa.error, 1);
                mbar_wait_bounded(&full[s], par, 100000000ull);
                mbar_wait_bounded(&full[s ^ 1], par ^ (s ? 1u : 0u), 100000000ull);
            }
            __syncthreads();
            return;
        }
        const long long row = tile / TPR;
        const int       r0  = (int)(tile - row * TPR) * CR;
        const int       k1  = r0 + m;
        const cpx<T>*   in  = in0 + s * TILE + m * RSI + t;
        {
            // The tile's rows of four-step scratch have landed in shared memory
            // and are never read again: drop their L2 lines without write-back.
            const char* g = reinterpret_cast<const char*>(src + row * (a.src_stride / 2) + (long long)r0 * N2);
            if ((reinterpret_cast<uintptr_t>(g) & 127) == 0) {
                for (int q = tid; q < CR * ROWB / 128; q += NT) l2_discard(g + (size_t)q * 128);
            }
        }
        cpx<T>          v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = in[i * TT];
        });
        fence_proxy_async_smem();
        __syncthreads();    // stage s consumed: refill it with the tile after next
        if (tid == 0 && tile + 2 * (long long)gridDim.x < tiles) issue(tile + 2 * (long long)gridDim.x, s);
        stage_compute_tab<P, 0>(v, t, stw);
        run_stages_full<P, X, SH, 0>(v, xch, m, t, stw);
        T*      dst = reinterpret_cast<T*>(a.dst) + row * a.dst_stride + pk<LP>(t * N1 + k1);
        const T sc  = T(a.scale);
        const T sim = a.conj_out ? -sc : sc;
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            __stcs(dst + 2 * i * TT * N1, v[i].re * sc);    // streaming: keep L2 for the scratch
            __stcs(dst + 2 * i * TT * N1 + PK, v[i].im * sim);
        });
    }
}


}    // namespace pcxg
