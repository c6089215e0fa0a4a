// Batched power-of-two FFT kernels (forward DFT; inverse by conjugation).
//
//  * k_single  — N <= 4096: one CTA transforms M whole rows held in shared
//                memory (Stockham radix-16 stages, padded exchange buffer).
//  * k_colpass — N >= 8192, pass 1 of a four-step: C columns of the N1 x N2
//                view, FFT along n1, optional inter-pass twiddle W_N^(k1*n2).
//  * k_rowpass — pass 2: CR rows, FFT along n2, written transposed (natural
//                order) or row-permuted (bit_reversed / unordered).
// The intermediate goes through a scratch buffer sized so that one chunk of
// the batch stays resident in L2 between the two passes.
//
// Reference behaviour restated here: forward X[k] = sum x[n] e^{-2 pi i nk/N}
// (fft.hpp:728-750), inverse with optional 1/N (fft.hpp:828-853), orders
// normal / bit_reversed / unordered (fft.hpp:540-544), zero-extension of a
// short source (fft.hpp:759-820, node_along 1759-1795).
#pragma once

#include "pcx_core.cuh"

namespace pcxg {

struct io_args {
    const void* src;
    void*       dst;
    long long   src_stride;    // reals between consecutive rows
    long long   dst_stride;
    long long   batch;         // rows in this launch
    int         src_len;       // valid source elements per row (zero-extended to N)
    int         lp_src;        // log2 pack width of source
    int         lp_dst;
    int         order_in;      // position map of the input  (0 natural)
    int         order_out;     // position map of the output (0 natural)
    int         conj_in;
    int         conj_out;
    double      scale;
};

// Copy `rows` rows of `rowf` reals from global (stride `gstride`) into shared
// memory (stride `sstride`).  When `valid` < row length, reals of elements at
// or past `valid` are zero and never read from global.
template<class T, int NT>
__device__ __forceinline__ void load_rows(T* __restrict__ s, int sstride, const T* __restrict__ g,
                                          long long gstride, int rows, int rowf, int valid, int lp,
                                          bool vec_ok) {
    constexpr int V = 16 / sizeof(T);
    if (vec_ok) {
        const int q_per_row = rowf / V;
        const int total     = rows * q_per_row;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int r = q / q_per_row, c = (q - r * q_per_row) * V;
            const float4 val = __ldg(reinterpret_cast<const float4*>(g + r * gstride + c));
            *reinterpret_cast<float4*>(s + r * sstride + c) = val;
        }
    } else {
        const int total = rows * rowf;
        const int P     = 1 << lp;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int r = q / rowf, f = q - r * rowf;
            const int e = ((f >> (lp + 1)) << lp) | (f & (P - 1));
            s[r * sstride + f] = e < valid ? g[r * gstride + f] : T(0);
        }
    }
}

template<class T, int NT>
__device__ __forceinline__ void store_rows(T* __restrict__ g, long long gstride, const T* __restrict__ s,
                                           int sstride, int rows, int rowf, bool vec_ok) {
    constexpr int V = 16 / sizeof(T);
    if (vec_ok) {
        const int q_per_row = rowf / V;
        const int total     = rows * q_per_row;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int r = q / q_per_row, c = (q - r * q_per_row) * V;
            *reinterpret_cast<float4*>(g + r * gstride + c) =
                *reinterpret_cast<const float4*>(s + r * sstride + c);
        }
    } else {
        const int total = rows * rowf;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int r = q / rowf, f = q - r * rowf;
            g[r * gstride + f] = s[r * sstride + f];
        }
    }
}

// Exchange-buffer layouts (complex units), padded by one slot per 16 so the
// strided Stockham writes do not collide in shared-memory banks.
template<int L, int M>
struct xch_blocked {    // transform m contiguous
    static constexpr int LP   = L + (L >= 16 ? L / 16 : 0);
    static constexpr int size = M * LP;
    __device__ static __forceinline__ int idx(int m, int l) { return m * LP + l + (L >= 16 ? (l >> 4) : 0); }
};
template<int L, int M>
struct xch_interleaved {    // element-major, the M transforms side by side
    static constexpr int LP   = L + (L >= 16 ? L / 16 : 0);
    static constexpr int size = M * LP;
    __device__ static __forceinline__ int idx(int m, int l) { return (l + (L >= 16 ? (l >> 4) : 0)) * M + m; }
};

// Run stages 1..NST-1 through the exchange buffer; on entry v holds stage-0
// outputs, on exit v holds the final outputs of the last stage.
template<class P, class X, class T, int E>
__device__ __forceinline__ void run_stages(cpx<T> (&v)[E], cpx<T>* xch, int m, int t,
                                           const cpx<T>* __restrict__ twL) {
    static_for<P::NST - 1>([&](auto sc) {
        constexpr int S = decltype(sc)::value;    // stage whose outputs we write
        constexpr int G = E / (1 << P::rbits(S));
        __syncthreads();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int g = i % G, j = i / G;
            xch[X::idx(m, stage_out_index<P, S>(t, g, j))] = v[i];
        });
        __syncthreads();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = xch[X::idx(m, t + i * P::TT)];
        });
        stage_compute<P, S + 1>(v, t, twL);
    });
}

template<class T>
__device__ __forceinline__ int row_reals(int len, int lp) {
    const int P = 1 << lp;
    return ((len + P - 1) >> lp) * 2 * P;
}

// ----------------------------------------------------------------------------
// Single-CTA transforms, N = 2^LOGL <= 4096, M rows per CTA.
template<class T, int LOGL, int NT>
__global__ void __launch_bounds__(NT) k_single(io_args a, const cpx<T>* __restrict__ twL) {
    using P                = splan<LOGL>;
    constexpr int L        = P::L;
    constexpr int E        = P::E;
    constexpr int TT       = P::TT;
    constexpr int M        = NT / TT;
    using X                = xch_blocked<L, M>;
    extern __shared__ __align__(16) unsigned char smem[];
    T*      raw = reinterpret_cast<T*>(smem);
    cpx<T>* xch = reinterpret_cast<cpx<T>*>(smem);

    const int       tid   = threadIdx.x;
    const int       m     = tid / TT;
    const int       t     = tid - m * TT;
    const long long row0  = (long long)blockIdx.x * M;
    const int       rows  = (int)min((long long)M, a.batch - row0);
    const int       rin   = row_reals<T>(L, a.lp_src);
    const int       rout  = row_reals<T>(L, a.lp_dst);
    const T*        src   = reinterpret_cast<const T*>(a.src) + row0 * a.src_stride;
    T*              dst   = reinterpret_cast<T*>(a.dst) + row0 * a.dst_stride;
    constexpr int   V     = 16 / sizeof(T);
    const bool      vin   = a.src_len >= L && (reinterpret_cast<uintptr_t>(src) % 16 == 0) &&
                     (a.src_stride % V == 0) && (rin % V == 0);
    const bool vout = (reinterpret_cast<uintptr_t>(dst) % 16 == 0) && (a.dst_stride % V == 0) && (rout % V == 0);

    load_rows<T, NT>(raw, rin, src, a.src_stride, rows, rin, min(a.src_len, L), a.lp_src, vin);
    __syncthreads();

    cpx<T>    v[E];
    const int Pin = 1 << a.lp_src;
    static_for<E>([&](auto ic) {
        constexpr int i   = decltype(ic)::value;
        const uint32_t p  = order_pos(t + i * TT, a.order_in, LOGL);
        const uint32_t o  = m * rin + pk_re(p, a.lp_src);
        const T        re = raw[o], im = raw[o + Pin];
        v[i]              = {re, a.conj_in ? -im : im};
    });
    stage_compute<P, 0>(v, t, twL);
    run_stages<P, X>(v, xch, m, t, twL);
    __syncthreads();

    // Last stage: value v[g + j*G] is frequency k = t + g*TT + j*Ns.
    {
        constexpr int S    = P::NST - 1;
        constexpr int G    = E / (1 << P::rbits(S));
        const int     Pout = 1 << a.lp_dst;
        const T       sc   = T(a.scale);
        const T       sim  = a.conj_out ? -sc : sc;
        static_for<E>([&](auto ic) {
            constexpr int  i = decltype(ic)::value;
            constexpr int  g = i % G, j = i / G;
            const uint32_t k = stage_out_index<P, S>(t, g, j);
            const uint32_t o = m * rout + pk_re(order_pos(k, a.order_out, LOGL), a.lp_dst);
            raw[o]           = v[i].re * sc;
            raw[o + Pout]    = v[i].im * sim;
        });
    }
    __syncthreads();
    store_rows<T, NT>(dst, a.dst_stride, raw, rout, rows, rout, vout);
}

template<class T, int LOGL, int NT>
constexpr int single_smem_bytes() {
    using P          = splan<LOGL>;
    constexpr int M  = NT / P::TT;
    constexpr int xb = xch_blocked<P::L, M>::size * (int)sizeof(cpx<T>);
    // raw rows: at most 2*L reals each (pack width <= L)
    constexpr int rb = M * 2 * P::L * (int)sizeof(T);
    return xb > rb ? xb : rb;
}

// ----------------------------------------------------------------------------
// Four-step passes.  View of one transform: n = n1*N2 + n2, k = k2*N1 + k1.
struct pass_args {
    io_args        io;
    int            log_n1, log_n2;
    int            tiles_per_row;     // CTAs per transform
    int            twiddle;           // multiply by W_N^(k_this * k_other) after the FFT
    int            row_map;           // row pass: 0 identity, 1 bit-reverse rows (log_n1 bits)
    int            transposed_out;    // row pass: write X[k*N1 + row] (natural order)
    const void*    tw_hi;             // W_N^(i*LO), i < N/LO
    const void*    tw_lo;             // W_N^i, i < LO
    int            log_lo;
};

template<class T>
__device__ __forceinline__ cpx<T> tw_big(const cpx<T>* __restrict__ hi, const cpx<T>* __restrict__ lo,
                                         uint32_t e, int log_lo) {
    const cpx<T> h = ldg_cpx(hi + (e >> log_lo));
    const cpx<T> l = ldg_cpx(lo + (e & ((1u << log_lo) - 1u)));
    return cmul(h, l);
}

// Column pass: C columns (n2 = c0..c0+C-1) of N1 = 2^LOGL rows each.
template<class T, int LOGL, int C, int NT>
__global__ void __launch_bounds__(NT) k_colpass(pass_args a, const cpx<T>* __restrict__ twL) {
    using P              = splan<LOGL>;
    constexpr int L      = P::L;
    constexpr int E      = P::E;
    constexpr int TT     = P::TT;
    static_assert(NT == C * TT, "column pass thread count");
    using X = xch_interleaved<L, C>;
    extern __shared__ __align__(16) unsigned char smem[];
    T*      raw = reinterpret_cast<T*>(smem);
    cpx<T>* xch = reinterpret_cast<cpx<T>*>(smem);

    const io_args& io  = a.io;
    const int      tid = threadIdx.x;
    const int      c   = tid % C;
    const int      t   = tid / C;
    const long long row  = blockIdx.x / a.tiles_per_row;
    const int       cg   = blockIdx.x - (int)(row * a.tiles_per_row);
    const int       c0   = cg * C;
    const int       N2   = 1 << a.log_n2;
    const T*        src  = reinterpret_cast<const T*>(io.src) + row * io.src_stride;
    T*              dst  = reinterpret_cast<T*>(io.dst) + row * io.dst_stride;
    constexpr int   SEG  = 2 * C;    // reals per row segment (pack width divides C)
    constexpr int   V    = 16 / sizeof(T);

    // gather: row n1 segment = elements [n1*N2 + c0, +C)
    {
        const int  Pin = 1 << io.lp_src;
        const bool full = io.src_len >= (L << a.log_n2);
        for (int q = tid; q < L * (SEG / V); q += NT) {
            const int  n1   = q / (SEG / V);
            const int  f    = (q - n1 * (SEG / V)) * V;
            const long long gbase = (long long)pk_re((uint32_t)n1 * N2 + c0, io.lp_src);
            if (full) {
                *reinterpret_cast<float4*>(raw + n1 * SEG + f) =
                    __ldg(reinterpret_cast<const float4*>(src + gbase + f));
            } else {
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int ff = f + u;
                    const int e  = n1 * N2 + c0 + (((ff >> (io.lp_src + 1)) << io.lp_src) | (ff & (Pin - 1)));
                    raw[n1 * SEG + ff] = e < io.src_len ? src[gbase + ff] : T(0);
                }
            }
        }
    }
    __syncthreads();

    cpx<T>    v[E];
    const int Pin = 1 << io.lp_src;
    static_for<E>([&](auto ic) {
        constexpr int  i  = decltype(ic)::value;
        const int      n1 = t + i * TT;
        const uint32_t o  = n1 * SEG + pk_re(c, io.lp_src);
        const T        re = raw[o], im = raw[o + Pin];
        v[i]              = {re, io.conj_in ? -im : im};
    });
    stage_compute<P, 0>(v, t, twL);
    run_stages<P, X>(v, xch, c, t, twL);
    __syncthreads();

    {
        constexpr int S    = P::NST - 1;
        constexpr int G    = E / (1 << P::rbits(S));
        const int     Pout = 1 << io.lp_dst;
        const T       sc   = T(io.scale);
        const T       sim  = io.conj_out ? -sc : sc;
        const auto*   hi   = reinterpret_cast<const cpx<T>*>(a.tw_hi);
        const auto*   lo   = reinterpret_cast<const cpx<T>*>(a.tw_lo);
        static_for<E>([&](auto ic) {
            constexpr int  i  = decltype(ic)::value;
            constexpr int  g  = i % G, j = i / G;
            const uint32_t k1 = stage_out_index<P, S>(t, g, j);
            cpx<T>         w  = v[i];
            if (a.twiddle) w = cmul(w, tw_big(hi, lo, k1 * (uint32_t)(c0 + c), a.log_lo));
            const uint32_t o = k1 * SEG + pk_re(c, io.lp_dst);
            raw[o]           = w.re * sc;
            raw[o + Pout]    = w.im * sim;
        });
    }
    __syncthreads();
    for (int q = tid; q < L * (SEG / V); q += NT) {
        const int       k1    = q / (SEG / V);
        const int       f     = (q - k1 * (SEG / V)) * V;
        const long long gbase = (long long)pk_re((uint32_t)k1 * N2 + c0, io.lp_dst);
        *reinterpret_cast<float4*>(dst + gbase + f) = *reinterpret_cast<const float4*>(raw + k1 * SEG + f);
    }
}

// Row pass: CR consecutive rows (r0..r0+CR-1) of N2 = 2^LOGL elements.
template<class T, int LOGL, int CR, int NT>
__global__ void __launch_bounds__(NT) k_rowpass(pass_args a, const cpx<T>* __restrict__ twL) {
    using P              = splan<LOGL>;
    constexpr int L      = P::L;
    constexpr int E      = P::E;
    constexpr int TT     = P::TT;
    static_assert(NT == CR * TT, "row pass thread count");
    using X = xch_blocked<L, CR>;
    extern __shared__ __align__(16) unsigned char smem[];
    T*      raw = reinterpret_cast<T*>(smem);
    cpx<T>* xch = reinterpret_cast<cpx<T>*>(smem);

    const io_args&  io  = a.io;
    const int       tid = threadIdx.x;
    const int       m   = tid / TT;
    const int       t   = tid - m * TT;
    const long long trf = blockIdx.x / a.tiles_per_row;
    const int       rg  = blockIdx.x - (int)(trf * a.tiles_per_row);
    const int       r0  = rg * CR;
    const int       N1  = 1 << a.log_n1;
    const T*        src = reinterpret_cast<const T*>(io.src) + trf * io.src_stride;
    T*              dst = reinterpret_cast<T*>(io.dst) + trf * io.dst_stride;
    constexpr int   RR  = 2 * L;    // reals per row (pack width divides L)
    constexpr int   V   = 16 / sizeof(T);

    // CR consecutive rows are one contiguous run of CR*RR reals.
    {
        const T* g = src + (long long)r0 * RR;
        for (int q = tid; q < CR * RR / V; q += NT) {
            *reinterpret_cast<float4*>(raw + q * V) = __ldg(reinterpret_cast<const float4*>(g + q * V));
        }
    }
    __syncthreads();

    cpx<T>    v[E];
    const int Pin = 1 << io.lp_src;
    static_for<E>([&](auto ic) {
        constexpr int  i  = decltype(ic)::value;
        const uint32_t p  = order_pos(t + i * TT, io.order_in, LOGL);
        const uint32_t o  = m * RR + pk_re(p, io.lp_src);
        const T        re = raw[o], im = raw[o + Pin];
        v[i]              = {re, io.conj_in ? -im : im};
    });
    stage_compute<P, 0>(v, t, twL);
    run_stages<P, X>(v, xch, m, t, twL);
    __syncthreads();

    const int  r      = r0 + m;
    const int  rowdft = a.row_map ? (int)brev(r, a.log_n1) : r;    // DFT index of this row
    const int  Pout   = 1 << io.lp_dst;
    const T    sc     = T(io.scale);
    const T    sim    = io.conj_out ? -sc : sc;
    constexpr int TS  = 2 * CR + 1;    // transposed staging row stride (reals), odd to spread banks
    {
        constexpr int S  = P::NST - 1;
        constexpr int G  = E / (1 << P::rbits(S));
        const auto*   hi = reinterpret_cast<const cpx<T>*>(a.tw_hi);
        const auto*   lo = reinterpret_cast<const cpx<T>*>(a.tw_lo);
        static_for<E>([&](auto ic) {
            constexpr int  i = decltype(ic)::value;
            constexpr int  g = i % G, j = i / G;
            const uint32_t k = stage_out_index<P, S>(t, g, j);
            cpx<T>         w = v[i];
            if (a.twiddle) w = cmul(w, tw_big(hi, lo, k * (uint32_t)rowdft, a.log_lo));
            uint32_t o;
            if (a.transposed_out) {
                o = k * TS + pk_re(m, io.lp_dst);
            } else {
                o = m * RR + pk_re(order_pos(k, io.order_out, LOGL), io.lp_dst);
            }
            raw[o]        = w.re * sc;
            raw[o + Pout] = w.im * sim;
        });
    }
    __syncthreads();
    if (a.transposed_out) {
        // frequency k of rows r0..r0+CR-1 -> elements k*N1 + r0 .. +CR (one segment)
        for (int q = tid; q < L * 2 * CR; q += NT) {
            const int k = q / (2 * CR), f = q - k * (2 * CR);
            dst[(long long)pk_re((uint32_t)k * N1 + r0, io.lp_dst) + f] = raw[k * TS + f];
        }
    } else {
        for (int q = tid; q < CR * RR / V; q += NT) {
            const int mm   = q / (RR / V);
            const int f    = (q - mm * (RR / V)) * V;
            const int rr   = r0 + mm;
            const int drow = a.row_map ? (int)brev(rr, a.log_n1) : rr;
            *reinterpret_cast<float4*>(dst + (long long)drow * RR + f) =
                *reinterpret_cast<const float4*>(raw + mm * RR + f);
        }
    }
}

}    // namespace pcxg
