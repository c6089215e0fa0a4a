// Fused overlap-save correlation / convolution (reference fxcorr.hpp:102-136).
//
// One work item = one block of one channel: load the window of N_fft input
// samples, forward FFT, multiply by conj(K) (correlation) or K (convolution)
// with K = FFT(g)/N_fft, inverse FFT, write the `step` valid outputs.  The
// forward FFT's last stage leaves frequency t + i*TT in v[i] — exactly the
// element pattern the inverse's first stage reads — so no exchange separates
// the two transforms.
//
// Work is claimed in order from a device counter by persistent CTAs.  In
// place, block b's outputs overwrite samples that the windows of blocks
// b-1 .. b-h still read, so each block publishes "window read" (the call's
// epoch in flags[item]) and waits for its h predecessors before writing.
// Predecessors were claimed earlier by resident CTAs that never wait before
// publishing, so the wait always ends; it is still bounded (about one second
// of %globaltimer), after which the block records an error and gives up.
#pragma once

#include "pcx_fft_kernels.cuh"

namespace pcxg {

struct xc_args {
    const void*   src;
    void*         dst;
    long long     src_stride;    // reals between channels
    long long     dst_stride;
    long long     len;           // samples per channel
    int           lp;            // log2 pack width of the signal
    int           step;          // outputs per block
    int           nblk;          // blocks per channel
    long long     total;         // channels * nblk
    int           in_shift;      // window of block b starts at b*step - in_shift
    int           out_shift;     // output m of a block is circular index m + out_shift
    int           conj_kernel;   // 1: multiply by conj(K) (correlation); 0: by K (convolution)
    int           inplace;       // publish / wait on window reads
    int           hwait;         // predecessors whose windows overlap this block's outputs
    unsigned      epoch;
    unsigned*     flags;
    unsigned*     counter;
    int*          error;
    const void*   kspec;         // K / N_fft, natural order, interleaved complex
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr unsigned long long XC_WAIT_NS = 1000000000ull;    // 1 s

// Load M windows (one per group m) of L samples into interleaved complex
// shared memory, zero outside [0, len).
template<class T, int L, int NT>
__device__ __forceinline__ void xc_load(cpx<T>* s, const xc_args& a, long long item0, int M) {
    const T*  src = reinterpret_cast<const T*>(a.src);
    const int P   = 1 << a.lp;
    for (int q = threadIdx.x; q < M * L; q += NT) {
        const int       m    = q / L;
        const int       e    = q - m * L;
        const long long item = item0 + m;
        cpx<T>          v    = {T(0), T(0)};
        if (item < a.total) {
            const long long ch  = item / a.nblk;
            const long long blk = item - ch * a.nblk;
            const long long pos = blk * a.step - a.in_shift + e;
            if (pos >= 0 && pos < a.len) {
                const long long o = ch * a.src_stride + ((pos >> a.lp) << (a.lp + 1)) + (pos & (P - 1));
                v                 = {src[o], src[o + P]};
            }
        }
        s[q] = v;
    }
}

template<class T, int LOGN, int EPT, int M>
__global__ void __launch_bounds__(M * splan<LOGN, EPT>::TT) k_fxcorr(xc_args a, const cpx<T>* __restrict__ twL) {
    using P          = splan<LOGN, EPT>;
    constexpr int L  = P::L;
    constexpr int E  = P::E;
    constexpr int TT = P::TT;
    constexpr int NT = M * TT;
    using X          = xch_blocked<L, M>;
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<T>*               buf = reinterpret_cast<cpx<T>*>(smem);
    __shared__ long long  s_item;
    __shared__ int        s_abort;
    const int             tid = threadIdx.x;
    const int             m   = tid / TT;
    const int             t   = tid - m * TT;
    const cpx<T>* __restrict__ ks = reinterpret_cast<const cpx<T>*>(a.kspec);
    T*        dst = reinterpret_cast<T*>(a.dst);
    const int Pk  = 1 << a.lp;

    for (;;) {
        if (tid == 0) {
            s_item  = (long long)atomicAdd(a.counter, (unsigned)M);
            s_abort = 0;
        }
        __syncthreads();
        const long long item0 = s_item;
        if (item0 >= a.total) break;
        xc_load<T, L, NT>(buf, a, item0, M);
        __syncthreads();
        if (a.inplace && tid == 0) {
            __threadfence();
            for (int mm = 0; mm < M && item0 + mm < a.total; ++mm) st_release(a.flags + item0 + mm, a.epoch);
        }
        cpx<T> v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = buf[m * L + t + i * TT];
        });
        stage_compute<P, 0>(v, t, twL);
        run_stages<P, X>(v, buf, m, t, twL);
        // spectral product, conjugated for the inverse: u = conj(X * conj(K)) or conj(X * K)
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const cpx<T>  k = ldg_cpx(ks + t + i * TT);
            const cpx<T>  c = {v[i].re, -v[i].im};
            v[i]            = a.conj_kernel ? cmul(c, k) : cmulc(c, k);
        });
        stage_compute<P, 0>(v, t, twL);
        run_stages<P, X>(v, buf, m, t, twL);

        const long long item = item0 + m;
        if (a.inplace) {
            if (tid == 0) {
                for (int mm = 0; mm < M && item0 + mm < a.total; ++mm) {
                    const long long it  = item0 + mm;
                    const long long blk = it % a.nblk;
                    for (int d = 1; d <= a.hwait && d <= blk; ++d) {
                        const unsigned* f = a.flags + (it - d);
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
                        if (s_abort) break;
                    }
                    if (s_abort) break;
                }
            }
            __syncthreads();
            if (s_abort) return;    // every thread of the CTA leaves together
        }
        if (item < a.total) {
            const long long ch  = item / a.nblk;
            const long long blk = item - ch * a.nblk;
            const long long b0  = blk * a.step;
            T*              d   = dst + ch * a.dst_stride;
            static_for<E>([&](auto ic) {
                constexpr int   i  = decltype(ic)::value;
                const int       mo = t + i * TT - a.out_shift;
                const long long e  = b0 + mo;
                if (mo >= 0 && mo < a.step && e < a.len) {
                    const long long o = ((e >> a.lp) << (a.lp + 1)) + (e & (Pk - 1));
                    d[o]              = v[i].re;
                    d[o + Pk]         = -v[i].im;
                }
            });
        }
        __syncthreads();
    }
}

template<class T, int LOGN, int EPT, int M>
constexpr int fxcorr_smem_bytes() {
    return xch_blocked<(1 << LOGN), M>::size * (int)sizeof(cpx<T>);
}

// ---------------------------------------------------------------------------
// Kernel-gradient pass: for every block, the spectrum product
// FFT(x window) * conj(FFT(gy block zero-padded)) is accumulated per CTA in
// `acc` (grid x N_fft, interleaved complex; read-modify-write, L2 resident).
// gg = IFFT(sum over CTAs of acc)[0..K).
struct kg_args {
    const void* x;
    const void* gy;
    long long   stride;       // reals between channels (x and gy)
    long long   len;
    int         lp;
    int         step;
    int         nblk;
    long long   total;
    unsigned*   counter;
    void*       acc;          // [gridDim.x][N] complex
    void*       xspec;        // [gridDim.x][N] complex, per-CTA spectrum scratch
    int*        error;        // set when a bounded wait gave up (forms with bulk copies)
};

template<class T, int LOGN, int EPT>
__global__ void __launch_bounds__(splan<LOGN, EPT>::TT) k_fxcorr_kgrad(kg_args a, const cpx<T>* __restrict__ twL) {
    using P          = splan<LOGN, EPT>;
    constexpr int L  = P::L;
    constexpr int E  = P::E;
    constexpr int TT = P::TT;
    using X          = xch_blocked<L, 1>;
    extern __shared__ __align__(16) unsigned char smem[];
    cpx<T>*              buf = reinterpret_cast<cpx<T>*>(smem);
    __shared__ long long s_item;
    const int            t   = threadIdx.x;
    cpx<T>*              acc = reinterpret_cast<cpx<T>*>(a.acc) + (long long)blockIdx.x * L;
    cpx<T>*              xs  = reinterpret_cast<cpx<T>*>(a.xspec) + (long long)blockIdx.x * L;
    for (int e = t; e < L; e += TT) acc[e] = {T(0), T(0)};

    xc_args la{};
    la.len        = a.len;
    la.lp         = a.lp;
    la.step       = a.step;
    la.nblk       = a.nblk;
    la.total      = a.total;
    la.src_stride = a.stride;
    la.src        = a.x;
    for (;;) {
        if (t == 0) s_item = (long long)atomicAdd(a.counter, 1u);
        __syncthreads();
        const long long item = s_item;
        if (item >= a.total) break;
        // x window [b*step, b*step + N)
        xc_load<T, L, TT>(buf, la, item, 1);
        __syncthreads();
        cpx<T> v[E];
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = buf[t + i * TT];
        });
        stage_compute<P, 0>(v, t, twL);
        run_stages<P, X>(v, buf, 0, t, twL);
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            xs[t + i * TT]  = v[i];
        });
        __syncthreads();
        // gy block [b*step, b*step + step), zero-padded to N
        {
            const T*        gy  = reinterpret_cast<const T*>(a.gy);
            const long long ch  = item / a.nblk;
            const long long blk = item - ch * a.nblk;
            const int       Pk  = 1 << a.lp;
            for (int e = t; e < L; e += TT) {
                const long long pos = blk * a.step + e;
                cpx<T>          w   = {T(0), T(0)};
                if (e < a.step && pos < a.len) {
                    const long long o = ch * a.stride + ((pos >> a.lp) << (a.lp + 1)) + (pos & (Pk - 1));
                    w                 = {gy[o], gy[o + Pk]};
                }
                buf[e] = w;
            }
        }
        __syncthreads();
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            v[i]            = buf[t + i * TT];
        });
        stage_compute<P, 0>(v, t, twL);
        run_stages<P, X>(v, buf, 0, t, twL);
        static_for<E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const int     k = t + i * TT;
            acc[k]          = acc[k] + cmulc(xs[k], v[i]);
        });
        __syncthreads();
    }
}

// Sum the per-CTA spectra and conjugate (for an inverse by forward FFT).
template<class T>
__global__ void k_kgrad_reduce(const cpx<T>* __restrict__ acc, int ctas, int n, cpx<T>* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    cpx<T> s = {T(0), T(0)};
    for (int c = 0; c < ctas; ++c) s = s + acc[(long long)c * n + k];
    out[k] = s;
}

}    // namespace pcxg
