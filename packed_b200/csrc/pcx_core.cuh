// Device building blocks shared by every FFT / correlation kernel.
//
// Data model (reference: vector.hpp:26-382, element_access.hpp:8-11):
//   packed split-complex at pack width P = 2^lp — element i has its real part
//   at offset ((i >> lp) << (lp + 1)) | (i & (P - 1)) and its imaginary part
//   P reals further.  P = 1 is interleaved complex (std::vector<std::complex>,
//   types.hpp:119-148); it is also the layout of the internal scratch rows.
//
// Transform model: every kernel computes a FORWARD DFT (sign -i, no scale,
// reference fft.hpp:728-750).  The inverse is conj(F(conj(x))) * scale, so the
// conjugations and the 1/N are folded into the loads and stores.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>

namespace pcxg {

template<class T>
struct alignas(2 * sizeof(T)) cpx {
    T re, im;
};

template<class T>
__device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return {a.re + b.re, a.im + b.im}; }
template<class T>
__device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return {a.re - b.re, a.im - b.im}; }
template<class T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
    return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
// a * conj(b)
template<class T>
__device__ __forceinline__ cpx<T> cmulc(cpx<T> a, cpx<T> b) {
    return {fma(a.re, b.re, a.im * b.im), fma(a.im, b.re, -a.re * b.im)};
}

template<class T>
__device__ __forceinline__ cpx<T> ldg_cpx(const cpx<T>* p);
template<>
__device__ __forceinline__ cpx<float> ldg_cpx(const cpx<float>* p) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return {v.x, v.y};
}
template<>
__device__ __forceinline__ cpx<double> ldg_cpx(const cpx<double>* p) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return {v.x, v.y};
}

// ---- compile-time loops -------------------------------------------------
template<class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template<int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- exact 32nd roots of unity (cos(2*pi*k/32), k = 0..8) ---------------
__host__ __device__ constexpr double cos32_tab(int k) {
    constexpr double c[9] = {1.0,
                             0.98078528040323044912618223613424,
                             0.92387953251128675612818318939679,
                             0.83146961230254523707878837761791,
                             0.70710678118654752440084436210485,
                             0.55557023301960222474283081394853,
                             0.38268343236508977172845998403040,
                             0.19509032201612826784828486847702,
                             0.0};
    return c[k];
}
__host__ __device__ constexpr double cos32(int k) {
    k = ((k % 32) + 32) % 32;
    if (k > 16) k = 32 - k;
    return k <= 8 ? cos32_tab(k) : -cos32_tab(16 - k);
}
__host__ __device__ constexpr double sin32(int k) { return cos32(k - 8); }

// a * W^K32 with W = exp(-2*pi*i/32); trivial factors cost no multiply.
template<int K32, class T>
__device__ __forceinline__ cpx<T> mulw(cpx<T> a) {
    constexpr int k = ((K32 % 32) + 32) % 32;
    constexpr T   h = T(0.70710678118654752440084436210485);
    if constexpr (k == 0) {
        return a;
    } else if constexpr (k == 8) {
        return {a.im, -a.re};
    } else if constexpr (k == 16) {
        return {-a.re, -a.im};
    } else if constexpr (k == 24) {
        return {-a.im, a.re};
    } else if constexpr (k == 4) {
        return {(a.re + a.im) * h, (a.im - a.re) * h};
    } else if constexpr (k == 12) {
        return {(a.im - a.re) * h, -(a.re + a.im) * h};
    } else if constexpr (k == 20) {
        return {-(a.re + a.im) * h, (a.re - a.im) * h};
    } else if constexpr (k == 28) {
        return {(a.re - a.im) * h, (a.re + a.im) * h};
    } else {
        constexpr T c = T(cos32(k));
        constexpr T s = T(sin32(k));
        return {fma(c, a.re, s * a.im), fma(c, a.im, -s * a.re)};
    }
}

// In-register forward DFT of the R values v[O + i*S] (i < R), natural order
// out, radix-2/4 decimation in time.  R is a power of two <= 32.
template<int R, int S, int O, class T, int E>
__device__ __forceinline__ void dft(cpx<T> (&v)[E]) {
    if constexpr (R == 2) {
        cpx<T> a = v[O], b = v[O + S];
        v[O]     = a + b;
        v[O + S] = a - b;
    } else if constexpr (R == 4) {
        cpx<T> x0 = v[O], x1 = v[O + S], x2 = v[O + 2 * S], x3 = v[O + 3 * S];
        cpx<T> a = x0 + x2, b = x0 - x2, c = x1 + x3, d = x1 - x3;
        v[O]         = a + c;
        v[O + 2 * S] = a - c;
        v[O + S]     = {b.re + d.im, b.im - d.re};
        v[O + 3 * S] = {b.re - d.im, b.im + d.re};
    } else if constexpr (R > 4) {
        dft<R / 2, 2 * S, O>(v);
        dft<R / 2, 2 * S, O + S>(v);
        cpx<T> t[R];
        static_for<R / 2>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            cpx<T>        e = v[O + 2 * k * S];
            cpx<T>        o = mulw<k * (32 / R)>(v[O + (2 * k + 1) * S]);
            t[k]            = e + o;
            t[k + R / 2]    = e - o;
        });
        static_for<R>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            v[O + k * S]    = t[k];
        });
    }
}

// ---- stage plan for an L = 2^LOGL point Stockham FFT ---------------------
// Radix-16 stages first (stage 0 carries no twiddles), remainder radix last.
// Each thread owns E values (E = EPT, or L when smaller); in every stage
// thread t holds the elements t + m*TT (m < E) of its transform, TT = L / E
// threads per transform.  A radix-R stage runs E/R butterflies per thread.
template<int LOGL_, int EPT = 16>
struct splan {
    static constexpr int LOGL = LOGL_;
    static constexpr int L    = 1 << LOGL;
    static constexpr int E    = L < EPT ? L : EPT;
    static constexpr int TT   = L / E;
    static constexpr int NST  = (LOGL + 3) / 4;
    __host__ __device__ static constexpr int rbits(int s) { return s < LOGL / 4 ? 4 : LOGL % 4; }
    __host__ __device__ static constexpr int nsbits(int s) {
        int b = 0;
        for (int i = 0; i < s; ++i) b += rbits(i);
        return b;
    }
};

// Butterflies of stage S.  twL: table W_L^i (i < L).
template<class P, int S, class T, int E>
__device__ __forceinline__ void stage_compute(cpx<T> (&v)[E], int t, const cpx<T>* __restrict__ twL) {
    static_assert(E == P::E, "register count");
    constexpr int LOGL   = P::LOGL;
    constexpr int RB     = P::rbits(S);
    constexpr int R      = 1 << RB;
    constexpr int NSB    = P::nsbits(S);
    constexpr int G      = E / R;
    constexpr int TWSH   = LOGL - NSB - RB;
    static_for<G>([&](auto gc) {
        constexpr int g = decltype(gc)::value;
        cpx<T>        a[R];
        static_for<R>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            a[j]            = v[g + j * G];
        });
        if constexpr (NSB > 0) {
            const int b = t + g * P::TT;
            const int k = b & ((1 << NSB) - 1);
            static_for<R - 1>([&](auto jc) {
                constexpr int j = decltype(jc)::value + 1;
                a[j]            = cmul(a[j], ldg_cpx(twL + ((j * k) << TWSH)));
            });
        }
        dft<R, 1, 0>(a);
        static_for<R>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            v[g + j * G]    = a[j];
        });
    });
}

// Output index of value v[g + j*G] after stage S (thread t).  After the last
// stage value v[i] holds frequency t + i*TT.
template<class P, int S>
__device__ __forceinline__ int stage_out_index(int t, int g, int j) {
    constexpr int RB  = P::rbits(S);
    constexpr int NSB = P::nsbits(S);
    const int     b   = t + g * P::TT;
    return ((b >> NSB) << (NSB + RB)) + (b & ((1 << NSB) - 1)) + (j << NSB);
}

// ---- index helpers ----------------------------------------------------------
__device__ __forceinline__ uint32_t pk_re(uint32_t i, int lp) {
    return ((i >> lp) << (lp + 1)) | (i & ((1u << lp) - 1u));
}
__device__ __forceinline__ uint32_t brev(uint32_t k, int bits) {
    return bits == 0 ? 0u : (__brev(k) >> (32 - bits));
}
// Order codes: 0 normal, 1 bit_reversed, 2 unordered (reference fft.hpp:540-544).
// Position that holds frequency k in a length-2^bits transform.  The
// reference's unordered order keeps frequency bitrev(sigma(p)) at position p,
// sigma moving bits (0,1,2,3) of p to (2,1,3,0); this returns sigma^-1(bitrev(k)).
__device__ __forceinline__ uint32_t unsigma(uint32_t q) {
    return (q & ~15u) | ((q >> 2) & 1u) | (q & 2u) | (((q >> 3) & 1u) << 2) | ((q & 1u) << 3);
}
__device__ __forceinline__ uint32_t order_pos(uint32_t k, int order, int bits) {
    if (order == 0) return k;
    uint32_t r = brev(k, bits);
    return order == 1 ? r : unsigma(r);
}

}    // namespace pcxg
