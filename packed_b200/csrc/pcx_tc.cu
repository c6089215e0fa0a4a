// Tensor-core FFT: radix-16 stages as dense DFT-matrix products on the
// fifth-generation tensor cores (tcgen05.mma, FP32 accumulation in TMEM).
//
// A radix-16 stage over 128 butterflies is D = X * A^T with X the 128 x 32
// real matrix of twiddled inputs (16 complex per row: reals then
// imaginaries) and A the 32 x 32 real form of the 16-point DFT,
//   [[C, S], [-S, C]],  C = cos(2 pi jk/16), S = sin(2 pi jk/16).
// Operands are split so that the products recover FP32-level accuracy:
//   PREC_BF16: x = hi + lo in bfloat16, D = Xh Ah + Xh Al + Xl Ah (three
//              products, kind::f16);
//   PREC_TF32: the same split in tf32 (kind::tf32);
//   PREC_BF16X6: x = hi + mid + lo in bfloat16 and the six products whose
//              parts add up to at most the second order (kind::f16).
// The dropped lo*lo term and the representation error of hi + lo set the
// accuracy (about 2^-16 per stage for bfloat16, 2^-21 for tf32).
//
// k_tcfft (the two passes of 2^13..2^16 points): one CTA of 128 threads
// transforms T rows; thread i owns TMEM lane i (one butterfly per 128-row
// block).  k_tcp (whole rows of 2^8..2^12 points): persistent CTAs of 256
// threads, one round of products per radix-16 stage.  Twiddles, the remainder radix-2/4/8 stage and
// the data movement stay on the CUDA cores; one elected thread issues the
// MMAs and commits them to an mbarrier.  Every mbarrier wait is bounded.
#include "pcx_fft_v2.cuh"
#include "pcx_host.hpp"
#include "pcx_tmem.cuh"

#include <algorithm>
#include <cuda_bf16.h>

namespace pcxg {
namespace tc {

constexpr int NT = 128;
enum : int { PREC_BF16 = 0, PREC_TF32 = 1, PREC_BF16X6 = 2 };

template<int PREC>
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    if constexpr (PREC != PREC_TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
            : "memory");
    }
}
// The same product with A read from tensor memory (a_tmem: its first column;
// row m of A in lane m, K along the columns, 32 bits per column).
template<int PREC>
__device__ __forceinline__ void umma_ta(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    if constexpr (PREC != PREC_TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
            "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
            "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
            : "memory");
    }
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; lbo = byte step between K-adjacent core matrices,
// sbo = byte step between 8-row groups.
__device__ __forceinline__ uint64_t sdesc(const void* p, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((smem_u32(p) >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;    // descriptor version of this architecture
    return d;                  // base offset 0, no swizzle
}

// Operand element type and its per-MMA K.
template<int PREC>
struct op_traits;
template<>
struct op_traits<PREC_BF16> {
    using elem                      = uint16_t;
    static constexpr int NS         = 2;    // parts of each operand
    static constexpr int K_PER_MMA  = 16;
    static constexpr int PER_CHUNK  = 8;    // elements per 16-byte core-matrix row
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
    __device__ static elem bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
    __device__ static float fl(elem e) { return __bfloat162float(__ushort_as_bfloat16(e)); }
    __device__ static void split(float x, elem (&p)[NS]) {
        p[0] = bf(x);
        p[1] = bf(x - fl(p[0]));
    }
    // the constant operand's parts, each rounded from the exact remainder
    __device__ static void split_exact(double v, elem (&p)[NS]) {
        p[0] = __bfloat16_as_ushort(__double2bfloat16(v));
        p[1] = __bfloat16_as_ushort(__double2bfloat16(v - (double)fl(p[0])));
    }
    // two adjacent K elements (lo, hi) rounded together into one 32-bit word
    // (the same round-to-nearest per element as bf()), and back to floats
    __device__ static uint32_t pk2(float lo, float hi) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
    __device__ static float2 unpk2(uint32_t w) {
        return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
    }
    // split() of two adjacent elements, parts packed in pairs
    __device__ static void split2(float lo, float hi, uint32_t (&w)[NS]) {
        w[0]           = pk2(lo, hi);
        const float2 f = unpk2(w[0]);
        w[1]           = pk2(lo - f.x, hi - f.y);
    }
};
template<>
struct op_traits<PREC_BF16X6> : op_traits<PREC_BF16> {
    static constexpr int NS = 3;
    __device__ static void split(float x, elem (&p)[NS]) {
        p[0]          = bf(x);
        const float r = x - fl(p[0]);    // exact
        p[1]          = bf(r);
        p[2]          = bf(r - fl(p[1]));
    }
    __device__ static void split_exact(double v, elem (&p)[NS]) {
        p[0] = __bfloat16_as_ushort(__double2bfloat16(v));
        p[1] = __bfloat16_as_ushort(__double2bfloat16(v - (double)fl(p[0])));
        p[2] = __bfloat16_as_ushort(__double2bfloat16(v - (double)fl(p[0]) - (double)fl(p[1])));
    }
    __device__ static void split2(float lo, float hi, uint32_t (&w)[NS]) {
        w[0]            = pk2(lo, hi);
        const float2 f0 = unpk2(w[0]);
        const float  rl = lo - f0.x, rh = hi - f0.y;    // exact
        w[1]            = pk2(rl, rh);
        const float2 f1 = unpk2(w[1]);
        w[2]            = pk2(rl - f1.x, rh - f1.y);
    }
};
template<>
struct op_traits<PREC_TF32> {
    using elem                      = uint32_t;
    static constexpr int NS         = 2;
    static constexpr int K_PER_MMA  = 8;
    static constexpr int PER_CHUNK  = 4;
    static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
    __device__ static uint32_t to_tf32(float x) {
        uint32_t r;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
        return r;
    }
    __device__ static void split(float x, elem (&p)[NS]) {
        p[0] = to_tf32(x);
        p[1] = to_tf32(x - __uint_as_float(p[0]));
    }
    __device__ static void split_exact(double v, elem (&p)[NS]) {
        p[0] = to_tf32((float)v);
        p[1] = to_tf32((float)(v - (double)__uint_as_float(p[0])));
    }
};

// Products of the split operands, smallest first: (part of X, part of A).
template<int NS>
struct split_products;
template<>
struct split_products<2> {
    static constexpr int NP = 3;
    __host__ __device__ static constexpr int x(int p) { return p == 0 ? 1 : 0; }
    __host__ __device__ static constexpr int a(int p) { return p == 1 ? 1 : 0; }
};
template<>
struct split_products<3> {
    static constexpr int NP = 6;
    __host__ __device__ static constexpr int x(int p) { return p == 0 ? 2 : (p == 1 || p == 3) ? 1 : 0; }
    __host__ __device__ static constexpr int a(int p) { return p == 2 ? 2 : (p == 1 || p == 4) ? 1 : 0; }
};

// Byte offset of element (row, k) of a rows x 32 K-major operand stored as
// [k chunk][8-row group][row in group][element in chunk].
template<int PREC, int ROWS>
__device__ __forceinline__ uint32_t op_off(int row, int k) {
    using O                 = op_traits<PREC>;
    constexpr uint32_t ROWB = 16;
    constexpr uint32_t CM   = 8 * ROWB;           // core matrix bytes
    constexpr uint32_t LBO  = (ROWS / 8) * CM;    // next K chunk
    return (uint32_t)(k / O::PER_CHUNK) * LBO + (uint32_t)(row / 8) * CM + (uint32_t)(row % 8) * ROWB +
           (uint32_t)(k % O::PER_CHUNK) * (uint32_t)sizeof(typename O::elem);
}

struct tc_args {
    const float* src;
    float*       dst;
    long long    batch;    // rows (mode 2) or transforms (mode 1)
    int          conj;
    float        scale;
    const void*  twN;    // W_N^i
    int*         error;
    // two-pass forms of a transform of N * 2^lg_other points
    int          lg_other;    // mode 1: log2 of the row length; mode 2: log2 of the rows per transform
    const void*  tw_hi;       // W_M^(i * 2^lg_other), M = N * 2^lg_other (mode 1)
    const void*  tw_lo;       // W_M^i, i < 2^lg_other (mode 1)
};

// The two passes of a transform of 2^13..2^16 points (whole rows of 2^8..2^12
// points run in k_tcp below), one launch each:
//   1: column pass of a two-pass transform of M = N * C points laid out as
//      N rows of C (C = 2^lg_other): each CTA transforms T adjacent columns
//      of one transform, multiplies output k of column c by W_M^(c k) and
//      writes it back to the same place (the input conjugated for the inverse);
//   2: row pass: each CTA transforms T rows of N points of the column pass's
//      output (R = 2^lg_other rows per transform) and writes output k of row
//      j to element k * R + j, the transform's natural order (the output
//      conjugated and scaled for the inverse).
// Modes 1 and 2 read and write whole 8-point packs of T >= 8 adjacent columns.
// Smem plan: work[2][T*N] complex | B parts (32 x 32).  Tensor memory: the
// accumulator (columns 0..31), then the operand rows, one 32-element K row per
// part (ACOLS 32-bit columns each).
template<int LOGN, int PREC>
struct tc_cfg {
    static constexpr int N     = 1 << LOGN;
    static constexpr int T     = N >= 2048 ? 1 : 2048 / N;    // rows per CTA: >= 128 butterflies per stage
    static constexpr int R0B   = LOGN % 4;                    // remainder stage (CUDA cores) first
    static constexpr int NTC   = LOGN / 4;                    // radix-16 tensor-core stages
    static constexpr int OPB   = (int)sizeof(typename op_traits<PREC>::elem);
    static constexpr int NS    = op_traits<PREC>::NS;
    static constexpr int BBYTE = 32 * 32 * OPB;
    static constexpr int ACOLS = 32 * OPB / 4;
    static constexpr int TCOLS = 32 + NS * ACOLS <= 64 ? 64 : 128;
    // padded work layout (one pad element per 8): faster wherever it keeps
    // three CTAs per SM or there is no remainder stage (measured per form)
    static constexpr bool PAD  = PREC != PREC_TF32 || LOGN % 4 == 0;
    static constexpr int  WORK = T * N + (PAD ? T * N / 8 : 0);    // complex per work buffer
    static constexpr int  SMEM = 2 * WORK * 8 + NS * BBYTE;
    static_assert(32 + NS * ACOLS <= TCOLS, "accumulator and operand rows in the allocation");
};

template<int LOGN, int PREC, int MODE>
__global__ void __launch_bounds__(NT, 1) k_tcfft(tc_args a) {
    static_assert((MODE == 1 || MODE == 2) && tc_cfg<LOGN, PREC>::T % 8 == 0,
                  "the two passes move whole packs of columns (whole rows: k_tcp)");
    using C  = tc_cfg<LOGN, PREC>;
    using O  = op_traits<PREC>;
    using E  = typename O::elem;
    constexpr int N   = C::N;
    constexpr int T   = C::T;
    constexpr int NB  = T * N / 16;    // radix-16 butterflies per stage in this CTA
    extern __shared__ __align__(128) unsigned char smem[];
    // work buffers: element i at wp(i) = i + i/8 (a pad after every 8 elements
    // keeps the strided Stockham stores and the per-pack row accesses on
    // distinct banks), or at i
    auto        wp    = [](int i) { return C::PAD ? i + (i >> 3) : i; };
    cpx<float>* work0 = reinterpret_cast<cpx<float>*>(smem);
    cpx<float>* work1 = work0 + C::WORK;
    constexpr int  NS = C::NS;    // parts of each split operand
    unsigned char* opB[NS];       // the DFT matrix A (the twiddled inputs X go to tensor memory)
    static_for<NS>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        opB[i]          = reinterpret_cast<unsigned char*>(work1 + C::WORK) + i * C::BBYTE;
    });
    __shared__ uint64_t mbar;
    __shared__ uint32_t tslot;
    bool                aborted = false;
    const int  tid  = threadIdx.x;
    const int  warp = tid / 32;
    const auto* twN = reinterpret_cast<const cpx<float>*>(a.twN);
    const long long row0 = (long long)blockIdx.x * T;
    const int       rows = MODE == 1 ? T : (int)min((long long)T, a.batch - row0);

    if (warp == 0) {
        tmem_alloc(&tslot, C::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        fence_barrier_init();
    }
    // constant operand: the 32 x 32 real DFT matrix, split
    for (int q = tid; q < 32 * 32; q += NT) {
        const int n = q / 32, k = q % 32;
        const int nn = n % 16, kk = k % 16;
        double    s, c;
        sincospi(2.0 * (double)((nn * kk) % 16) / 16.0, &s, &c);
        double v;
        if (n < 16) v = k < 16 ? c : s;
        else v = k < 16 ? -s : c;
        E part[NS];
        O::split_exact(v, part);
        static_for<NS>([&](auto ic) {
            constexpr int i                                       = decltype(ic)::value;
            *reinterpret_cast<E*>(opB[i] + op_off<PREC, 32>(n, k)) = part[i];
        });
    }
    const bool conj_in  = MODE != 2 && a.conj;
    const bool conj_out = MODE != 1 && a.conj;
    if constexpr (MODE == 1) {
        // T adjacent columns c0.. of one transform, one pack of 8 columns of
        // one row per thread and step (four 16-byte loads)
        const long long cols = 1LL << a.lg_other;
        const long long gpt  = cols / T;
        const long long tr   = (long long)blockIdx.x / gpt;
        const long long c0   = ((long long)blockIdx.x % gpt) * T;
        const float*    base = a.src + tr * (2 * N * cols);
        const float     cj   = conj_in ? -1.f : 1.f;
        for (int q = tid; q < T * N / 8; q += NT) {
            const int     i  = q % N, jg = q / N;
            const float4* s  = reinterpret_cast<const float4*>(base + 2 * (i * cols + c0 + 8 * jg));
            const float4  r0 = __ldg(s), r1 = __ldg(s + 1), i0 = __ldg(s + 2), i1 = __ldg(s + 3);
            const int     b0 = (8 * jg) * N + i;
            work0[wp(b0 + 0 * N)] = {r0.x, cj * i0.x};
            work0[wp(b0 + 1 * N)] = {r0.y, cj * i0.y};
            work0[wp(b0 + 2 * N)] = {r0.z, cj * i0.z};
            work0[wp(b0 + 3 * N)] = {r0.w, cj * i0.w};
            work0[wp(b0 + 4 * N)] = {r1.x, cj * i1.x};
            work0[wp(b0 + 5 * N)] = {r1.y, cj * i1.y};
            work0[wp(b0 + 6 * N)] = {r1.z, cj * i1.z};
            work0[wp(b0 + 7 * N)] = {r1.w, cj * i1.w};
        }
    } else
    // rows in natural order (conjugated for the inverse); missing rows are zero
    // (one 64-byte pack of 8 samples per thread and step, 16-byte loads)
    for (int q = tid; q < T * N / 8; q += NT) {
        const int r = q / (N / 8), pk8 = q % (N / 8);
        float4    r0 = {0.f, 0.f, 0.f, 0.f}, r1 = r0, i0 = r0, i1 = r0;
        if (r < rows) {
            const float4* s = reinterpret_cast<const float4*>(a.src + (row0 + r) * (2 * N) + pk8 * 16);
            r0              = __ldg(s);
            r1              = __ldg(s + 1);
            i0              = __ldg(s + 2);
            i1              = __ldg(s + 3);
        }
        const float      cj = conj_in ? -1.f : 1.f;
        cpx<float>*      w  = work0 + wp(r * N + pk8 * 8);    // 8 elements, no pad inside
        w[0] = {r0.x, cj * i0.x};
        w[1] = {r0.y, cj * i0.y};
        w[2] = {r0.z, cj * i0.z};
        w[3] = {r0.w, cj * i0.w};
        w[4] = {r1.x, cj * i1.x};
        w[5] = {r1.y, cj * i1.y};
        w[6] = {r1.z, cj * i1.z};
        w[7] = {r1.w, cj * i1.w};
    }
    fence_proxy_async_smem();    // B is read by the products (async proxy)
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = tslot;
    cpx<float>*    in    = work0;
    cpx<float>*    out   = work1;
    int            ns    = 1;    // size of the sub-transforms done so far

    // remainder stage (radix 2, 4 or 8) on the CUDA cores, no twiddles
    if constexpr (C::R0B > 0) {
        constexpr int R  = 1 << C::R0B;
        constexpr int NR = T * N / R;
        for (int b = tid; b < NR; b += NT) {
            const int  tr = b / (N / R), bl = b % (N / R);
            cpx<float> x[R];
            static_for<R>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                x[j]            = in[wp(tr * N + bl + j * (N / R))];
            });
            dft<R, 1, 0>(x);
            static_for<R>([&](auto jc) {
                constexpr int j              = decltype(jc)::value;
                out[wp(tr * N + bl * R + j)] = x[j];
            });
        }
        ns = R;
        cpx<float>* t = in;
        in            = out;
        out           = t;
        __syncthreads();
    }

    uint32_t phase    = 0;
    int      tw_shift = LOGN - 4 - __ffs(ns) + 1;    // log2(N / (16 ns))
    // twiddle j of a butterfly at position k is W_{16 ns}^(jk): one or two of
    // the six factors W^(qk), q = 1,2,3,4,8,12, read from the W_N table
    // (W_{16 ns}^e = W_N^(e * N / (16 ns))); each block's factors are
    // requested while the previous block's products run
    auto load_f = [&](cpx<float>(&g)[6], int nsx, int shx, int mbx) {
        const int kx = ((mbx + tid) % (N / 16)) & (nsx - 1);
        if (nsx > 1) {
            g[0] = ldg_cpx(twN + ((kx) << shx));
            g[1] = ldg_cpx(twN + ((2 * kx) << shx));
            g[2] = ldg_cpx(twN + ((3 * kx) << shx));
            g[3] = ldg_cpx(twN + ((4 * kx) << shx));
            g[4] = ldg_cpx(twN + ((8 * kx) << shx));
            g[5] = ldg_cpx(twN + ((12 * kx) << shx));
        }
    };
    cpx<float> fn[6] = {};
    load_f(fn, ns, tw_shift, 0);
    for (int st = 0; st < C::NTC; ++st) {
        for (int mb = 0; mb < NB; mb += 128) {
            const int  b  = mb + tid;
            const int  tr = b / (N / 16), bl = b % (N / 16);
            const int  k  = bl & (ns - 1);
            cpx<float> x[16];
            cpx<float> f[6];
            static_for<6>([&](auto qc) { f[decltype(qc)::value] = fn[decltype(qc)::value]; });
            static_for<16>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                cpx<float>    v = in[wp(tr * N + bl + j * (N / 16))];
                if constexpr (j > 0) {
                    if (ns > 1) v = cmul(v, stw_factor<4, j>(f));
                }
                x[j] = v;
            });
            // operand rows (reals 0..15 then imaginaries 16..31), one 16-byte
            // core-matrix row per store
            static_for<32 / O::PER_CHUNK>([&](auto cc) {
                constexpr int c = decltype(cc)::value;
                uint32_t      part[NS][4];
                if constexpr (PREC == PREC_TF32) {
                    static_for<4>([&](auto qc) {
                        constexpr int q  = decltype(qc)::value;
                        constexpr int kk = c * 4 + q;
                        E             e[NS];
                        O::split(kk < 16 ? x[kk & 15].re : x[kk & 15].im, e);
                        static_for<NS>([&](auto ic) { part[decltype(ic)::value][q] = e[decltype(ic)::value]; });
                    });
                } else {
                    // bfloat16: adjacent pairs rounded together, one word per pair and part
                    static_for<4>([&](auto qc) {
                        constexpr int q  = decltype(qc)::value;
                        constexpr int kk = c * 8 + 2 * q;
                        uint32_t      w[NS];
                        O::split2(kk < 16 ? x[kk & 15].re : x[kk & 15].im,
                                  kk + 1 < 16 ? x[(kk + 1) & 15].re : x[(kk + 1) & 15].im, w);
                        static_for<NS>([&](auto ic) { part[decltype(ic)::value][q] = w[decltype(ic)::value]; });
                    });
                }
                static_for<NS>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    tmem_st4_nowait(taddr + ((uint32_t)(32 * warp) << 16) + 32 + (uint32_t)(i * C::ACOLS + 4 * c),
                                    part[i][0], part[i][1], part[i][2], part[i][3]);
                });
            });
            tmem_wait_st();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                constexpr uint32_t LBO_B = (32 / 8) * 128, SBO = 128;
                constexpr int      KS    = 32 / O::K_PER_MMA;               // MMAs per product
                constexpr int      CH    = O::K_PER_MMA / O::PER_CHUNK;     // chunks per MMA (2)
                constexpr uint32_t KCOL  = O::K_PER_MMA * C::OPB / 4;       // A columns per product's K
                using SP                 = split_products<NS>;
                uint32_t           acc   = 0;
                static_for<SP::NP>([&](auto pc) {
                    constexpr int        p  = decltype(pc)::value;
                    const uint32_t       xa = taddr + 32 + (uint32_t)(SP::x(p) * C::ACOLS);
                    const unsigned char* ab = opB[SP::a(p)];
                    for (int ks = 0; ks < KS; ++ks) {
                        umma_ta<PREC>(taddr, xa + ks * KCOL, sdesc(ab + ks * CH * LBO_B, LBO_B, SBO), O::IDESC, acc);
                        acc = 1;
                    }
                });
                umma_commit(&mbar);
            }
            if (mb + 128 < NB) {
                load_f(fn, ns, tw_shift, mb + 128);
            } else if (st + 1 < C::NTC) {
                load_f(fn, ns * 16, tw_shift - 4, 0);
            }
            const bool ok = mbar_wait_bounded(&mbar, phase);
            if (__syncthreads_or(!ok)) {
                // give up: record it and let the MMAs in flight finish before TMEM is freed
                if (tid == 0) {
                    atomicExch(a.error, 1);
                    mbar_wait_bounded(&mbar, phase, 100000000ull);
                }
                aborted = true;
                break;
            }
            phase ^= 1;
            tc_fence_after();
            uint32_t r[32];
            tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16), r);
            // outputs of this butterfly, Stockham placement
            const int base = tr * N + (bl / ns) * ns * 16 + k;
            static_for<16>([&](auto jc) {
                constexpr int j        = decltype(jc)::value;
                out[wp(base + j * ns)] = {__uint_as_float(r[j]), __uint_as_float(r[j + 16])};
            });
            tc_fence_before();
            __syncthreads();    // operands and accumulator free for the next block
        }
        if (aborted) break;
        ns *= 16;
        tw_shift -= 4;
        cpx<float>* t = in;
        in            = out;
        out           = t;
        __syncthreads();
    }
    if (!aborted && MODE == 1) {
        const int         lgo  = a.lg_other;
        const long long   cols = 1LL << lgo;
        const long long   gpt  = cols / T;
        const long long   tr   = (long long)blockIdx.x / gpt;
        const int         c0   = (int)(((long long)blockIdx.x % gpt) * T);
        const cpx<float>* th   = reinterpret_cast<const cpx<float>*>(a.tw_hi);
        const cpx<float>* tl   = reinterpret_cast<const cpx<float>*>(a.tw_lo);
        float*            base = a.dst + tr * (2 * N * cols);
        for (int q = tid; q < T * N / 8; q += NT) {
            const int k = q % N, jg = q / N;
            float     re[8], im[8];
            static_for<8>([&](auto ec) {
                constexpr int  e  = decltype(ec)::value;
                const uint32_t ex = (uint32_t)(c0 + 8 * jg + e) * (uint32_t)k;    // < M
                const cpx<float> t =
                    cmul(ldg_cpx(th + (ex >> lgo)), ldg_cpx(tl + (ex & (uint32_t)(cols - 1))));
                const cpx<float> o = cmul(in[wp((8 * jg + e) * N + k)], t);
                re[e]              = o.re;
                im[e]              = o.im;
            });
            float4* d = reinterpret_cast<float4*>(base + 2 * (k * cols + c0 + 8 * jg));
            d[0]      = make_float4(re[0], re[1], re[2], re[3]);
            d[1]      = make_float4(re[4], re[5], re[6], re[7]);
            d[2]      = make_float4(im[0], im[1], im[2], im[3]);
            d[3]      = make_float4(im[4], im[5], im[6], im[7]);
        }
    } else if (!aborted && MODE == 2) {
        const float     sc   = a.scale, sim = conj_out ? -a.scale : a.scale;
        const long long R    = 1LL << a.lg_other;    // rows per transform; T divides R
        const long long tr   = row0 / R;
        const long long j0   = row0 % R;
        float*          base = a.dst + tr * (2 * N * R);
        for (int q = tid; q < T * N / 8; q += NT) {
            const int         k = q % N, jg = q / N;
            auto              w = [&](int e) { return in[wp((8 * jg + e) * N + k)]; };
            float4*           d = reinterpret_cast<float4*>(base + 2 * (k * R + j0 + 8 * jg));
            d[0] = make_float4(w(0).re * sc, w(1).re * sc, w(2).re * sc, w(3).re * sc);
            d[1] = make_float4(w(4).re * sc, w(5).re * sc, w(6).re * sc, w(7).re * sc);
            d[2] = make_float4(w(0).im * sim, w(1).im * sim, w(2).im * sim, w(3).im * sim);
            d[3] = make_float4(w(4).im * sim, w(5).im * sim, w(6).im * sim, w(7).im * sim);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, C::TCOLS);
}

// ---------------------------------------------------------------------------
// Persistent form for whole rows (N = 2^8..2^12): each CTA of 256 threads
// takes items of 4096 points (T = 4096 / N rows) in turn, so the DFT matrix
// and the TMEM columns are set up once per CTA, not once per row group.  A
// radix-16 stage is one round: every thread builds the operand row of one of
// the item's 256 butterflies and writes it to its own TMEM lane (warps 0-3 the
// first block of 128 rows, warps 4-7 the second, each in its own lane
// quarter), thread 0 issues two M = 128 products with A read from tensor
// memory (into TMEM columns 0..31 and 32..63), and every thread reads its own
// butterfly's 32 outputs back from its lane.  The work buffer is updated in
// place (all of a stage's reads land in the operands before the first write);
// shared memory holds only it and the DFT matrix, and the CTAs per SM are set
// by tensor memory and registers (three in the bfloat16 form, two in the
// others).  Work element p sits at p + 2*(p/16): the strided reads of the
// operand build, the Stockham writes and the packs of 8 contiguous elements
// of the row copies are all conflict-free, and the first stage's 16
// contiguous outputs per thread go out as 16-byte stores.
// The same kernel runs a list of items of mixed sizes (the ragged batch's
// transforms of up to 4096 points), each with its own rows.
constexpr int TP_NT  = 256;
constexpr int TP_PTS = 4096;    // points per item
constexpr int TP_MAXR = TP_PTS / 256;    // rows per item at N = 256

using tcp_item = tc_item;    // lg 8..12, rows 1 .. 4096 / N, one source and destination row each
static_assert(sizeof(((tc_item*)nullptr)->src) / sizeof(const float*) == TP_MAXR, "rows per item");

struct tcp_args {
    // uniform form: `batch` rows of 2^lg points at src/dst (2N reals apart)
    const float*    src;
    float*          dst;
    long long       batch;
    int             lg;
    // list form (when items != nullptr)
    const tcp_item* items;
    int             nitems;
    int             conj;     // inputs and outputs conjugated (the inverse)
    float           scale;    // on the outputs
    const void*     tw;       // W_M^i, i < M = 2^tw_lg (tw_lg >= every item's lg)
    int             tw_lg;
    int*            error;
};

template<int PREC>
struct tcp_cfg {
    using O                    = op_traits<PREC>;
    static constexpr int NS    = O::NS;
    static constexpr int OPB   = (int)sizeof(typename O::elem);
    static constexpr int WORK  = TP_PTS + TP_PTS / 8;           // complex, padded
    static constexpr int BBYTE = 32 * 32 * OPB;
    static constexpr int SMEM  = WORK * 8 + NS * BBYTE;
    // tensor memory: the two accumulators (columns 0..63), then the operand
    // rows, one 32-element K row per block and part (ACOLS 32-bit columns)
    static constexpr int ACOLS = 32 * OPB / 4;
    static constexpr int USED  = 64 + 2 * NS * ACOLS;
    static constexpr int TCOLS = USED <= 128 ? 128 : 256;
    static constexpr int MINB  = TCOLS <= 128 ? 3 : 2;    // CTAs per SM (tensor memory, registers)
    static_assert(USED <= TCOLS && MINB * TCOLS <= 512, "tensor memory of the resident CTAs");
};

__device__ __forceinline__ int tcp_wp(int p) { return p + 2 * (p >> 4); }

// One item of N = 2^LOGN points: rows s_src[r] -> s_dst[r], r < rows.  False
// when the bounded wait for the products gave up (the CTA then leaves).
template<int LOGN, int PREC>
__device__ __forceinline__ bool tcp_run(const tcp_args& a, int rows, const float* const* s_src, float* const* s_dst,
                                        cpx<float>* work, unsigned char* const (&opB)[op_traits<PREC>::NS],
                                        uint32_t taddr,
                                        uint64_t* mbar, uint32_t& phase) {
    using O           = op_traits<PREC>;
    using C           = tcp_cfg<PREC>;
    using E           = typename O::elem;
    constexpr int NS  = O::NS;
    constexpr int N   = 1 << LOGN;
    constexpr int T   = TP_PTS / N;
    constexpr int R0B = LOGN % 4;
    constexpr int NTC = LOGN / 4;
    const int     tid = threadIdx.x;
    const int     warp = tid / 32;
    const float   cj   = a.conj ? -1.f : 1.f;
    // this thread's operand row: lane tid % 128 (its warp's quarter), block tid / 128
    const uint32_t arow = taddr + ((uint32_t)(32 * (warp % 4)) << 16) + 64 + (uint32_t)((warp / 4) * NS * C::ACOLS);
    const auto*   tw   = reinterpret_cast<const cpx<float>*>(a.tw);
    const int  tr = tid / (N / 16), bl = tid % (N / 16);
    // the first tensor-core stage's twiddle factors (W_{16 ns}^(qk), q =
    // 1,2,3,4,8,12, from the W_M table); each later stage's are requested
    // while the previous stage's products run
    cpx<float> fn[6] = {};
    auto       load_f = [&](int nsx) {
        if (nsx > 1) {
            const int k  = bl & (nsx - 1);
            const int sh = a.tw_lg - 4 - (__ffs(nsx) - 1);
            fn[0]        = ldg_cpx(tw + ((k) << sh));
            fn[1]        = ldg_cpx(tw + ((2 * k) << sh));
            fn[2]        = ldg_cpx(tw + ((3 * k) << sh));
            fn[3]        = ldg_cpx(tw + ((4 * k) << sh));
            fn[4]        = ldg_cpx(tw + ((8 * k) << sh));
            fn[5]        = ldg_cpx(tw + ((12 * k) << sh));
        }
    };
    load_f(1 << R0B);
    // rows in natural order (conjugated for the inverse); missing rows are
    // zero.  Two 8-point packs per thread, all loads first.
    static_assert(T * N / 8 == 2 * TP_NT, "two packs per thread");
    {
        float4 v[2][4];
        static_for<2>([&](auto uc) {
            constexpr int u   = decltype(uc)::value;
            const int     q   = tid + u * TP_NT;
            const int     r   = q / (N / 8), pk8 = q % (N / 8);
            v[u][0] = v[u][1] = v[u][2] = v[u][3] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (r < rows) {
                const float4* s = reinterpret_cast<const float4*>(s_src[r] + pk8 * 16);
                static_for<4>([&](auto hc) { v[u][decltype(hc)::value] = __ldg(s + decltype(hc)::value); });
            }
        });
        static_for<2>([&](auto uc) {
            constexpr int u   = decltype(uc)::value;
            const int     q   = tid + u * TP_NT;
            const int     r   = q / (N / 8), pk8 = q % (N / 8);
            const float4 &r0 = v[u][0], &r1 = v[u][1], &i0 = v[u][2], &i1 = v[u][3];
            float4*       w   = reinterpret_cast<float4*>(work + tcp_wp(r * N + pk8 * 8));    // 8 contiguous elements
            w[0]              = make_float4(r0.x, cj * i0.x, r0.y, cj * i0.y);
            w[1]              = make_float4(r0.z, cj * i0.z, r0.w, cj * i0.w);
            w[2]              = make_float4(r1.x, cj * i1.x, r1.y, cj * i1.y);
            w[3]              = make_float4(r1.z, cj * i1.z, r1.w, cj * i1.w);
        });
    }
    __syncthreads();
    int ns = 1;
    // remainder stage (radix 2, 4 or 8) on the CUDA cores, in place
    if constexpr (R0B > 0) {
        constexpr int R = 1 << R0B;
        constexpr int U = 16 / R;    // butterflies per thread
        cpx<float>    x[16];
        static_for<U>([&](auto uc) {
            constexpr int u  = decltype(uc)::value;
            const int     b  = tid + u * TP_NT;
            const int     tr = b / (N / R), bl = b % (N / R);
            static_for<R>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                x[u * R + j]    = work[tcp_wp(tr * N + bl + j * (N / R))];
            });
        });
        __syncthreads();
        static_for<U>([&](auto uc) {
            constexpr int u  = decltype(uc)::value;
            const int     b  = tid + u * TP_NT;
            const int     tr = b / (N / R), bl = b % (N / R);
            dft<R, 1, u * R>(x);
            static_for<R>([&](auto jc) {
                constexpr int j                     = decltype(jc)::value;
                work[tcp_wp(tr * N + bl * R + j)] = x[u * R + j];
            });
        });
        ns = R;
        __syncthreads();
    }
    for (int st = 0; st < NTC; ++st) {
        const int  k = bl & (ns - 1);
        cpx<float> x[16];
        // twiddle j of the butterfly: W_{16 ns}^(jk), from the six factors
        static_for<16>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            cpx<float>    v = work[tcp_wp(tr * N + bl + j * (N / 16))];
            if constexpr (j > 0) {
                if (ns > 1) v = cmul(v, stw_factor<4, j>(fn));
            }
            x[j] = v;
        });
        // operand row tid (reals 0..15 then imaginaries 16..31) into this
        // thread's tensor-memory lane, four columns at a time
        static_for<32 / O::PER_CHUNK>([&](auto cc) {
            constexpr int c = decltype(cc)::value;
            uint32_t      part[NS][4];
            if constexpr (PREC == PREC_TF32) {
                static_for<4>([&](auto qc) {
                    constexpr int q  = decltype(qc)::value;
                    constexpr int kk = c * 4 + q;
                    E             e[NS];
                    O::split(kk < 16 ? x[kk & 15].re : x[kk & 15].im, e);
                    static_for<NS>([&](auto ic) { part[decltype(ic)::value][q] = e[decltype(ic)::value]; });
                });
            } else {
                // bfloat16: adjacent pairs rounded together, one word per pair and part
                static_for<4>([&](auto qc) {
                    constexpr int q  = decltype(qc)::value;
                    constexpr int kk = c * 8 + 2 * q;
                    uint32_t      w[NS];
                    O::split2(kk < 16 ? x[kk & 15].re : x[kk & 15].im,
                              kk + 1 < 16 ? x[(kk + 1) & 15].re : x[(kk + 1) & 15].im, w);
                    static_for<NS>([&](auto ic) { part[decltype(ic)::value][q] = w[decltype(ic)::value]; });
                });
            }
            static_for<NS>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                tmem_st4_nowait(arow + (uint32_t)(i * C::ACOLS + 4 * c), part[i][0], part[i][1], part[i][2],
                                part[i][3]);
            });
        });
        tmem_wait_st();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            constexpr uint32_t LBO_B = (32 / 8) * 128, SBO = 128;
            constexpr int      KS    = 32 / O::K_PER_MMA;
            constexpr int      CH    = O::K_PER_MMA / O::PER_CHUNK;
            constexpr uint32_t KCOL  = O::K_PER_MMA * C::OPB / 4;    // A columns per product's K
            using SP                 = split_products<NS>;
            static_for<2>([&](auto bc) {
                constexpr int blk = decltype(bc)::value;
                uint32_t      acc = 0;
                static_for<SP::NP>([&](auto pc) {
                    constexpr int        p  = decltype(pc)::value;
                    const uint32_t       xa = taddr + 64 + (uint32_t)((blk * NS + SP::x(p)) * C::ACOLS);
                    const unsigned char* ab = opB[SP::a(p)];
                    for (int ks = 0; ks < KS; ++ks) {
                        umma_ta<PREC>(taddr + 32 * blk, xa + ks * KCOL, sdesc(ab + ks * CH * LBO_B, LBO_B, SBO),
                                      O::IDESC, acc);
                        acc = 1;
                    }
                });
            });
            umma_commit(mbar);
        }
        if (st + 1 < NTC) load_f(ns * 16);
        const bool ok = mbar_wait_bounded(mbar, phase);
        if (__syncthreads_or(!ok)) {
            // give up: record it and let the products in flight finish before TMEM is freed
            if (tid == 0) {
                atomicExch(a.error, 1);
                mbar_wait_bounded(mbar, phase, 100000000ull);
            }
            return false;
        }
        phase ^= 1;
        tc_fence_after();
        uint32_t r[32];
        tmem_ld32(taddr + ((uint32_t)(32 * (warp % 4)) << 16) + 32 * (warp / 4), r);
        // outputs of this butterfly, Stockham placement, in place
        const int base = tr * N + (bl / ns) * ns * 16 + k;
        if (ns == 1) {
            // sixteen contiguous outputs: eight 16-byte stores
            float4* w = reinterpret_cast<float4*>(work + tcp_wp(base));
            static_for<8>([&](auto jc) {
                constexpr int j = decltype(jc)::value;
                w[j]            = make_float4(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 16]),
                                              __uint_as_float(r[2 * j + 1]), __uint_as_float(r[2 * j + 17]));
            });
        } else {
            static_for<16>([&](auto jc) {
                constexpr int j                = decltype(jc)::value;
                work[tcp_wp(base + j * ns)] = {__uint_as_float(r[j]), __uint_as_float(r[j + 16])};
            });
        }
        tc_fence_before();
        __syncthreads();    // operands, accumulator and work free for the next stage
        ns *= 16;
    }
    // natural order out (conjugated and scaled for the inverse)
    const float sc = a.scale, sim = a.conj ? -a.scale : a.scale;
    static_for<2>([&](auto uc) {
        const int q = tid + decltype(uc)::value * TP_NT;
        const int r = q / (N / 8), pk8 = q % (N / 8);
        if (r < rows) {
            const float4* w  = reinterpret_cast<const float4*>(work + tcp_wp(r * N + pk8 * 8));
            const float4  w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
            float4*       d  = reinterpret_cast<float4*>(s_dst[r] + pk8 * 16);
            d[0]             = make_float4(w0.x * sc, w0.z * sc, w1.x * sc, w1.z * sc);
            d[1]             = make_float4(w2.x * sc, w2.z * sc, w3.x * sc, w3.z * sc);
            d[2]             = make_float4(w0.y * sim, w0.w * sim, w1.y * sim, w1.w * sim);
            d[3]             = make_float4(w2.y * sim, w2.w * sim, w3.y * sim, w3.w * sim);
        }
    });
    __syncthreads();    // the work buffer and row pointers are free for the next item
    return true;
}

template<int PREC>
__global__ void __launch_bounds__(TP_NT, tcp_cfg<PREC>::MINB) k_tcp(tcp_args a) {
    using C          = tcp_cfg<PREC>;
    using O          = op_traits<PREC>;
    using E          = typename O::elem;
    constexpr int NS = O::NS;
    extern __shared__ __align__(128) unsigned char smem[];
    cpx<float>*    work = reinterpret_cast<cpx<float>*>(smem);
    unsigned char* opBw[NS];
    static_for<NS>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        opBw[i]         = smem + C::WORK * 8 + i * C::BBYTE;
    });
    __shared__ uint64_t     mbar;
    __shared__ uint32_t     tslot;
    __shared__ const float* s_src[TP_MAXR];
    __shared__ float*       s_dst[TP_MAXR];
    const int               tid  = threadIdx.x;
    const int               warp = tid / 32;
    if (warp == 0) {
        tmem_alloc(&tslot, C::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        fence_barrier_init();
    }
    // constant operand, once per CTA: the 32 x 32 real DFT matrix, split
    for (int q = tid; q < 32 * 32; q += TP_NT) {
        const int n = q / 32, k = q % 32;
        const int nn = n % 16, kk = k % 16;
        double    s, c;
        sincospi(2.0 * (double)((nn * kk) % 16) / 16.0, &s, &c);
        double v;
        if (n < 16) v = k < 16 ? c : s;
        else v = k < 16 ? -s : c;
        E part[NS];
        O::split_exact(v, part);
        static_for<NS>([&](auto ic) {
            constexpr int i                                        = decltype(ic)::value;
            *reinterpret_cast<E*>(opBw[i] + op_off<PREC, 32>(n, k)) = part[i];
        });
    }
    fence_proxy_async_smem();    // B is read by the products (async proxy)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t  taddr  = tslot;
    uint32_t        phase  = 0;
    const long long nitems = a.items ? (long long)a.nitems : (a.batch + (TP_PTS >> a.lg) - 1) / (TP_PTS >> a.lg);
    for (long long j = blockIdx.x; j < nitems; j += gridDim.x) {
        int lg, rows;
        if (a.items) {
            const tcp_item& it = a.items[j];
            lg                 = it.lg;
            rows               = it.rows;
            if (tid < rows) {
                s_src[tid] = it.src[tid];
                s_dst[tid] = it.dst[tid];
            }
        } else {
            const int       T  = TP_PTS >> a.lg;
            const long long r0 = j * T;
            lg                 = a.lg;
            rows               = (int)min((long long)T, a.batch - r0);
            if (tid < rows) {
                s_src[tid] = a.src + (r0 + tid) * (2LL << lg);
                s_dst[tid] = a.dst + (r0 + tid) * (2LL << lg);
            }
        }
        __syncthreads();
        bool ok = true;
        switch (lg) {
        case 8: ok = tcp_run<8, PREC>(a, rows, s_src, s_dst, work, opBw, taddr, &mbar, phase); break;
        case 9: ok = tcp_run<9, PREC>(a, rows, s_src, s_dst, work, opBw, taddr, &mbar, phase); break;
        case 10: ok = tcp_run<10, PREC>(a, rows, s_src, s_dst, work, opBw, taddr, &mbar, phase); break;
        case 11: ok = tcp_run<11, PREC>(a, rows, s_src, s_dst, work, opBw, taddr, &mbar, phase); break;
        case 12: ok = tcp_run<12, PREC>(a, rows, s_src, s_dst, work, opBw, taddr, &mbar, phase); break;
        default: break;
        }
        if (!ok) break;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, C::TCOLS);
}

}    // namespace tc
}    // namespace pcxg

using namespace pcxg;

namespace {
template<int LOGN, int PREC, int MODE>
cudaError_t launch_tc(const tc::tc_args& a, cudaStream_t st) {
    using C   = tc::tc_cfg<LOGN, PREC>;
    auto kern = tc::k_tcfft<LOGN, PREC, MODE>;
    cudaError_t e = smem_attr_cached(reinterpret_cast<const void*>(kern), C::SMEM);
    if (e != cudaSuccess) return e;
    // mode 1: one CTA per T columns of a transform; otherwise per T rows
    const long long grid = MODE == 1 ? a.batch * ((1LL << a.lg_other) / C::T) : (a.batch + C::T - 1) / C::T;
    if (grid == 0) return cudaSuccess;
    kern<<<(unsigned)grid, tc::NT, C::SMEM, st>>>(a);
    return cudaGetLastError();
}
// The persistent whole-row form: resident CTAs, at most one per item.
template<int PREC>
cudaError_t launch_tcp(const tc::tcp_args& a, long long nitems, int sms, cudaStream_t st) {
    using C   = tc::tcp_cfg<PREC>;
    auto kern = tc::k_tcp<PREC>;
    cudaError_t e = smem_attr_cached(reinterpret_cast<const void*>(kern), C::SMEM);
    if (e != cudaSuccess) return e;
    if (nitems <= 0) return cudaSuccess;
    // C::MINB CTAs per SM (the tensor memory each allocates and the register
    // bound of __launch_bounds__); more would wait in tcgen05.alloc
    const long long grid = std::max<long long>(1, std::min<long long>(nitems, (long long)C::MINB * sms));
    kern<<<(unsigned)grid, tc::TP_NT, C::SMEM, st>>>(a);
    return cudaGetLastError();
}
// passes of the two-pass form: sub-transforms of 2^6..2^8 points
template<int PREC, int MODE>
cudaError_t dispatch_tc_pass(int log_n, const tc::tc_args& a, cudaStream_t st) {
    switch (log_n) {
    case 6: return launch_tc<6, PREC, MODE>(a, st);
    case 7: return launch_tc<7, PREC, MODE>(a, st);
    case 8: return launch_tc<8, PREC, MODE>(a, st);
    default: return cudaErrorNotSupported;
    }
}
}    // namespace

cudaError_t pcx_tc_list_launch(int precision, const pcxg::tc_item* items, int nitems, int conj, float scale,
                               const void* tw, int tw_lg, int* error, int sms, cudaStream_t st) {
    tc::tcp_args a{};
    a.items  = items;
    a.nitems = nitems;
    a.conj   = conj;
    a.scale  = scale;
    a.tw     = tw;
    a.tw_lg  = tw_lg;
    a.error  = error;
    return precision == 0   ? launch_tcp<tc::PREC_BF16>(a, nitems, sms, st)
           : precision == 1 ? launch_tcp<tc::PREC_TF32>(a, nitems, sms, st)
                            : launch_tcp<tc::PREC_BF16X6>(a, nitems, sms, st);
}

// Tensor-core transform of `batch` contiguous rows (pack 8, natural order).
extern "C" int pcx_tc_fft_exec(pcx_plan plan, void* dst, const void* src, int direction, int normalize,
                               size_t batch, int precision, void* stream) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        if (plan->dtype != PCX_F32 || plan->order != PCX_ORDER_NORMAL) {
            return pcx_fail(PCX_ERR_UNSUPPORTED, "tensor-core form: complex64, natural order");
        }
        const bool two = plan->two_pass && plan->log_n1 >= 6 && plan->log_n1 <= 8 && plan->log_n2 >= 6 &&
                         plan->log_n2 <= 8;
        if (!two && (plan->log_n < 8 || plan->log_n > 12)) {
            return pcx_fail(PCX_ERR_UNSUPPORTED, "tensor-core form built for 2^8 <= N <= 2^16");
        }
        if (precision < 0 || precision > 2) return pcx_fail(PCX_ERR_INVALID, "precision: 0 bf16x3, 1 tf32x3, 2 bf16x6");
        if ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) % 16 != 0) {
            return pcx_fail(PCX_ERR_INVALID, "data pointers must be 16-byte aligned");
        }
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (two) {
            // column pass into the plan's scratch (one L2-sized chunk of
            // transforms at a time), row pass out to dst in natural order
            const size_t per   = plan->n * sizeof(cpx<float>);
            const size_t chunk = plan->chunk_rows(batch);
            std::lock_guard<std::mutex> g(plan->mu);
            if (plan->scratch_bytes < chunk * per) {
                if (plan->scratch) cudaFree(plan->scratch);
                plan->scratch       = nullptr;
                plan->scratch_bytes = 0;
                PCX_CUDA_TRY(cudaMalloc(&plan->scratch, chunk * per));
                plan->scratch_bytes = chunk * per;
            }
            for (size_t r0 = 0; r0 < batch; r0 += chunk) {
                const size_t rows = std::min(chunk, batch - r0);
                tc::tc_args  c{};
                c.src      = static_cast<const float*>(src) + r0 * 2 * plan->n;
                c.dst      = static_cast<float*>(plan->scratch);
                c.batch    = (long long)rows;
                c.conj     = direction == PCX_INVERSE;
                c.scale    = 1.0f;
                c.twN      = plan->twN1;
                c.error    = plan->err;
                c.lg_other = plan->log_n2;
                c.tw_hi    = plan->tw_hi;
                c.tw_lo    = plan->tw_lo;
                tc::tc_args r = c;
                r.src      = static_cast<const float*>(plan->scratch);
                r.dst      = static_cast<float*>(dst) + r0 * 2 * plan->n;
                r.batch    = (long long)(rows << plan->log_n1);
                r.scale    = (direction == PCX_INVERSE && normalize) ? 1.0f / (float)plan->n : 1.0f;
                r.twN      = plan->twN2;
                r.lg_other = plan->log_n1;
                cudaError_t e1 = precision == 0   ? dispatch_tc_pass<tc::PREC_BF16, 1>(plan->log_n1, c, st)
                                 : precision == 1 ? dispatch_tc_pass<tc::PREC_TF32, 1>(plan->log_n1, c, st)
                                                  : dispatch_tc_pass<tc::PREC_BF16X6, 1>(plan->log_n1, c, st);
                PCX_CUDA_TRY(e1);
                cudaError_t e2 = precision == 0   ? dispatch_tc_pass<tc::PREC_BF16, 2>(plan->log_n2, r, st)
                                 : precision == 1 ? dispatch_tc_pass<tc::PREC_TF32, 2>(plan->log_n2, r, st)
                                                  : dispatch_tc_pass<tc::PREC_BF16X6, 2>(plan->log_n2, r, st);
                PCX_CUDA_TRY(e2);
            }
            return PCX_OK;
        }
        // whole rows: the persistent form, items of 4096 points, the plan's
        // full W_N table
        tc::tcp_args a{};
        a.src    = static_cast<const float*>(src);
        a.dst    = static_cast<float*>(dst);
        a.batch  = (long long)batch;
        a.lg     = plan->log_n;
        a.conj   = direction == PCX_INVERSE;
        a.scale  = (direction == PCX_INVERSE && normalize) ? 1.0f / (float)plan->n : 1.0f;
        a.tw     = plan->twL;
        a.tw_lg  = plan->log_n;
        a.error  = plan->err;
        const long long items = ((long long)batch + (tc::TP_PTS >> plan->log_n) - 1) / (tc::TP_PTS >> plan->log_n);
        cudaError_t     e     = precision == 0   ? launch_tcp<tc::PREC_BF16>(a, items, plan->sms, st)
                                : precision == 1 ? launch_tcp<tc::PREC_TF32>(a, items, plan->sms, st)
                                                 : launch_tcp<tc::PREC_BF16X6>(a, items, plan->sms, st);
        PCX_CUDA_TRY(e);
        return PCX_OK;
    });
}
