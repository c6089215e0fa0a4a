// Element-wise expressions over packed split-complex vectors on the device:
// the evaluation that pcxo::vector expression templates do on the CPU in the
// reference (vector_arithm.hpp:405-1140: +, -, *, / between vectors, with
// complex scalars, conj).  The host compiles an expression tree into a short
// postfix program; one grid-stride kernel walks it for every element with a
// small stack in registers, reading each operand at its own pack width and
// writing the destination at its pack width.  Memory-bound: one read per
// operand vector and one write per element.
#include "pcx_core.cuh"
#include "pcx_host.hpp"

#include <algorithm>
#include <string>

using namespace pcxg;

namespace {

constexpr int MAX_DEPTH = 8;

template<class T>
struct vprog {
    int      n_ops;
    int      code[PCX_EXPR_MAX_OPS];
    int      arg[PCX_EXPR_MAX_OPS];
    T        sre[PCX_EXPR_MAX_OPS];
    T        sim[PCX_EXPR_MAX_OPS];
    const T* vec[PCX_EXPR_MAX_VECS];
    int      lp[PCX_EXPR_MAX_VECS];
};

template<class T>
__device__ __forceinline__ cpx<T> cdiv(cpx<T> a, cpx<T> b) {
    const T d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

template<class T>
__global__ void k_vec_eval(vprog<T> p, T* __restrict__ dst, int lpd, long long n) {
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += step) {
        cpx<T> st[MAX_DEPTH];
        int    sp = 0;
        for (int q = 0; q < p.n_ops; ++q) {
            const int c = p.code[q];
            if (c == PCX_OP_VEC) {
                const int       k = p.arg[q];
                const long long P = 1LL << p.lp[k];
                const long long o = ((e >> p.lp[k]) << (p.lp[k] + 1)) + (e & (P - 1));
                st[sp++]          = {p.vec[k][o], p.vec[k][o + P]};
            } else if (c == PCX_OP_SCALAR) {
                st[sp++] = {p.sre[q], p.sim[q]};
            } else if (c == PCX_OP_CONJ) {
                st[sp - 1].im = -st[sp - 1].im;
            } else {
                const cpx<T> b = st[--sp];
                const cpx<T> a = st[sp - 1];
                cpx<T>       r;
                if (c == PCX_OP_ADD) r = {a.re + b.re, a.im + b.im};
                else if (c == PCX_OP_SUB) r = {a.re - b.re, a.im - b.im};
                else if (c == PCX_OP_MUL) r = cmul(a, b);
                else r = cdiv(a, b);
                st[sp - 1] = r;
            }
        }
        const long long P = 1LL << lpd;
        const long long o = ((e >> lpd) << (lpd + 1)) + (e & (P - 1));
        dst[o]            = st[0].re;
        dst[o + P]        = st[0].im;
    }
}

int check_pack(int pack, const char* what) {
    if (pack < 1 || (pack & (pack - 1)) != 0) {
        return pcx_fail(PCX_ERR_INVALID, std::string(what) + " pack size (which is " + std::to_string(pack) +
                                             ") is not a power of two");
    }
    return PCX_OK;
}

template<class T>
int launch(void* dst, int pack_dst, size_t n, const pcx_expr_op* ops, int n_ops, const void* const* vecs,
           const int* packs, int n_vecs, cudaStream_t st) {
    vprog<T> p{};
    p.n_ops = n_ops;
    for (int q = 0; q < n_ops; ++q) {
        p.code[q] = ops[q].code;
        p.arg[q]  = ops[q].arg;
        p.sre[q]  = T(ops[q].re);
        p.sim[q]  = T(ops[q].im);
    }
    for (int k = 0; k < n_vecs; ++k) {
        p.vec[k] = static_cast<const T*>(vecs[k]);
        p.lp[k]  = __builtin_ctz(packs[k]);
    }
    int dev = 0, sms = 148;
    PCX_CUDA_TRY(cudaGetDevice(&dev));
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    const long long blocks = std::min<long long>(((long long)n + 255) / 256, (long long)sms * 8);
    k_vec_eval<T><<<(unsigned)blocks, 256, 0, st>>>(p, static_cast<T*>(dst), __builtin_ctz(pack_dst), (long long)n);
    PCX_CUDA_TRY(cudaGetLastError());
    return PCX_OK;
}

}    // namespace

extern "C" int pcx_vec_eval(int dtype, void* dst, int pack_dst, size_t n, const pcx_expr_op* ops, int n_ops,
                            const void* const* vecs, const int* vec_packs, int n_vecs, void* stream) {
    return pcx_guard([&]() -> int {
        if (dtype != PCX_F32 && dtype != PCX_F64) return pcx_fail(PCX_ERR_INVALID, "unknown dtype");
        if (int rc = check_pack(pack_dst, "destination")) return rc;
        if (n_ops < 1 || n_ops > PCX_EXPR_MAX_OPS) return pcx_fail(PCX_ERR_INVALID, "expression has 0 or too many nodes");
        if (n_vecs < 0 || n_vecs > PCX_EXPR_MAX_VECS) return pcx_fail(PCX_ERR_INVALID, "expression has too many vectors");
        if (!ops || (n_vecs > 0 && (!vecs || !vec_packs))) return pcx_fail(PCX_ERR_INVALID, "null expression data");
        for (int k = 0; k < n_vecs; ++k) {
            if (!vecs[k]) return pcx_fail(PCX_ERR_INVALID, "null operand vector");
            if (int rc = check_pack(vec_packs[k], "operand")) return rc;
        }
        // the program must leave exactly one value and stay within the stack
        int depth = 0, peak = 0;
        for (int q = 0; q < n_ops; ++q) {
            const int c = ops[q].code;
            if (c == PCX_OP_VEC) {
                if (ops[q].arg < 0 || ops[q].arg >= n_vecs) return pcx_fail(PCX_ERR_INVALID, "operand index out of range");
                ++depth;
            } else if (c == PCX_OP_SCALAR) {
                ++depth;
            } else if (c == PCX_OP_CONJ) {
                if (depth < 1) return pcx_fail(PCX_ERR_INVALID, "malformed expression");
            } else if (c == PCX_OP_ADD || c == PCX_OP_SUB || c == PCX_OP_MUL || c == PCX_OP_DIV) {
                if (depth < 2) return pcx_fail(PCX_ERR_INVALID, "malformed expression");
                --depth;
            } else {
                return pcx_fail(PCX_ERR_INVALID, "unknown expression node");
            }
            peak = std::max(peak, depth);
        }
        if (depth != 1) return pcx_fail(PCX_ERR_INVALID, "malformed expression");
        if (peak > MAX_DEPTH) return pcx_fail(PCX_ERR_UNSUPPORTED, "expression nested too deeply (stack of 8)");
        if (n == 0) return PCX_OK;
        if (!dst) return pcx_fail(PCX_ERR_INVALID, "null destination");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        return dtype == PCX_F64 ? launch<double>(dst, pack_dst, n, ops, n_ops, vecs, vec_packs, n_vecs, st)
                                : launch<float>(dst, pack_dst, n, ops, n_ops, vecs, vec_packs, n_vecs, st);
    });
}
