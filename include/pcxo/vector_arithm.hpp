// pcxo/vector_arithm.hpp — element-wise expressions over packed vectors
// (reference vector_arithm.hpp:405-1140), evaluated on the GPU.
//
// `a + b`, `a - b`, `a * b`, `a / b` between vectors (or std::vector of
// std::complex, or nested expressions), the same with a complex scalar on
// either side, and `conj(e)` build a lazy expression; assigning it to a
// pcxo::vector (`v = a * conj(b) + 2.F;`) or calling `pcxo::assign(dest, e)`
// compiles it into a short postfix program that one kernel evaluates for
// every element (pcx_vec_eval), each operand read at its own pack width.
// Vector operands are held by reference, as the reference's expressions
// are, and must stay alive until the assignment; they must be in device or
// managed memory (pcxo::vector's default allocator).  The assignment returns
// after the GPU has finished.
#ifndef PCXO_VECTOR_ARITHM_HPP
#define PCXO_VECTOR_ARITHM_HPP

#include "types.hpp"

#include <complex>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace pcxo {

namespace detail_ {
struct vexpr_base {};

template<typename E>
concept vexpr_node = std::derived_from<std::remove_cvref_t<E>, vexpr_base>;
template<typename V>
concept vexpr_leaf = (!vexpr_node<V>) && requires { typename cx_vector_traits<std::remove_cvref_t<V>>::real_type; } &&
                     floating_point<typename cx_vector_traits<std::remove_cvref_t<V>>::real_type>;
template<typename E>
concept vexpr = vexpr_node<E> || vexpr_leaf<E>;

// Postfix program of one expression (the C ABI's pcx_expr_op list).
struct vexpr_program {
    pcx_expr_op ops[PCX_EXPR_MAX_OPS]{};
    int         n_ops = 0;
    const void* vecs[PCX_EXPR_MAX_VECS]{};
    int         packs[PCX_EXPR_MAX_VECS]{};
    int         n_vecs = 0;
    uZ          size   = 0;
    bool        sized  = false;

    void push(int code, int arg = 0, double re = 0, double im = 0) {
        if (n_ops == PCX_EXPR_MAX_OPS) throw std::invalid_argument("vector expression has more than 32 nodes");
        ops[n_ops++] = pcx_expr_op{code, arg, re, im};
    }
    int operand(const void* p, int pack, uZ n) {
        if (!sized) {
            size  = n;
            sized = true;
        } else if (n != size) {
            throw std::invalid_argument(std::string("source size (which is ") + std::to_string(n) +
                                        " is not equal to expression size (which is " + std::to_string(size) + ")");
        }
        for (int k = 0; k < n_vecs; ++k) {
            if (vecs[k] == p && packs[k] == pack) return k;
        }
        if (n_vecs == PCX_EXPR_MAX_VECS) throw std::invalid_argument("vector expression has more than 8 vectors");
        if (!device_accessible(p)) {
            throw std::invalid_argument("vector expression operands must be in device or managed memory");
        }
        vecs[n_vecs]  = p;
        packs[n_vecs] = pack;
        return n_vecs++;
    }
};

// A vector operand, held by reference.
template<typename V>
struct vexpr_ref : vexpr_base {
    using real_type = typename cx_vector_traits<std::remove_cvref_t<V>>::real_type;
    const V* v;
    void     emit(vexpr_program& p) const {
        using tr = cx_vector_traits<std::remove_cvref_t<V>>;
        p.push(PCX_OP_VEC, p.operand(tr::re_data(*v), static_cast<int>(tr::pack_size), tr::size(*v)));
    }
};
template<typename T>
struct vexpr_scalar : vexpr_base {
    using real_type = T;
    std::complex<T> s;
    void            emit(vexpr_program& p) const { p.push(PCX_OP_SCALAR, 0, s.real(), s.imag()); }
};
template<int Code, typename L, typename R>
struct vexpr_bin : vexpr_base {
    using real_type = typename L::real_type;
    L    l;
    R    r;
    void emit(vexpr_program& p) const {
        l.emit(p);
        r.emit(p);
        p.push(Code);
    }
};
template<typename E>
struct vexpr_conj : vexpr_base {
    using real_type = typename E::real_type;
    E    e;
    void emit(vexpr_program& p) const {
        e.emit(p);
        p.push(PCX_OP_CONJ);
    }
};

// node of an operand: vectors by reference, expression nodes by value
template<typename X>
auto as_node(const X& x) {
    if constexpr (vexpr_node<X>) {
        return x;
    } else {
        return vexpr_ref<X>{{}, &x};
    }
}
template<typename E>
using node_t = decltype(as_node(std::declval<const E&>()));
template<typename E>
using real_of = typename node_t<E>::real_type;

template<typename E, typename S>
concept vexpr_scalar_of = vexpr<E> && (!vexpr<S>) && std::is_convertible_v<S, std::complex<real_of<E>>>;

template<int Code, typename A, typename B>
auto make_bin(const A& a, const B& b) {
    static_assert(std::same_as<real_of<A>, real_of<B>>, "operands of one real type");
    return vexpr_bin<Code, node_t<A>, node_t<B>>{{}, as_node(a), as_node(b)};
}
}    // namespace detail_

// ---- operators (reference vector_arithm.hpp:450-495)
#define PCXO_VEXPR_BINOP(OP, CODE)                                                                        \
    template<typename A, typename B>                                                                      \
        requires detail_::vexpr<A> && detail_::vexpr<B>                                                   \
    auto operator OP(const A& a, const B& b) {                                                            \
        return detail_::make_bin<CODE>(a, b);                                                             \
    }                                                                                                     \
    template<typename E, typename S>                                                                      \
        requires detail_::vexpr_scalar_of<E, S>                                                           \
    auto operator OP(const E& e, S s) {                                                                   \
        using T = detail_::real_of<E>;                                                                    \
        return detail_::vexpr_bin<CODE, detail_::node_t<E>, detail_::vexpr_scalar<T>>{                    \
            {}, detail_::as_node(e), detail_::vexpr_scalar<T>{{}, std::complex<T>(s)}};                   \
    }                                                                                                     \
    template<typename S, typename E>                                                                      \
        requires detail_::vexpr_scalar_of<E, S>                                                           \
    auto operator OP(S s, const E& e) {                                                                   \
        using T = detail_::real_of<E>;                                                                    \
        return detail_::vexpr_bin<CODE, detail_::vexpr_scalar<T>, detail_::node_t<E>>{                    \
            {}, detail_::vexpr_scalar<T>{{}, std::complex<T>(s)}, detail_::as_node(e)};                   \
    }
PCXO_VEXPR_BINOP(+, PCX_OP_ADD)
PCXO_VEXPR_BINOP(-, PCX_OP_SUB)
PCXO_VEXPR_BINOP(*, PCX_OP_MUL)
PCXO_VEXPR_BINOP(/, PCX_OP_DIV)
#undef PCXO_VEXPR_BINOP

template<typename E>
    requires detail_::vexpr<E>
auto conj(const E& e) {
    return detail_::vexpr_conj<detail_::node_t<E>>{{}, detail_::as_node(e)};
}

// dest = expression on the GPU (reference vector.hpp:177-182, subrange::assign 494-506).
template<typename D, typename E>
    requires detail_::vexpr_leaf<D> && detail_::vexpr<E>
void assign(D& dest, const E& expression, cudaStream_t stream = nullptr) {
    using dt = cx_vector_traits<std::remove_cvref_t<D>>;
    static_assert(std::same_as<typename dt::real_type, detail_::real_of<E>>, "expression of the vector's real type");
    detail_::vexpr_program p;
    detail_::as_node(expression).emit(p);
    const uZ n = dt::size(dest);
    if (p.sized && p.size != n) {
        throw std::invalid_argument(std::string("source size (which is ") + std::to_string(p.size) +
                                    " is not equal to subrange size (which is " + std::to_string(n) + ")");
    }
    auto* d = dt::re_data(dest);
    if (!detail_::device_accessible(d)) throw std::invalid_argument("destination must be in device or managed memory");
    detail_::check(pcx_vec_eval(std::same_as<typename dt::real_type, double> ? PCX_F64 : PCX_F32, d,
                                static_cast<int>(dt::pack_size), n, p.ops, p.n_ops, p.vecs, p.packs, p.n_vecs, stream));
    detail_::check_cuda(cudaStreamSynchronize(stream));
}

}    // namespace pcxo
#endif
