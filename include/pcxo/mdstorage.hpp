// pcxo/mdstorage.hpp — drop-in for the multidimensional packed storage of
// the reference (mdstorage.hpp:1012-1498): named axes, left/right layouts,
// the inner axis stored as packed split-complex rows padded to
// lcm(2*PackSize, Alignment) reals (calc_storage_size, mdstorage.hpp:857-863),
// slicing by axis (get_dynamic_slice_offset, mdstorage.hpp:370-391), and rows
// that fft_unit accepts as vectors.  Storage is CUDA managed memory by
// default, so slices are usable on the host and the GPU alike.
//
// Batched GPU calls over every inner row at once:
//   pcxo::md::fft_rows(unit, storage)            forward transform of all rows
//   pcxo::md::ifft_rows<Norm>(unit, storage)     inverse of all rows
//   pcxo::md::fxcorr_rows(unit, storage)         correlation of all rows, in place
#ifndef PCXO_MDSTORAGE_HPP
#define PCXO_MDSTORAGE_HPP

#include "fft.hpp"
#include "fxcorr.hpp"

#include <array>
#include <numeric>

namespace pcxo::md {

enum class layout {
    left,     // first declared axis most contiguous
    right     // last declared axis most contiguous
};

template<layout Layout, auto... Axes>
struct basis {
    static constexpr uZ     size       = sizeof...(Axes);
    static constexpr layout layout_tag = Layout;

    std::array<uZ, size> extents{};    // declaration order (static storage only)

    constexpr basis() = default;
    template<std::unsigned_integral... U>
        requires(sizeof...(U) == size)
    constexpr explicit basis(U... e)
    : extents{static_cast<uZ>(e)...} {}

    // declaration index of axis A
    template<auto A>
    static constexpr auto index_of() -> uZ {
        uZ   idx = 0, found = size;
        auto chk = [&](auto v) {
            if constexpr (std::same_as<decltype(v), decltype(A)>) {
                if (found == size && v == A) found = idx;
            }
            ++idx;
        };
        (chk(Axes), ...);
        return found;
    }
    template<auto A>
    static constexpr bool contains() {
        return index_of<A>() < size;
    }
    // position in layout order (0 = innermost) of declaration index d
    static constexpr auto layout_pos(uZ d) -> uZ { return Layout == layout::left ? d : size - 1 - d; }
};
template<auto... Axes>
using left_basis = basis<layout::left, Axes...>;
template<auto... Axes>
using right_basis = basis<layout::right, Axes...>;

// A view over some of the axes of a storage: extents and strides in layout
// order ([0] is the innermost axis when present).
template<typename T, uZ PackSize, uZ Rank, typename B>
class sslice {
public:
    sslice(T* ptr, std::array<uZ, Rank> ext, std::array<uZ, Rank> stride, std::array<uZ, Rank> decl, bool inner)
    : m_ptr(ptr)
    , m_ext(ext)
    , m_stride(stride)
    , m_decl(decl)
    , m_inner(inner) {}

    [[nodiscard]] auto data() const -> T* { return m_ptr; }
    [[nodiscard]] auto size() const -> uZ {
        uZ n = 1;
        for (auto e: m_ext) n *= e;
        return n;
    }
    // inner axis present and it is the only axis: usable as a packed vector
    [[nodiscard]] auto vector_like() const -> bool { return Rank == 1 && m_inner; }
    [[nodiscard]] auto extents() const -> const std::array<uZ, Rank>& { return m_ext; }
    [[nodiscard]] auto strides() const -> const std::array<uZ, Rank>& { return m_stride; }
    [[nodiscard]] auto decl_axes() const -> const std::array<uZ, Rank>& { return m_decl; }
    [[nodiscard]] auto has_inner() const -> bool { return m_inner; }

    [[nodiscard]] auto operator[](uZ i) const -> cx_ref<T, false, PackSize>
        requires(Rank == 1)
    {
        return cx_ref<T, false, PackSize>(m_ptr + (m_inner ? pidx<PackSize>(i) : i * m_stride[0]));
    }

    // remove the axis with declaration index d, fixing it at i
    template<auto Axis>
        requires(B::template contains<Axis>() && Rank > 1)
    [[nodiscard]] auto slice(uZ i) const -> sslice<T, PackSize, Rank - 1, B> {
        return slice_decl(B::template index_of<Axis>(), i);
    }

    template<uZ R = Rank>
        requires(R > 1)
    [[nodiscard]] auto slice_decl(uZ d, uZ i) const -> sslice<T, PackSize, Rank - 1, B> {
        std::array<uZ, Rank - 1> e{}, s{}, dd{};
        uZ                       p = Rank;
        for (uZ q = 0; q < Rank; ++q)
            if (m_decl[q] == d) p = q;
        if (p == Rank) throw std::invalid_argument("axis not present in this slice");
        if (i >= m_ext[p]) throw std::out_of_range("slice index out of range");
        const bool inner_here = m_inner && p == 0;
        T*         ptr        = m_ptr + (inner_here ? pidx<PackSize>(i) : m_stride[p] * i);
        for (uZ q = 0, o = 0; q < Rank; ++q) {
            if (q == p) continue;
            e[o]  = m_ext[q];
            s[o]  = m_stride[q];
            dd[o] = m_decl[q];
            ++o;
        }
        return {ptr, e, s, dd, m_inner && p != 0};
    }

private:
    T*                   m_ptr;
    std::array<uZ, Rank> m_ext;
    std::array<uZ, Rank> m_stride;
    std::array<uZ, Rank> m_decl;
    bool                 m_inner;
};

template<typename T,
         auto Basis,
         uZ   PackSize      = default_pack_size<T>,
         uZ   Alignment     = default_pack_size<T>,
         typename Allocator = managed_allocator<T>>
class dynamic_storage {
    using B                 = std::remove_cvref_t<decltype(Basis)>;
    static constexpr uZ N   = B::size;
    static constexpr uZ ALN = std::lcm(PackSize * 2, Alignment);
    using alloc_traits      = std::allocator_traits<Allocator>;

public:
    using real_type = T;
    static constexpr uZ pack_size = PackSize;

    // extents in declaration order
    template<std::unsigned_integral... U>
        requires(sizeof...(U) == N)
    explicit dynamic_storage(U... extents)
    : dynamic_storage(Allocator{}, extents...) {}

    template<std::unsigned_integral... U>
        requires(sizeof...(U) == N)
    explicit dynamic_storage(Allocator alloc, U... extents)
    : m_alloc(std::move(alloc)) {
        const std::array<uZ, N> decl{static_cast<uZ>(extents)...};
        for (uZ d = 0; d < N; ++d) m_ext[B::layout_pos(d)] = decl[d];
        // calc_storage_size (mdstorage.hpp:857-863): padded inner row times outer extents
        m_row  = (m_ext[0] * 2 + ALN - 1) / ALN * ALN;
        m_size = m_row;
        for (uZ i = 1; i < N; ++i) m_size *= m_ext[i];
        m_ptr = m_size ? alloc_traits::allocate(m_alloc, m_size) : nullptr;
        if (m_ptr) {
            detail_::check_cuda(cudaMemset(m_ptr, 0, m_size * sizeof(T)));
            detail_::check_cuda(cudaDeviceSynchronize());
        }
    }
    dynamic_storage(const dynamic_storage&)            = delete;
    dynamic_storage& operator=(const dynamic_storage&) = delete;
    dynamic_storage(dynamic_storage&& o) noexcept
    : m_alloc(std::move(o.m_alloc))
    , m_ext(o.m_ext)
    , m_row(o.m_row)
    , m_size(o.m_size)
    , m_ptr(std::exchange(o.m_ptr, nullptr)) {}
    ~dynamic_storage() {
        if (m_ptr) alloc_traits::deallocate(m_alloc, m_ptr, m_size);
    }

    template<auto Axis>
        requires(B::template contains<Axis>())
    [[nodiscard]] auto extent() const noexcept -> uZ {
        return m_ext[B::layout_pos(B::template index_of<Axis>())];
    }
    [[nodiscard]] auto data() noexcept -> T* { return m_ptr; }
    [[nodiscard]] auto data() const noexcept -> const T* { return m_ptr; }
    [[nodiscard]] auto storage_size() const noexcept -> uZ { return m_size; }
    // reals between consecutive inner rows
    [[nodiscard]] auto row_stride() const noexcept -> uZ { return m_row; }
    // number of inner rows (product of the outer extents)
    [[nodiscard]] auto rows() const noexcept -> uZ { return m_row ? m_size / m_row : 0; }
    [[nodiscard]] auto inner_extent() const noexcept -> uZ { return m_ext[0]; }

    [[nodiscard]] auto as_slice() const -> sslice<T, PackSize, N, B> {
        std::array<uZ, N> stride{}, decl{};
        // layout axis q >= 1 advances by the padded row times the extents inside it
        uZ s = m_row;
        for (uZ q = 1; q < N; ++q) {
            stride[q] = s;
            s *= m_ext[q];
        }
        stride[0] = 1;
        for (uZ d = 0; d < N; ++d) decl[B::layout_pos(d)] = d;
        return {m_ptr, m_ext, stride, decl, true};
    }
    // slice<Axis>(i): the storage with Axis fixed at i (mdstorage.hpp:370-391)
    template<auto Axis>
        requires(B::template contains<Axis>() && N > 1)
    [[nodiscard]] auto slice(uZ i) const -> sslice<T, PackSize, N - 1, B> {
        return as_slice().slice_decl(B::template index_of<Axis>(), i);
    }

private:
    [[no_unique_address]] Allocator m_alloc;
    std::array<uZ, N>               m_ext{};    // layout order
    uZ                              m_row  = 0;
    uZ                              m_size = 0;
    T*                              m_ptr  = nullptr;
};

// ---- batched GPU calls over the inner rows ---------------------------------
template<typename Unit, typename Storage>
void fft_rows(Unit& unit, Storage& s) {
    if (s.inner_extent() != unit.size()) {
        throw std::invalid_argument(std::string("input size (which is ") + std::to_string(s.inner_extent()) +
                                    ") is not equal to fft size (which is " + std::to_string(unit.size()) + ")");
    }
    unit.template fft_batch<Storage::pack_size>(s.data(), s.data(), s.rows(), s.row_stride(), s.row_stride());
}
template<bool Normalized = true, typename Unit, typename Storage>
void ifft_rows(Unit& unit, Storage& s) {
    if (s.inner_extent() != unit.size()) {
        throw std::invalid_argument(std::string("input size (which is ") + std::to_string(s.inner_extent()) +
                                    " is not equal to fft size (which is " + std::to_string(unit.size()) + ")");
    }
    unit.template ifft_batch<Normalized, Storage::pack_size>(s.data(), s.data(), s.rows(), s.row_stride(),
                                                              s.row_stride());
}
template<typename Unit, typename Storage>
void fxcorr_rows(Unit& unit, Storage& s) {
    unit.template correlate<Storage::pack_size>(s.data(), s.data(), s.inner_extent(), s.rows(), s.row_stride(),
                                                s.row_stride());
}

}    // namespace pcxo::md

namespace pcxo {
// A one-axis slice whose axis is the inner one is a packed vector.
template<typename T, uZ P, typename B>
struct cx_vector_traits<md::sslice<T, P, 1, B>> {
    using real_type               = T;
    static constexpr uZ pack_size = P;
    static auto re_data(const md::sslice<T, P, 1, B>& v) -> T* {
        if (!v.vector_like()) throw std::invalid_argument("slice is not contiguous along the inner axis");
        return v.data();
    }
    static auto size(const md::sslice<T, P, 1, B>& v) -> uZ { return v.extents()[0]; }
};
}    // namespace pcxo
#endif
