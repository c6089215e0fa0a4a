// pcxo/vector.hpp — drop-in for pcxo::vector (reference vector.hpp:26-382):
// an owning packed split-complex vector.  Storage holds ceil(n/P) packs of
// P reals followed by P imaginaries, zero-filled on construction; element i
// lives at data()[pidx<P>(i)] (real) and P reals further (imaginary).
#ifndef PCXO_VECTOR_HPP
#define PCXO_VECTOR_HPP

#include "types.hpp"
#include "vector_arithm.hpp"

#include <algorithm>
#include <cstring>
#include <iterator>
#include <memory>

namespace pcxo {

// Proxy reference to one packed element (reference element_access.hpp:306-400).
template<typename T, bool Const, uZ PackSize>
class cx_ref {
public:
    using real_pointer = std::conditional_t<Const, const T*, T*>;
    explicit cx_ref(real_pointer p) noexcept
    : m_ptr(p) {}

    [[nodiscard]] auto value() const -> std::complex<T> { return {m_ptr[0], m_ptr[PackSize]}; }
    operator std::complex<T>() const { return value(); }    // NOLINT(*explicit*)

    auto operator=(const std::complex<T>& v) const -> const cx_ref&
        requires(!Const)
    {
        m_ptr[0]        = v.real();
        m_ptr[PackSize] = v.imag();
        return *this;
    }
    template<typename U>
        requires std::is_arithmetic_v<U> && (!Const) && (!std::same_as<U, T>)
    auto operator=(const std::complex<U>& v) const -> const cx_ref& {
        return *this = std::complex<T>(static_cast<T>(v.real()), static_cast<T>(v.imag()));
    }
    template<typename U>
        requires std::is_arithmetic_v<U> && (!Const)
    auto operator=(U v) const -> const cx_ref& {
        return *this = std::complex<T>(static_cast<T>(v), 0);
    }
    auto operator=(const cx_ref& other) const -> const cx_ref&
        requires(!Const)
    {
        return *this = other.value();
    }

private:
    real_pointer m_ptr;
};

// Random-access iterator over packed elements (reference element_access.hpp:20-160).
template<typename T, bool Const, uZ PackSize>
class iterator {
public:
    using real_pointer      = std::conditional_t<Const, const T*, T*>;
    using difference_type   = std::ptrdiff_t;
    using value_type        = std::complex<T>;
    using reference         = cx_ref<T, Const, PackSize>;
    using iterator_category = std::random_access_iterator_tag;
    static constexpr uZ pack_size = PackSize;

    iterator() noexcept = default;
    iterator(real_pointer base, difference_type idx) noexcept
    : m_base(base)
    , m_idx(idx) {}

    auto operator*() const -> reference { return reference(m_base + pidx<PackSize>(static_cast<uZ>(m_idx))); }
    auto operator[](difference_type n) const -> reference { return *(*this + n); }
    auto operator++() -> iterator& {
        ++m_idx;
        return *this;
    }
    auto operator++(int) -> iterator {
        auto c = *this;
        ++m_idx;
        return c;
    }
    auto operator--() -> iterator& {
        --m_idx;
        return *this;
    }
    auto operator+=(difference_type n) -> iterator& {
        m_idx += n;
        return *this;
    }
    friend auto operator+(iterator it, difference_type n) -> iterator { return it += n; }
    friend auto operator-(iterator a, const iterator& b) -> difference_type { return a.m_idx - b.m_idx; }
    friend bool operator==(const iterator& a, const iterator& b) { return a.m_idx == b.m_idx && a.m_base == b.m_base; }
    auto        aligned() const -> bool { return m_idx % static_cast<difference_type>(PackSize) == 0; }
    auto        real_ptr() const -> real_pointer { return m_base + pidx<PackSize>(static_cast<uZ>(m_idx)); }

private:
    real_pointer    m_base = nullptr;
    difference_type m_idx  = 0;
};

template<typename T, uZ PackSize = default_pack_size<T>, typename Allocator = managed_allocator<T>>
    requires packed_floating_point<T, PackSize>
class vector {
    using alloc_traits = std::allocator_traits<Allocator>;

public:
    using real_type       = T;
    using real_pointer    = T*;
    using allocator_type  = Allocator;
    using size_type       = uZ;
    using reference       = cx_ref<T, false, PackSize>;
    using const_reference = cx_ref<T, true, PackSize>;
    using iterator        = pcxo::iterator<T, false, PackSize>;
    using const_iterator  = pcxo::iterator<T, true, PackSize>;
    static constexpr size_type pack_size = PackSize;

    vector() noexcept = default;
    explicit vector(size_type size, const allocator_type& allocator = allocator_type())
    : m_allocator(allocator)
    , m_size(size)
    , m_ptr(size ? alloc_traits::allocate(m_allocator, real_size(size)) : nullptr) {
        if (m_ptr) zero_reals(m_ptr, real_size(size));
    }
    template<typename U>
        requires std::is_convertible_v<U, std::complex<T>>
    vector(size_type size, U value, const allocator_type& allocator = allocator_type())
    : vector(size, allocator) {
        for (size_type i = 0; i < size; ++i) (*this)[i] = std::complex<T>(value);
    }
    vector(const vector& other)
    : vector(other.m_size, other.m_allocator) {
        if (m_ptr) copy_reals(m_ptr, other.m_ptr, real_size(m_size));
    }
    vector(vector&& other) noexcept
    : m_allocator(std::move(other.m_allocator))
    , m_size(std::exchange(other.m_size, 0))
    , m_ptr(std::exchange(other.m_ptr, nullptr)) {}
    ~vector() { deallocate(); }

    auto operator=(const vector& other) -> vector& {
        if (this != &other) {
            if (num_packs(other.m_size) != num_packs(m_size)) {
                deallocate();
                m_ptr = other.m_size ? alloc_traits::allocate(m_allocator, real_size(other.m_size)) : nullptr;
            }
            m_size = other.m_size;
            if (m_ptr) copy_reals(m_ptr, other.m_ptr, real_size(m_size));
        }
        return *this;
    }
    // v = expression: element-wise on the GPU (reference vector.hpp:177-182)
    template<typename E>
        requires detail_::vexpr_node<E>
    auto operator=(const E& expression) -> vector& {
        pcxo::assign(*this, expression);
        return *this;
    }
    auto operator=(vector&& other) noexcept -> vector& {
        if (this != &other) {
            deallocate();
            m_size = std::exchange(other.m_size, 0);
            m_ptr  = std::exchange(other.m_ptr, nullptr);
        }
        return *this;
    }

    [[nodiscard]] auto operator[](size_type idx) noexcept -> reference { return reference(m_ptr + packed_idx(idx)); }
    [[nodiscard]] auto operator[](size_type idx) const noexcept -> const_reference {
        return const_reference(m_ptr + packed_idx(idx));
    }
    [[nodiscard]] auto at(size_type idx) -> reference {
        if (idx >= size()) {
            throw std::out_of_range(std::string("idx (which is") + std::to_string(idx) +
                                    std::string(") >= vector size (which is ") + std::to_string(size()) +
                                    std::string(")"));
        }
        return (*this)[idx];
    }
    [[nodiscard]] auto data() noexcept -> real_pointer { return m_ptr; }
    [[nodiscard]] auto data() const noexcept -> const T* { return m_ptr; }
    [[nodiscard]] constexpr auto size() const noexcept -> size_type { return m_size; }
    [[nodiscard]] constexpr auto length() const noexcept -> size_type { return m_size; }
    [[nodiscard]] auto get_allocator() const -> allocator_type { return m_allocator; }

    void resize(size_type new_size) {
        if (num_packs(new_size) != num_packs(m_size)) {
            T* p = new_size ? alloc_traits::allocate(m_allocator, real_size(new_size)) : nullptr;
            if (p) {
                zero_reals(p, real_size(new_size));
                if (m_ptr) copy_reals(p, m_ptr, std::min(real_size(new_size), real_size(m_size)));
            }
            deallocate();
            m_ptr = p;
        }
        m_size = new_size;
    }

    auto begin() noexcept -> iterator { return iterator(m_ptr, 0); }
    auto end() noexcept -> iterator { return iterator(m_ptr, static_cast<std::ptrdiff_t>(m_size)); }
    auto begin() const noexcept -> const_iterator { return const_iterator(m_ptr, 0); }
    auto end() const noexcept -> const_iterator { return const_iterator(m_ptr, static_cast<std::ptrdiff_t>(m_size)); }

    static constexpr auto num_packs(size_type n) -> size_type { return (n + PackSize - 1) / PackSize; }
    static constexpr auto real_size(size_type n) -> size_type { return num_packs(n) * PackSize * 2; }
    static constexpr auto packed_idx(size_type idx) -> size_type { return idx + idx / PackSize * PackSize; }

private:
    static void zero_reals(T* p, size_type n) {
        if (detail_::device_accessible(p)) {
            detail_::check_cuda(cudaMemset(p, 0, n * sizeof(T)));
            detail_::check_cuda(cudaDeviceSynchronize());
        } else {
            std::memset(static_cast<void*>(p), 0, n * sizeof(T));
        }
    }
    static void copy_reals(T* dst, const T* src, size_type n) {
        if (n == 0) return;
        // works for host, managed and device storage alike
        detail_::check_cuda(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyDefault));
    }
    void deallocate() noexcept {
        if (m_ptr) alloc_traits::deallocate(m_allocator, m_ptr, real_size(m_size));
        m_ptr  = nullptr;
        m_size = 0;
    }

    [[no_unique_address]] allocator_type m_allocator{};
    size_type                            m_size = 0;
    real_pointer                         m_ptr  = nullptr;
};

template<typename T, uZ P, typename A>
struct cx_vector_traits<vector<T, P, A>> {
    using real_type               = T;
    static constexpr uZ pack_size = P;
    static auto re_data(vector<T, P, A>& v) -> T* { return v.data(); }
    static auto re_data(const vector<T, P, A>& v) -> const T* { return v.data(); }
    static auto size(const vector<T, P, A>& v) -> uZ { return v.size(); }
};

}    // namespace pcxo
#endif
