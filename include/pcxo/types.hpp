// pcxo/types.hpp — drop-in for the reference's scalar types, pack-size
// concepts and the cx_vector_traits customisation point (reference
// inc/types.hpp:11-154, inc/element_access.hpp:8-11, 413-485), plus the
// allocators whose memory the GPU can reach.
#ifndef PCXO_TYPES_HPP
#define PCXO_TYPES_HPP

#include "../pcx_cuda.h"

#include <complex>
#include <cstddef>
#include <cstdint>
#include <new>
#include <ranges>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

namespace pcxo {

using f32 = float;
using f64 = double;
using uZ  = std::size_t;
using iZ  = std::ptrdiff_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;

template<uZ N>
concept pack_size = N > 0 && (N & (N - 1)) == 0;

template<typename T>
concept floating_point = std::same_as<T, float> || std::same_as<T, double>;

template<typename T, uZ PackSize>
concept packed_floating_point = floating_point<T> && pack_size<PackSize>;

// 32 bytes of reals per pack: 8 floats / 4 doubles (types.hpp:70-72).
template<typename T>
    requires floating_point<T>
constexpr const uZ default_pack_size = 32 / sizeof(T);

constexpr uZ dynamic_size = 0;

// Packed index of element idx (element_access.hpp:8-11).
template<uZ PackSize>
constexpr auto pidx(uZ idx) -> uZ {
    return idx + idx / PackSize * PackSize;
}

namespace detail_ {
[[noreturn]] inline void throw_status(int rc) {
    const char* msg = pcx_last_error();
    if (rc == PCX_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(std::string("pcx_cuda: ") + msg);
}
inline void check(int rc) {
    if (rc != PCX_OK) throw_status(rc);
}
inline void check_cuda(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}
// True when the GPU can dereference p directly (device or managed memory).
inline bool device_accessible(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template<typename T>
struct is_std_complex : std::false_type {};
template<typename T>
struct is_std_complex<std::complex<T>> : std::true_type {
    using real_type = T;
};
}    // namespace detail_

/**
 * Memory reachable from host and GPU alike (cudaMallocManaged), 256-byte
 * aligned.  pcxo::vector uses it by default so that element access on the
 * host and transforms on the GPU work on the same storage.
 */
template<typename T>
class managed_allocator {
public:
    using value_type      = T;
    using is_always_equal = std::true_type;

    managed_allocator() noexcept = default;
    template<typename U>
    explicit managed_allocator(const managed_allocator<U>&) noexcept {}

    [[nodiscard]] auto allocate(uZ n) -> T* {
        void* p = nullptr;
        if (cudaMallocManaged(&p, n * sizeof(T) > 0 ? n * sizeof(T) : 1) != cudaSuccess) {
            (void)cudaGetLastError();
            throw std::bad_alloc();
        }
        return static_cast<T*>(p);
    }
    void deallocate(T* p, uZ) noexcept { cudaFree(p); }

    template<typename U>
    struct rebind {
        using other = managed_allocator<U>;
    };
};
template<typename T, typename U>
bool operator==(const managed_allocator<T>&, const managed_allocator<U>&) noexcept {
    return true;
}

/**
 * Device-only memory (cudaMalloc): fastest for data that never needs element
 * access from the host; transfer with cudaMemcpy.
 */
template<typename T>
class device_allocator {
public:
    using value_type      = T;
    using is_always_equal = std::true_type;

    device_allocator() noexcept = default;
    template<typename U>
    explicit device_allocator(const device_allocator<U>&) noexcept {}

    [[nodiscard]] auto allocate(uZ n) -> T* {
        void* p = nullptr;
        if (cudaMalloc(&p, n * sizeof(T) > 0 ? n * sizeof(T) : 1) != cudaSuccess) {
            (void)cudaGetLastError();
            throw std::bad_alloc();
        }
        return static_cast<T*>(p);
    }
    void deallocate(T* p, uZ) noexcept { cudaFree(p); }

    template<typename U>
    struct rebind {
        using other = device_allocator<U>;
    };
};
template<typename T, typename U>
bool operator==(const device_allocator<T>&, const device_allocator<U>&) noexcept {
    return true;
}

// The reference's default allocator name (allocators.hpp:11-48).  It hands
// out managed memory so existing code runs on the GPU unchanged; CUDA aligns
// every managed allocation to at least 256 bytes, so any Alignment up to 256
// (the reference's default is 64) is met, and larger ones are rejected at
// compile time.
template<typename T, std::align_val_t Alignment = std::align_val_t{64}>
class aligned_allocator : public managed_allocator<T> {
    static_assert(static_cast<std::size_t>(Alignment) <= 256 &&
                      (static_cast<std::size_t>(Alignment) & (static_cast<std::size_t>(Alignment) - 1)) == 0,
                  "aligned_allocator: managed memory is aligned to 256 bytes; Alignment must be a power of two <= 256");

public:
    aligned_allocator() noexcept = default;
    template<typename U>
    aligned_allocator(const aligned_allocator<U, Alignment>&) noexcept {}

    template<typename U>
    struct rebind {
        using other = aligned_allocator<U, Alignment>;
    };
};

/**
 * Customisation point (types.hpp:113-148): real_type, pack_size,
 * re_data(v) -> T*, size(v).  Specialised for pcxo::vector and for
 * contiguous ranges of std::complex<T> (pack size 1).
 */
template<typename V>
struct cx_vector_traits {
    using real_type               = void;
    static constexpr uZ pack_size = 0;
};

template<typename R>
    requires std::ranges::contiguous_range<R> && detail_::is_std_complex<std::ranges::range_value_t<R>>::value
struct cx_vector_traits<R> {
    using real_type               = typename detail_::is_std_complex<std::ranges::range_value_t<R>>::real_type;
    static constexpr uZ pack_size = 1;

    static auto re_data(R& v) -> real_type* { return reinterpret_cast<real_type*>(std::ranges::data(v)); }
    static auto re_data(const R& v) -> const real_type* {
        return reinterpret_cast<const real_type*>(std::ranges::data(v));
    }
    static auto size(const R& v) -> uZ { return std::ranges::size(v); }
};

template<typename V>
concept complex_vector = cx_vector_traits<std::remove_cvref_t<V>>::pack_size != 0;

template<typename T, typename V>
concept complex_vector_of = std::same_as<T, typename cx_vector_traits<std::remove_cvref_t<V>>::real_type>;

}    // namespace pcxo

namespace pcx = pcxo;

#endif
