// pcxo/fft.hpp — drop-in for pcxo::fft_unit (reference fft.hpp:540-2166)
// running on the GPU through libpcx_cuda.so.
//
// Same template parameters, constructors, method names, argument meanings
// and exceptions as the reference.  Calls are synchronous, as the
// reference's are: each returns after the GPU work has finished, so data may
// be read on the host straight away.  Data in device or managed memory is
// transformed in place on the GPU; data in ordinary host memory (e.g. a
// std::vector<std::complex<T>>) is staged through a device buffer.
// Differences from the reference, by design:
//   * ifft<false> in normal order returns the unnormalised inverse (the
//     reference normalises regardless, fft.hpp:851);
//   * the out-of-place ifft(dest, src) is the correct inverse in every order
//     (the reference's is not, fft.hpp:863-915);
//   * sub_size is validated but only a hint: the GPU picks its own schedule.
#ifndef PCXO_FFT_HPP
#define PCXO_FFT_HPP

#include "types.hpp"
#include "vector.hpp"

#include <memory>
#include <ranges>
#include <vector>

namespace pcxo {

enum class fft_order {
    normal,
    bit_reversed,
    unordered
};

// Strategy tags of the reference's CPU recursion (fft.hpp:546-563); accepted
// for source compatibility, no effect on the GPU.
struct strategy42 {};
struct strategy48 {};
struct strategy8 {};

namespace detail_ {
template<typename T>
constexpr int dtype_code() {
    return std::same_as<T, double> ? PCX_F64 : PCX_F32;
}

// A device view of caller data: the pointer itself when the GPU can reach
// it, otherwise a staged device copy that is written back on commit().
template<typename T>
class device_view {
public:
    device_view(T* host, uZ reals, bool copy_in)
    : m_host(host)
    , m_reals(reals) {
        if (device_accessible(host)) {
            m_dev = host;
            return;
        }
        check_cuda(cudaMalloc(&m_dev, reals * sizeof(T)));
        m_owned = true;
        if (copy_in) check_cuda(cudaMemcpy(m_dev, host, reals * sizeof(T), cudaMemcpyHostToDevice));
    }
    device_view(const device_view&)            = delete;
    device_view& operator=(const device_view&) = delete;
    ~device_view() {
        if (m_owned) cudaFree(m_dev);
    }
    T*   get() const { return static_cast<T*>(m_dev); }
    void commit() const {
        if (m_owned) check_cuda(cudaMemcpy(m_host, m_dev, m_reals * sizeof(T), cudaMemcpyDeviceToHost));
    }

private:
    T*    m_host;
    uZ    m_reals;
    void* m_dev   = nullptr;
    bool  m_owned = false;
};

constexpr uZ real_size(uZ n, uZ p) { return (n + p - 1) / p * 2 * p; }
}    // namespace detail_

template<typename T,
         fft_order Order      = fft_order::normal,
         typename Allocator   = managed_allocator<T>,
         uZ SubSize           = dynamic_size,
         uZ NodeSizeRec       = 4,
         typename Strategy    = strategy42,
         typename StrategyRec = strategy42>
    requires(std::same_as<T, float> || std::same_as<T, double>)
class fft_unit {
public:
    using real_type      = T;
    using allocator_type = Allocator;

    explicit fft_unit(uZ fft_size, allocator_type allocator = allocator_type())
        requires(SubSize != dynamic_size)
    : fft_unit(fft_size, SubSize, allocator, 0) {}

    explicit fft_unit(uZ fft_size, uZ sub_size = 2048, allocator_type allocator = allocator_type())
        requires(SubSize == dynamic_size)
    : fft_unit(fft_size, sub_size, allocator, 0) {}

    fft_unit(const fft_unit& other)
    : fft_unit(other.m_size, other.m_sub_size, other.m_alloc, 0) {
        m_stream = other.m_stream;
    }
    fft_unit(fft_unit&& other) noexcept = default;
    ~fft_unit()                         = default;
    fft_unit& operator=(const fft_unit&)     = delete;
    fft_unit& operator=(fft_unit&&) noexcept = delete;

    [[nodiscard]] constexpr auto size() const -> uZ { return m_size; }

    // Stream the unit enqueues on (default: the legacy default stream).
    void set_stream(cudaStream_t s) { m_stream = s; }

    // ---- raw pointer forms (fft.hpp:624-721)
    template<uZ PackSize = 1>
        requires pack_size<PackSize>
    void fft_raw(T* data) {
        run(data, data, m_size, PackSize, PackSize, PCX_FORWARD, true);
    }
    template<uZ PackSizeDest = 1, uZ PackSizeSrc = 1>
        requires pack_size<PackSizeDest> && pack_size<PackSizeSrc>
    void fft_raw(T* dest, const T* source) {
        run(dest, source, m_size, PackSizeDest, PackSizeSrc, PCX_FORWARD, true);
    }
    template<uZ PackSizeDest = 1, uZ PackSizeSrc = 1>
        requires pack_size<PackSizeDest> && pack_size<PackSizeSrc>
    void fft_raw(T* dest, const T* source, uZ source_size) {
        run(dest, source, source_size, PackSizeDest, PackSizeSrc, PCX_FORWARD, true);
    }
    template<bool Normalized = true, uZ PackSize = 1>
        requires pack_size<PackSize>
    void ifft_raw(T* data) {
        run(data, data, m_size, PackSize, PackSize, PCX_INVERSE, Normalized);
    }
    template<bool Normalized = true, uZ PackSizeDest = 1, uZ PackSizeSrc = 1>
        requires pack_size<PackSizeDest> && pack_size<PackSizeSrc>
    void ifft_raw(T* dest, const T* source) {
        run(dest, source, m_size, PackSizeDest, PackSizeSrc, PCX_INVERSE, Normalized);
    }

    // ---- container forms (fft.hpp:728-915)
    template<typename Vect_>
        requires complex_vector_of<T, Vect_>
    void operator()(Vect_& vector) {
        using tr = cx_vector_traits<Vect_>;
        if (tr::size(vector) != m_size) {
            throw std::invalid_argument(std::string("input size (which is ") + std::to_string(tr::size(vector)) +
                                        ") is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        auto* p = tr::re_data(vector);
        run(p, p, m_size, tr::pack_size, tr::pack_size, PCX_FORWARD, true);
    }

    template<typename DestVect_, typename SrcVect_>
        requires complex_vector_of<T, DestVect_> && complex_vector_of<T, SrcVect_>
    void operator()(DestVect_& dest, const SrcVect_& source) {
        using st = cx_vector_traits<SrcVect_>;
        using dt = cx_vector_traits<DestVect_>;
        if (dt::size(dest) != m_size) {
            throw std::invalid_argument(std::string("destination size (which is ") + std::to_string(dt::size(dest)) +
                                        ") is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        if (st::size(source) > m_size) {
            throw std::invalid_argument(std::string("source size (which is ") + std::to_string(st::size(source)) +
                                        ") is bigger than fft size (which is " + std::to_string(m_size) + ")");
        }
        check_repack<dt::pack_size, st::pack_size>(dt::re_data(dest), st::re_data(source));
        run(dt::re_data(dest), st::re_data(source), st::size(source), dt::pack_size, st::pack_size, PCX_FORWARD,
            true);
    }

    template<bool Normalized = true, typename Vect_>
        requires complex_vector_of<T, Vect_>
    void ifft(Vect_& vector) {
        using tr = cx_vector_traits<Vect_>;
        if (tr::size(vector) != m_size) {
            throw std::invalid_argument(std::string("input size (which is ") + std::to_string(tr::size(vector)) +
                                        " is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        auto* p = tr::re_data(vector);
        run(p, p, m_size, tr::pack_size, tr::pack_size, PCX_INVERSE, Normalized);
    }

    template<bool Normalized = true, typename DestVect_, typename SrcVect_>
        requires complex_vector_of<T, DestVect_> && complex_vector_of<T, SrcVect_>
    void ifft(DestVect_& dest, const SrcVect_& source) {
        using st = cx_vector_traits<SrcVect_>;
        using dt = cx_vector_traits<DestVect_>;
        if (dt::size(dest) != m_size) {
            throw std::invalid_argument(std::string("destination size (which is ") + std::to_string(dt::size(dest)) +
                                        ") is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        if (st::size(source) != m_size) {
            throw std::invalid_argument(std::string("source size (which is ") + std::to_string(st::size(source)) +
                                        ") is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        check_repack<dt::pack_size, st::pack_size>(dt::re_data(dest), st::re_data(source));
        run(dt::re_data(dest), st::re_data(source), m_size, dt::pack_size, st::pack_size, PCX_INVERSE, Normalized);
    }

    // ---- batched extension: `batch` rows of `size()` elements, row stride in reals
    template<uZ PackSize = default_pack_size<T>>
    void fft_batch(T* dest, const T* source, uZ batch, uZ dest_stride = 0, uZ src_stride = 0) {
        exec_batch(dest, source, batch, PackSize, PCX_FORWARD, true, dest_stride, src_stride);
    }
    template<bool Normalized = true, uZ PackSize = default_pack_size<T>>
    void ifft_batch(T* dest, const T* source, uZ batch, uZ dest_stride = 0, uZ src_stride = 0) {
        exec_batch(dest, source, batch, PackSize, PCX_INVERSE, Normalized, dest_stride, src_stride);
    }

    // ---- tensor-core form (no reference counterpart, pcx_tc_fft_exec):
    // `batch` contiguous device rows of size() complex64 elements at pack 8,
    // natural order, 2^8 <= size() <= 2^16.  `precision` picks how each
    // DFT-matrix operand is split: bf16x6 (three bfloat16 parts, six
    // products) and tf32x3 stay within FP32-level error, bf16x3 does not.
    enum class tc_precision : int { bf16x3 = 0, tf32x3 = 1, bf16x6 = 2 };
    void fft_batch_tensor_core(T* dest, const T* source, uZ batch, tc_precision precision = tc_precision::bf16x6)
        requires std::same_as<T, float>
    {
        detail_::check(pcx_tc_fft_exec(m_plan.get(), dest, source, PCX_FORWARD, 1, batch, static_cast<int>(precision),
                                       m_stream));
        sync();
    }
    template<bool Normalized = true>
    void ifft_batch_tensor_core(T* dest, const T* source, uZ batch, tc_precision precision = tc_precision::bf16x6)
        requires std::same_as<T, float>
    {
        detail_::check(pcx_tc_fft_exec(m_plan.get(), dest, source, PCX_INVERSE, Normalized ? 1 : 0, batch,
                                       static_cast<int>(precision), m_stream));
        sync();
    }

    // ---- adjoint (no reference counterpart; pcx_fft_vjp).  Given g_out, the
    // cotangent of the output of fft_batch (inverse = false) or ifft_batch
    // (inverse = true, scaled as Normalized says), writes g_in, the cotangent
    // of that call's input: the forward DFT's adjoint is the unnormalised
    // inverse, the inverse's is the forward scaled as the inverse was.
    // `batch` device rows at pack PackSize, row stride in reals (0: packed).
    template<bool Normalized = true, uZ PackSize = default_pack_size<T>>
    void vjp(T* g_in, const T* g_out, uZ batch = 1, bool inverse = false, uZ stride = 0) {
        const uZ row = detail_::real_size(m_size, PackSize);
        detail_::check(pcx_fft_vjp(m_plan.get(), g_in, g_out, (int)PackSize, inverse ? PCX_INVERSE : PCX_FORWARD,
                                   Normalized ? 1 : 0, batch, stride ? stride : row, m_stream));
        sync();
    }

    // Handle of the underlying C-ABI plan.
    [[nodiscard]] auto plan() const -> pcx_plan { return m_plan.get(); }

private:
    fft_unit(uZ fft_size, uZ sub_size, allocator_type alloc, int)
    : m_size(fft_size)
    , m_sub_size(sub_size)
    , m_alloc(alloc) {
        pcx_plan p = nullptr;
        detail_::check(pcx_plan_create(&p, fft_size, detail_::dtype_code<T>(), static_cast<int>(Order), sub_size));
        m_plan.reset(p);
    }

    template<uZ PD, uZ PS>
    static void check_repack(const T* dst, const T* src) {
        constexpr uZ reg = 32 / sizeof(T);
        if constexpr (PS != PD && std::max(PS, PD) > reg) {
            if (static_cast<const void*>(dst) == static_cast<const void*>(src)) {
                throw std::invalid_argument(std::string("cannot perform in-place repack from source pack size (which is ") +
                                            std::to_string(PS) + ") to destination pack size (which is " +
                                            std::to_string(PD) + ")");
            }
        }
    }

    void run(T* dest, const T* source, uZ src_len, uZ pd, uZ ps, int dir, bool norm) {
        const uZ rd = detail_::real_size(m_size, pd);
        const uZ rs = detail_::real_size(src_len, ps);
        if (static_cast<const void*>(dest) == static_cast<const void*>(source)) {
            detail_::device_view<T> v(dest, std::max(rd, rs), true);
            detail_::check(pcx_fft_exec(m_plan.get(), v.get(), v.get(), src_len, (int)pd, (int)ps, dir, norm, 1, rd, rs,
                                        m_stream));
            sync();
            v.commit();
            return;
        }
        detail_::device_view<T> d(dest, rd, false);
        detail_::device_view<T> s(const_cast<T*>(source), rs, true);
        detail_::check(
            pcx_fft_exec(m_plan.get(), d.get(), s.get(), src_len, (int)pd, (int)ps, dir, norm, 1, rd, rs, m_stream));
        sync();
        d.commit();
    }

    void exec_batch(T* dest, const T* source, uZ batch, uZ p, int dir, bool norm, uZ ds, uZ ss) {
        const uZ row = detail_::real_size(m_size, p);
        ds           = ds ? ds : row;
        ss           = ss ? ss : row;
        detail_::check(pcx_fft_exec(m_plan.get(), dest, source, m_size, (int)p, (int)p, dir, norm, batch, ds, ss,
                                    m_stream));
        sync();
    }

    // Wait for the stream, then turn a bounded device wait that gave up
    // (rows left unwritten, pcx_plan_status) into an exception.
    void sync() {
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_plan_status(m_plan.get()));
    }

    struct plan_deleter {
        void operator()(pcx_plan p) const noexcept { pcx_plan_destroy(p); }
    };

    uZ                                           m_size;
    uZ                                           m_sub_size;
    [[no_unique_address]] allocator_type         m_alloc;
    std::unique_ptr<pcx_plan_s, plan_deleter>    m_plan;
    cudaStream_t                                 m_stream = nullptr;
};

// ---- transform across vectors (reference fft.hpp:2167-2572)
namespace detail_ {
template<typename R>
decltype(auto) range_vector(R&& elem) {
    if constexpr (std::is_pointer_v<std::remove_cvref_t<R>>) {
        return *elem;
    } else {
        return std::forward<R>(elem);
    }
}
}    // namespace detail_

template<typename T, typename R>
concept range_of_complex_vector_of =
    std::ranges::range<R> &&
    complex_vector_of<T, std::remove_pointer_t<std::remove_cvref_t<std::ranges::range_value_t<R>>>>;

// fft_unit_par(size)(dest, source): dest and source are ranges of `size`
// vectors of equal length L; for every element position p < L the size-point
// transform of source[0][p] .. source[size-1][p] goes to dest[0][p] ..
// dest[size-1][p].  The reference's version is broken (its own test is
// disabled, tests/test_fft.cpp:719-754); this one computes that definition.
template<typename T,
         fft_order Order     = fft_order::normal,
         typename Allocator  = managed_allocator<T>,
         uZ NodeSizeStrategy = 4>
    requires(std::same_as<T, float> || std::same_as<T, double>)
class fft_unit_par {
public:
    using real_type      = T;
    using allocator_type = Allocator;
    using size_type      = uZ;

    explicit fft_unit_par(uZ size, allocator_type allocator = allocator_type{})
    : m_size(size)
    , m_alloc(allocator) {
        pcx_plan p = nullptr;
        detail_::check(pcx_plan_create(&p, size, detail_::dtype_code<T>(), static_cast<int>(Order), 2048));
        m_plan.reset(p);
    }

    [[nodiscard]] auto size() const -> uZ { return m_size; }
    void               set_stream(cudaStream_t s) { m_stream = s; }

    template<typename DestR_, typename SrcR_>
        requires range_of_complex_vector_of<T, DestR_> && range_of_complex_vector_of<T, SrcR_>
    void operator()(DestR_& dest, const SrcR_& source) {
        using dv = std::remove_pointer_t<std::remove_cvref_t<std::ranges::range_value_t<DestR_>>>;
        using sv = std::remove_pointer_t<std::remove_cvref_t<std::ranges::range_value_t<SrcR_>>>;
        using dt = cx_vector_traits<dv>;
        using st = cx_vector_traits<sv>;
        const uZ nd = static_cast<uZ>(std::ranges::distance(dest));
        const uZ ns = static_cast<uZ>(std::ranges::distance(source));
        if (nd != m_size) {
            throw std::invalid_argument(std::string("destination size (which is ") + std::to_string(nd) +
                                        " is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        if (ns != m_size) {
            throw std::invalid_argument(std::string("source size (which is ") + std::to_string(ns) +
                                        " is not equal to fft size (which is " + std::to_string(m_size) + ")");
        }
        std::vector<void*>       dptr;
        std::vector<const void*> sptr;
        std::vector<std::unique_ptr<detail_::device_view<T>>> staged;
        uZ len = 0;
        bool first = true;
        for (auto&& e: dest) {
            auto&    v = detail_::range_vector(e);
            const uZ n = dt::size(v);
            if (first) len = n;
            first = false;
            if (n != len) throw std::invalid_argument("all vectors of a parallel transform have the same size");
            staged.push_back(std::make_unique<detail_::device_view<T>>(dt::re_data(v), detail_::real_size(n, dt::pack_size), false));
            dptr.push_back(staged.back()->get());
        }
        const uZ nstaged_dest = staged.size();
        for (auto&& e: source) {
            auto&    v = detail_::range_vector(e);
            if (st::size(v) != len) throw std::invalid_argument("all vectors of a parallel transform have the same size");
            staged.push_back(std::make_unique<detail_::device_view<T>>(const_cast<T*>(st::re_data(v)),
                                                                       detail_::real_size(len, st::pack_size), true));
            sptr.push_back(staged.back()->get());
        }
        detail_::check(pcx_fft_par_exec(m_plan.get(), dptr.data(), sptr.data(), m_size, len, (int)dt::pack_size,
                                        (int)st::pack_size, PCX_FORWARD, 0, m_stream));
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_plan_status(m_plan.get()));
        for (uZ i = 0; i < nstaged_dest; ++i) staged[i]->commit();
    }

private:
    struct plan_deleter {
        void operator()(pcx_plan p) const noexcept { pcx_plan_destroy(p); }
    };
    uZ                                        m_size;
    [[no_unique_address]] allocator_type      m_alloc;
    std::unique_ptr<pcx_plan_s, plan_deleter> m_plan;
    cudaStream_t                              m_stream = nullptr;
};

}    // namespace pcxo
#endif
