// pcxo/fxcorr.hpp — drop-in for pcxo::fxcorr_unit (reference fxcorr.hpp:10-147)
// on the GPU: the overlap-save correlation y[n] = sum_{j<K} x[n+j] conj(g[j])
// runs as one fused kernel per call (forward FFT, conj(K) product, inverse,
// per block).  Constructors and operator() keep the reference's signatures;
// the FFT unit and scratch factory parameters are accepted for source
// compatibility (the GPU kernel keeps its block spectra on chip, so no
// scratch vector is used).  operator()(dest, src), empty in the reference,
// is implemented.  Calls are synchronous.
#ifndef PCXO_FXCORR_HPP
#define PCXO_FXCORR_HPP

#include "fft.hpp"

#include <memory>

namespace pcxo {

namespace detail_ {
template<typename T, typename Allocator = managed_allocator<T>>
class pseudo_vector_factory {
public:
    explicit pseudo_vector_factory(uZ size, const Allocator& allocator = Allocator{})
    : m_vector(size, allocator) {}
    pseudo_vector_factory(const pseudo_vector_factory&)            = delete;
    pseudo_vector_factory& operator=(const pseudo_vector_factory&) = delete;
    auto* operator()() { return &m_vector; }

private:
    pcxo::vector<T, default_pack_size<T>, Allocator> m_vector;
};
}    // namespace detail_

template<typename T,
         typename Allocator   = managed_allocator<T>,
         typename FFT_        = fft_unit<T, fft_order::unordered, Allocator>,
         typename TmpFactory_ = detail_::pseudo_vector_factory<T, Allocator>>
    requires(std::floating_point<T> && std::same_as<typename Allocator::value_type, T>)
class fxcorr_unit {
public:
    using real_type      = T;
    using allocator_type = Allocator;

    fxcorr_unit() = delete;
    template<uZ PG, typename GA>
    fxcorr_unit(const pcxo::vector<T, PG, GA>& g, uZ fft_size, allocator_type = allocator_type{})
    : m_n(fft_size) {
        init(g.data(), g.size(), PG);
    }
    template<uZ PG, typename GA>
    fxcorr_unit(const pcxo::vector<T, PG, GA>& g, std::shared_ptr<FFT_> fft_unit, allocator_type = allocator_type{})
    : m_n(fft_unit->size()) {
        init(g.data(), g.size(), PG);
    }
    template<uZ PG, typename GA>
    fxcorr_unit(const pcxo::vector<T, PG, GA>& g, std::shared_ptr<FFT_> fft_unit, TmpFactory_,
                allocator_type = allocator_type{})
    : m_n(fft_unit->size()) {
        init(g.data(), g.size(), PG);
    }

    fxcorr_unit(const fxcorr_unit&)     = default;
    fxcorr_unit(fxcorr_unit&&) noexcept = default;
    fxcorr_unit& operator=(const fxcorr_unit&)     = delete;
    fxcorr_unit& operator=(fxcorr_unit&&) noexcept = delete;

    void set_stream(cudaStream_t s) { m_stream = s; }

    // In place (fxcorr.hpp:102-136).
    template<typename Vect_>
        requires complex_vector_of<T, Vect_>
    void operator()(Vect_& vector) {
        using tr = cx_vector_traits<Vect_>;
        const uZ                n = tr::size(vector);
        detail_::device_view<T> v(tr::re_data(vector), detail_::real_size(n, tr::pack_size), true);
        const uZ                row = detail_::real_size(n, tr::pack_size);
        detail_::check(pcx_fxcorr_exec(m_h.get(), v.get(), v.get(), n, (int)tr::pack_size, 1, row, row, m_stream));
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_fxcorr_status(m_h.get()));
        v.commit();
    }

    // Out of place (the reference's overload is empty, fxcorr.hpp:138-140).
    template<typename DestVect_, typename SrcVect_>
        requires complex_vector_of<T, DestVect_> && complex_vector_of<T, SrcVect_>
    void operator()(DestVect_& dest, const SrcVect_& source) {
        using dt = cx_vector_traits<DestVect_>;
        using st = cx_vector_traits<SrcVect_>;
        static_assert(dt::pack_size == st::pack_size, "source and destination pack sizes must match");
        const uZ n = st::size(source);
        if (dt::size(dest) != n) throw std::invalid_argument("destination size is not equal to source size");
        const uZ                row = detail_::real_size(n, st::pack_size);
        detail_::device_view<T> d(dt::re_data(dest), row, false);
        detail_::device_view<T> s(const_cast<T*>(st::re_data(source)), row, true);
        detail_::check(pcx_fxcorr_exec(m_h.get(), d.get(), s.get(), n, (int)st::pack_size, 1, row, row, m_stream));
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_fxcorr_status(m_h.get()));
        d.commit();
    }

    // Batched extension: `channels` device rows of `len` elements.
    template<uZ PackSize = default_pack_size<T>>
    void correlate(T* dest, const T* source, uZ len, uZ channels, uZ dest_stride = 0, uZ src_stride = 0) {
        const uZ row = detail_::real_size(len, PackSize);
        detail_::check(pcx_fxcorr_exec(m_h.get(), dest, source, len, (int)PackSize, channels,
                                       dest_stride ? dest_stride : row, src_stride ? src_stride : row, m_stream));
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_fxcorr_status(m_h.get()));
    }

    // Adjoint: gx = d loss/dx (convolution of gy with g); gg (optional) = d loss/dg.
    template<uZ PackSize = default_pack_size<T>>
    void vjp(T* gx, T* gg, const T* gy, const T* x, uZ len, uZ channels = 1) {
        const uZ row = detail_::real_size(len, PackSize);
        detail_::check(pcx_fxcorr_vjp(m_h.get(), gx, gg, gy, x, len, (int)PackSize, channels, row, m_stream));
        detail_::check_cuda(cudaStreamSynchronize(m_stream));
        detail_::check(pcx_fxcorr_status(m_h.get()));
    }

private:
    void init(const T* g, uZ k, uZ pack_g) {
        detail_::device_view<T> gv(const_cast<T*>(g), detail_::real_size(k, pack_g), true);
        pcx_fxcorr h = nullptr;
        detail_::check(pcx_fxcorr_create(&h, gv.get(), k, (int)pack_g, m_n, detail_::dtype_code<T>()));
        m_h = std::shared_ptr<pcx_fxcorr_s>(h, [](pcx_fxcorr p) { pcx_fxcorr_destroy(p); });
    }

    uZ                            m_n;
    std::shared_ptr<pcx_fxcorr_s> m_h;
    cudaStream_t                  m_stream = nullptr;
};

}    // namespace pcxo
#endif
