// pcxo/ragged.hpp — many FFTs of uneven power-of-two sizes and overlap-save
// correlations in ONE persistent GPU launch (pcx_ragged_*).  No counterpart in
// the reference, which runs one transform per fft_unit call: this is the batch
// form of fft_unit<float> (natural order, pack 8) and fxcorr_unit<float>
// (out of place), built once from the buffers it will work on and replayed
// from a CUDA graph by each call.
//
//   pcxo::ragged_batch batch;
//   batch.add_fft(dst, src);                 // pcxo::vector<float> (or rows)
//   batch.add_xcorr(y, x, g, fft_size);      // y, x signal vectors, g kernel taps (all pack 8)
//   batch.build();                           // plans, tables, work queue, graph
//   batch();                                 // one replay, synchronous
//
// Every buffer must reach the GPU (device or managed memory, as pcxo::vector's
// default allocator gives) and be 16-byte aligned; its storage is used in
// place, so the objects must outlive the batch.  All FFTs are forward, or all
// inverse (normalised: then of one size).  With tensor_core (0 bf16 x3,
// 1 tf32 x3, 2 bf16 x6) the transforms of 2^8..2^12 points run in the
// tensor-core form, a second persistent launch in the same graph.
#ifndef PCXO_RAGGED_HPP
#define PCXO_RAGGED_HPP

#include "vector.hpp"

#include <memory>
#include <vector>

namespace pcxo {

/**
 * FFT size for an overlap-save correlation with a k-tap kernel: the power of
 * two N >= k + 7 that minimises the transform work per output sample,
 * 2 N log2(N) / (N - k + 1) (a forward and an inverse transform per block of
 * N - k + 1 outputs), over 128 <= N <= max_size; sizes above 8192 only for
 * kernels of more than 4096 taps.  The same model as the Python
 * packed_b200.correlation_fft_size.
 */
inline uZ correlation_fft_size(uZ k, uZ max_size = 16384) {
    uZ     best      = 0;
    double best_cost = 0;
    for (uZ n = 128, lg = 7; n <= max_size; n *= 2, ++lg) {
        if (n >= k + 7 && (n <= 8192 || k > 4096)) {
            const double cost = 2.0 * double(n) * double(lg) / double(n - k + 1);
            if (best == 0 || cost < best_cost) {
                best      = n;
                best_cost = cost;
            }
        }
    }
    if (best == 0) {
        throw std::invalid_argument("kernel size (which is " + std::to_string(k) + ") needs an FFT size above " +
                                    std::to_string(max_size));
    }
    return best;
}

class ragged_batch {
public:
    explicit ragged_batch(bool inverse = false, bool normalized = true, int tensor_core = -1)
    : m_inverse(inverse)
    , m_normalized(normalized)
    , m_tensor_core(tensor_core) {}
    ragged_batch(const ragged_batch&)            = delete;
    ragged_batch& operator=(const ragged_batch&) = delete;

    /** One transform of dst.size() points (a power of two in 2^5..2^18), src -> dst. */
    template<typename A1, typename A2>
    void add_fft(pcxo::vector<float, 8, A1>& dst, const pcxo::vector<float, 8, A2>& src) {
        if (dst.size() != src.size()) {
            throw std::invalid_argument("ragged FFT: source size (which is " + std::to_string(src.size()) +
                                        ") is not equal to destination size (which is " +
                                        std::to_string(dst.size()) + ")");
        }
        add_fft_raw(dst.data(), src.data(), dst.size());
    }
    /** Raw form: n points, pack-8 split-complex rows at device-reachable pointers. */
    void add_fft_raw(float* dst, const float* src, uZ n) {
        unbuild();
        m_sizes.push_back(n);
        m_dst.push_back(dst);
        m_src.push_back(src);
    }
    /** y[n] = sum_{j<K} x[n+j] conj(g[j]) over x.size() samples, overlap-save with fft_size points
     *  (a power of two in 2^7..2^14, at least K + 7; correlation_fft_size(K) gives a good one). */
    template<typename A1, typename A2, typename A3>
    void add_xcorr(pcxo::vector<float, 8, A1>& y, const pcxo::vector<float, 8, A2>& x,
                   const pcxo::vector<float, 8, A3>& g, uZ fft_size) {
        if (y.size() != x.size()) {
            throw std::invalid_argument("ragged correlation: output size (which is " + std::to_string(y.size()) +
                                        ") is not equal to signal size (which is " + std::to_string(x.size()) +
                                        ")");
        }
        unbuild();
        m_xlen.push_back(x.size());
        m_xk.push_back(g.size());
        m_xg.push_back(g.data());
        m_xn.push_back(fft_size);
        m_xdst.push_back(y.data());
        m_xsrc.push_back(x.data());
    }

    /** Plans, tables, the work queue and its graph (done by the first call if not before). */
    void build() {
        if (m_handle) return;
        pcx_ragged h = nullptr;
        detail_::check(pcx_ragged_create_tc(&h, PCX_F32, m_sizes.size(), m_sizes.data(), m_dst.data(),
                                            m_src.data(), m_inverse ? PCX_INVERSE : PCX_FORWARD, m_normalized ? 1 : 0,
                                            m_xlen.size(), m_xlen.data(), m_xk.data(), m_xg.data(), m_xn.data(),
                                            m_xdst.data(), m_xsrc.data(), m_tensor_core));
        m_handle.reset(h, [](pcx_ragged q) { pcx_ragged_destroy(q); });
    }

    /** One replay of the batch on `stream`, then waits for it; throws if a work item gave up waiting. */
    void operator()(cudaStream_t stream = nullptr) {
        build();
        detail_::check(pcx_ragged_exec(m_handle.get(), stream));
        detail_::check_cuda(cudaStreamSynchronize(stream));
        detail_::check(pcx_ragged_status(m_handle.get()));
    }

    /** Work items in the device queue (after build()). */
    [[nodiscard]] uZ items() const { return m_handle ? pcx_ragged_items(m_handle.get()) : 0; }
    [[nodiscard]] uZ fft_count() const { return m_sizes.size(); }
    [[nodiscard]] uZ xcorr_count() const { return m_xlen.size(); }

private:
    void unbuild() { m_handle.reset(); }

    bool                                               m_inverse;
    bool                                               m_normalized;
    int                                                m_tensor_core;
    std::vector<std::size_t>                           m_sizes;
    std::vector<void*>                                 m_dst;
    std::vector<const void*>                           m_src;
    std::vector<std::size_t>                           m_xlen, m_xk, m_xn;
    std::vector<const void*>                           m_xg;
    std::vector<void*>                                 m_xdst;
    std::vector<const void*>                           m_xsrc;
    std::shared_ptr<std::remove_pointer_t<pcx_ragged>> m_handle;
};

}    // namespace pcxo

#endif
