// Test infrastructure only: a C-ABI shim around the reference library's own
// headers (Dooez/packed, header-only C++/AVX2), compiled from the reference
// sources where they lie by oracle/Makefile into oracle/_ref/libpcx_ref.so.
// Nothing in the product links or loads this; tests and bench.py's CPU
// baseline leg use it as the checker / timed reference.
//
// Every entry point works on packed split-complex data at pack width 8
// (8 reals then 8 imaginaries per pack; element i at re[i + (i/8)*8],
// im at re + 8), the layout of pcxo::vector<float> (vector.hpp:26-382).
//
// The reference's fxcorr.hpp declares `friend auto ::conj` inside a class
// template, which GCC rejects as a private-member access (vector_arithm.hpp:1016),
// so the standard headers are pulled in first and `private` is widened for
// the reference headers only.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <ranges>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#define private public
#include "fft.hpp"
#include "fxcorr.hpp"
#undef private

namespace {

using fvec = pcxo::vector<float, 8, pcxo::aligned_allocator<float>>;

thread_local std::string g_err;

template<pcxo::fft_order Order>
int fft_inplace(std::size_t n, std::size_t sub, float* data, int dir, int norm) {
    auto unit = pcxo::fft_unit<float, Order>(n, sub);
    auto v    = fvec(n);
    std::memcpy(v.data(), data, sizeof(float) * 2 * n);
    if (dir == 0) {
        unit(v);
    } else if (norm) {
        unit.template ifft<true>(v);
    } else {
        unit.template ifft<false>(v);
    }
    std::memcpy(data, v.data(), sizeof(float) * 2 * n);
    return 0;
}

template<pcxo::fft_order Order>
int fft_oop(std::size_t n, std::size_t sub, float* dst, const float* src, std::size_t src_n, int dir,
            int norm) {
    auto unit = pcxo::fft_unit<float, Order>(n, sub);
    auto d    = fvec(n);
    auto s    = fvec(src_n);
    std::memcpy(s.data(), src, sizeof(float) * fvec::real_size(src_n));
    if (dir == 0) {
        unit(d, s);
    } else if (norm) {
        unit.template ifft<true>(d, s);
    } else {
        unit.template ifft<false>(d, s);
    }
    std::memcpy(dst, d.data(), sizeof(float) * 2 * n);
    return 0;
}

template<typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Overlap-save correlation with the reference's block loop (fxcorr.hpp:102-136)
// corrected: blocks start at packed index pidx<8>(offset) and whole elements are
// copied back.  The FFTs are the reference's own unordered fft_unit (the type
// fxcorr_unit uses, fxcorr.hpp:46) in its in-place forms, and the kernel
// spectrum is FFT(g)/N as in the fxcorr_unit constructor (fxcorr.hpp:62-69).
struct fixed_fxcorr {
    using fft_t = pcxo::fft_unit<float, pcxo::fft_order::unordered, pcxo::aligned_allocator<float>>;
    fft_t       fft;
    fvec        kernel;
    fvec        tmp;
    std::size_t overlap;

    fixed_fxcorr(const float* g, std::size_t k, std::size_t n)
    : fft(n, 2048)
    , kernel(n)
    , tmp(n)
    , overlap(k - 1) {
        auto gv = fvec(k);
        std::memcpy(gv.data(), g, sizeof(float) * fvec::real_size(k));
        fft(kernel, gv);
        auto* kp = kernel.data();
        for (std::size_t i = 0; i < 2 * n; ++i) {
            kp[i] /= static_cast<float>(n);
        }
    }

    void run(float* x, std::size_t s) {
        const std::size_t n    = fft.size();
        const std::size_t step = (n - overlap) / 8 * 8;
        std::size_t       off  = 0;
        while (off < s) {
            const std::size_t avail = std::min(n, s - off);
            std::memset(tmp.data(), 0, sizeof(float) * 2 * n);
            // copy whole elements of the block (zero-extended past the end)
            for (std::size_t i = 0; i < avail; ++i) {
                auto src                     = pcxo::pidx<8>(off + i);
                tmp.data()[pcxo::pidx<8>(i)]     = x[src];
                tmp.data()[pcxo::pidx<8>(i) + 8] = x[src + 8];
            }
            fft.template fft_raw<8>(tmp.data());
            float*       t  = tmp.data();
            const float* kp = kernel.data();
            for (std::size_t p = 0; p < n / 8; ++p) {
                for (std::size_t l = 0; l < 8; ++l) {
                    float ar = t[p * 16 + l], ai = t[p * 16 + 8 + l];
                    float br = kp[p * 16 + l], bi = -kp[p * 16 + 8 + l];
                    t[p * 16 + l]     = ar * br - ai * bi;
                    t[p * 16 + 8 + l] = ar * bi + ai * br;
                }
            }
            fft.template ifft_raw<false, 8>(tmp.data());
            const std::size_t l_step = std::min(step, s - off);
            for (std::size_t i = 0; i < l_step; ++i) {
                auto dst     = pcxo::pidx<8>(off + i);
                x[dst]       = tmp.data()[pcxo::pidx<8>(i)];
                x[dst + 8]   = tmp.data()[pcxo::pidx<8>(i) + 8];
            }
            off += l_step;
        }
    }
};

}    // namespace

extern "C" {

const char* ref_last_error() {
    return g_err.c_str();
}

// In-place transform through fft_unit<float, Order>::operator()/ifft (fft.hpp:728-853).
// order: 0 normal, 1 bit_reversed, 2 unordered.  dir: 0 forward, 1 inverse.
int ref_fft_f32(int order, std::size_t n, std::size_t sub_size, float* data, int dir, int norm) {
    return guarded([&] {
        switch (order) {
        case 0: return fft_inplace<pcxo::fft_order::normal>(n, sub_size, data, dir, norm);
        case 1: return fft_inplace<pcxo::fft_order::bit_reversed>(n, sub_size, data, dir, norm);
        default: return fft_inplace<pcxo::fft_order::unordered>(n, sub_size, data, dir, norm);
        }
    });
}

// Out-of-place transform through operator()(dest, src) / ifft(dest, src)
// (fft.hpp:759-820, 863-915); src holds src_n elements (zero-extended).
int ref_fft_oop_f32(int order, std::size_t n, std::size_t sub_size, float* dst, const float* src,
                    std::size_t src_n, int dir, int norm) {
    return guarded([&] {
        switch (order) {
        case 0: return fft_oop<pcxo::fft_order::normal>(n, sub_size, dst, src, src_n, dir, norm);
        case 1: return fft_oop<pcxo::fft_order::bit_reversed>(n, sub_size, dst, src, src_n, dir, norm);
        default: return fft_oop<pcxo::fft_order::unordered>(n, sub_size, dst, src, src_n, dir, norm);
        }
    });
}

// Forward out-of-place transform at pack widths pd / ps through
// fft_unit<float, Order>::fft_raw<PD, PS>(dest, source) (fft.hpp:645-670),
// for PD, PS in {1, 2, 4, 8}: the reference's pack conversions in its
// loads and stores (its AVX2 registers hold packs of at most 8 floats, so
// wider packs do not compile there, avx2_common.hpp:444).
int ref_fft_raw_packs_f32(int order, std::size_t n, std::size_t sub_size, float* dst, const float* src, int pd,
                          int ps) {
    return guarded([&] {
        auto run = [&]<pcxo::fft_order O>() {
            auto unit = pcxo::fft_unit<float, O>(n, sub_size);
            auto with = [&]<std::size_t PD>() {
                switch (ps) {
                case 1: unit.template fft_raw<PD, 1>(dst, src); return 0;
                case 2: unit.template fft_raw<PD, 2>(dst, src); return 0;
                case 4: unit.template fft_raw<PD, 4>(dst, src); return 0;
                case 8: unit.template fft_raw<PD, 8>(dst, src); return 0;
                default: g_err = "unsupported source pack"; return 1;
                }
            };
            switch (pd) {
            case 1: return with.template operator()<1>();
            case 2: return with.template operator()<2>();
            case 4: return with.template operator()<4>();
            case 8: return with.template operator()<8>();
            default: g_err = "unsupported destination pack"; return 1;
            }
        };
        return order == 0 ? run.template operator()<pcxo::fft_order::normal>()
                          : run.template operator()<pcxo::fft_order::bit_reversed>();
    });
}

// The reference's fxcorr_unit<float> exactly as shipped (fxcorr.hpp:62-136),
// in place on `data` (s elements).  Correct only for single-block inputs.
int ref_fxcorr_f32(const float* g, std::size_t k, std::size_t n_fft, float* data, std::size_t s) {
    return guarded([&] {
        auto gv = pcxo::vector<float>(k);
        std::memcpy(gv.data(), g, sizeof(float) * fvec::real_size(k));
        auto unit = pcxo::fxcorr_unit<float>(gv, n_fft);
        auto x    = pcxo::vector<float>(s);
        std::memcpy(x.data(), data, sizeof(float) * fvec::real_size(s));
        unit(x);
        std::memcpy(data, x.data(), sizeof(float) * fvec::real_size(s));
        return 0;
    });
}

// Corrected overlap-save on the reference's fft_unit (see fixed_fxcorr).
int ref_fxcorr_fixed_f32(const float* g, std::size_t k, std::size_t n_fft, float* data, std::size_t s) {
    return guarded([&] {
        fixed_fxcorr fx(g, k, n_fft);
        fx.run(data, s);
        return 0;
    });
}

// Batched in-place transforms over `batch` contiguous rows of n elements,
// split over `threads` std::threads with one fft_unit per thread (the unit is
// stateless after construction, fft.hpp:918-921).  Used as the timed CPU leg.
int ref_fft_batch_f32(int order, std::size_t n, std::size_t batch, float* data, int dir, int threads) {
    return guarded([&] {
        if (threads < 1) threads = 1;
        std::vector<std::thread> pool;
        std::atomic<int>         rc{0};
        for (int t = 0; t < threads; ++t) {
            pool.emplace_back([&, t] {
                try {
                    auto run = [&]<pcxo::fft_order O>() {
                        auto unit = pcxo::fft_unit<float, O>(n, 2048);
                        for (std::size_t b = t; b < batch; b += threads) {
                            float* p = data + b * 2 * n;
                            if (dir == 0) {
                                unit.template fft_raw<8>(p);
                            } else {
                                unit.template ifft_raw<true, 8>(p);
                            }
                        }
                    };
                    if (order == 0) {
                        run.template operator()<pcxo::fft_order::normal>();
                    } else {
                        run.template operator()<pcxo::fft_order::bit_reversed>();
                    }
                } catch (...) { rc = 1; }
            });
        }
        for (auto& th: pool) th.join();
        return rc.load();
    });
}

// Batched corrected overlap-save over `channels` rows of s elements each.
int ref_fxcorr_fixed_batch_f32(const float* g, std::size_t k, std::size_t n_fft, float* data, std::size_t s,
                               std::size_t channels, int threads) {
    return guarded([&] {
        if (threads < 1) threads = 1;
        std::vector<std::thread> pool;
        std::atomic<int>         rc{0};
        const std::size_t        row = fvec::real_size(s);
        for (int t = 0; t < threads; ++t) {
            pool.emplace_back([&, t] {
                try {
                    fixed_fxcorr fx(g, k, n_fft);
                    for (std::size_t c = t; c < channels; c += threads) fx.run(data + c * row, s);
                } catch (...) { rc = 1; }
            });
        }
        for (auto& th: pool) th.join();
        return rc.load();
    });
}

}    // extern "C"
