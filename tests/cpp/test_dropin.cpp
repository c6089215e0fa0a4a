// C++ drop-in check: the reference's own call patterns (tests/test_fft.cpp,
// tests/test_fxcorr.cpp of the reference) compiled against include/pcxo/*.hpp
// and run on the GPU.  Exit status 0 on success.
#include "pcxo/fft.hpp"
#include "pcxo/fxcorr.hpp"
#include "pcxo/mdstorage.hpp"
#include "pcxo/ragged.hpp"

#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

using cd = std::complex<double>;

static std::vector<cd> dft(const std::vector<cd>& x, int sign) {
    const std::size_t n = x.size();
    std::vector<cd>   X(n);
    for (std::size_t k = 0; k < n; ++k) {
        cd s = 0;
        for (std::size_t j = 0; j < n; ++j) s += x[j] * std::polar(1.0, sign * 2 * M_PI * double((j * k) % n) / n);
        X[k] = s;
    }
    return X;
}

template<typename V>
static double rel_err(const V& got, const std::vector<cd>& want) {
    double num = 0, den = 0;
    for (std::size_t i = 0; i < want.size(); ++i) {
        cd g = std::complex<double>(got[i]);
        num += std::norm(g - want[i]);
        den += std::norm(want[i]);
    }
    return std::sqrt(num / den);
}

static int fails = 0;
static void expect(bool ok, const char* what, double v = 0) {
    std::printf("%-44s %s %.3e\n", what, ok ? "ok  " : "FAIL", v);
    if (!ok) ++fails;
}

int main() {
    std::mt19937_64                        rng(0);
    std::uniform_real_distribution<float> u(-1, 1);
    constexpr float                        pi = 3.14159265358979323846f;
    for (std::size_t n: {64u, 1024u, 8192u}) {
        pcxo::vector<float>           v(n);
        std::vector<std::complex<float>> sv(n);
        std::vector<cd>                  x(n);
        for (std::size_t i = 0; i < n; ++i) {
            auto val = std::exp(std::complex<float>(0, 2 * pi * i / n * 13.37f));    // reference test input
            v[i]     = val;
            sv[i]    = val;
            x[i]     = cd(val);
        }
        const auto X = dft(x, -1);
        pcxo::fft_unit<float> unit(n);
        unit(v);
        expect(rel_err(v, X) < 2e-6, "fft_unit<float>(vector) normal", rel_err(v, X));
        unit.ifft(v);
        expect(rel_err(v, x) < 2e-6, "ifft(vector) round trip", rel_err(v, x));
        unit(sv);    // host std::vector<std::complex<float>>: staged
        expect(rel_err(sv, X) < 2e-6, "fft_unit(std::vector<complex>)", rel_err(sv, X));
        pcxo::vector<float> out(n);
        unit(out, v);
        expect(rel_err(out, X) < 2e-6, "fft_unit(dest, src)", rel_err(out, X));
        pcxo::fft_unit<float, pcxo::fft_order::bit_reversed> ubr(n);
        pcxo::vector<float>                                  w = v;
        ubr.fft_raw<8>(w.data());
        ubr.ifft_raw<true, 8>(w.data());
        expect(rel_err(w, x) < 2e-6, "bit_reversed fft_raw/ifft_raw", rel_err(w, x));
        // zero-extended source (fft.hpp:759-820)
        pcxo::vector<float> shortv(n / 2 + 3);
        std::vector<cd>     xs(n, 0.0);
        for (std::size_t i = 0; i < shortv.size(); ++i) {
            shortv[i] = std::complex<float>(u(rng), u(rng));
            xs[i]     = cd(std::complex<float>(shortv[i]));
        }
        unit(out, shortv);
        expect(rel_err(out, dft(xs, -1)) < 2e-6, "zero-extended out-of-place", rel_err(out, dft(xs, -1)));
    }
    {
        pcxo::vector<double> v(4096);
        std::vector<cd>      x(4096);
        for (std::size_t i = 0; i < 4096; ++i) x[i] = cd(u(rng), u(rng)), v[i] = x[i];
        pcxo::fft_unit<double> unit(4096);
        unit(v);
        expect(rel_err(v, dft(x, -1)) < 1e-13, "fft_unit<double>", rel_err(v, dft(x, -1)));
    }
    {    // fxcorr (tests/test_fxcorr.cpp: naive correlation ground truth)
        const std::size_t   k = 300, s = 10000, nf = 1024;
        pcxo::vector<float> g(k), f(s);
        std::vector<cd>     gd(k), fd(s), y(s);
        for (std::size_t i = 0; i < k; ++i) gd[i] = cd(u(rng), u(rng)), g[i] = gd[i];
        for (std::size_t i = 0; i < s; ++i) fd[i] = cd(u(rng), u(rng)), f[i] = fd[i];
        for (std::size_t i = 0; i < s; ++i) {
            cd acc = 0;
            for (std::size_t j = 0; j < k && i + j < s; ++j) acc += fd[i + j] * std::conj(gd[j]);
            y[i] = acc;
        }
        pcxo::fxcorr_unit<float> xc(g, nf);
        pcxo::vector<float>      dst(s);
        xc(dst, f);
        expect(rel_err(dst, y) < 2e-6, "fxcorr_unit(dest, src)", rel_err(dst, y));
        xc(f);
        expect(rel_err(f, y) < 2e-6, "fxcorr_unit(vector) in place", rel_err(f, y));
        // a host std::vector<std::complex<float>> (pack 1), in place and out of place
        std::vector<std::complex<float>> sv(s), so(s);
        for (std::size_t i = 0; i < s; ++i) sv[i] = std::complex<float>(fd[i]);
        xc(so, sv);
        expect(rel_err(so, y) < 2e-6, "fxcorr_unit(std::vector dest, src)", rel_err(so, y));
        xc(sv);
        expect(rel_err(sv, y) < 2e-6, "fxcorr_unit(std::vector) in place", rel_err(sv, y));
    }
    {    // ragged batch: FFTs of three sizes and a correlation in one persistent launch
        const std::size_t                sizes[] = {256, 2048, 8192};
        std::vector<pcxo::vector<float>> src, dst;
        std::vector<std::vector<cd>>     want;
        for (std::size_t n: sizes) {
            src.emplace_back(n);
            dst.emplace_back(n);
            std::vector<cd> x(n);
            for (std::size_t i = 0; i < n; ++i) x[i] = cd(u(rng), u(rng)), src.back()[i] = x[i];
            want.push_back(dft(x, -1));
        }
        const std::size_t   k = 300, s = 5000;
        pcxo::vector<float> g(k), x(s), yv(s);
        std::vector<cd>     gd(k), xd(s), y(s);
        for (std::size_t i = 0; i < k; ++i) gd[i] = cd(u(rng), u(rng)), g[i] = gd[i];
        for (std::size_t i = 0; i < s; ++i) xd[i] = cd(u(rng), u(rng)), x[i] = xd[i];
        for (std::size_t i = 0; i < s; ++i) {
            cd acc = 0;
            for (std::size_t j = 0; j < k && i + j < s; ++j) acc += xd[i + j] * std::conj(gd[j]);
            y[i] = acc;
        }
        pcxo::ragged_batch batch;
        for (std::size_t q = 0; q < 3; ++q) batch.add_fft(dst[q], src[q]);
        batch.add_xcorr(yv, x, g, pcxo::correlation_fft_size(k));
        batch();
        double worst = 0;
        for (std::size_t q = 0; q < 3; ++q) worst = std::max(worst, rel_err(dst[q], want[q]));
        expect(worst < 2e-6, "ragged_batch FFTs (256, 2048, 8192)", worst);
        expect(rel_err(yv, y) < 2e-6, "ragged_batch correlation", rel_err(yv, y));
        expect(batch.items() > 3, "ragged_batch work items");
        // the tensor-core form (bf16 x6) for the 256- and 2048-point transforms
        for (std::size_t q = 0; q < 3; ++q)
            for (std::size_t i = 0; i < dst[q].size(); ++i) dst[q][i] = std::complex<float>(0, 0);
        pcxo::ragged_batch tc(false, true, 2);
        for (std::size_t q = 0; q < 3; ++q) tc.add_fft(dst[q], src[q]);
        tc();
        worst = 0;
        for (std::size_t q = 0; q < 3; ++q) worst = std::max(worst, rel_err(dst[q], want[q]));
        expect(worst < 2e-6, "ragged_batch tensor-core form (256, 2048 on tcgen05; 8192)", worst);
    }
    {    // md::dynamic_storage (mdstorage.hpp): rows as vectors and batched row transforms
        enum class ax { x, y, z };
        using enum ax;
        constexpr auto basis = pcxo::md::left_basis<x, y, z>{};
        const unsigned nx = 1000, ny = 3, nz = 5;    // inner axis x, padded to whole packs
        auto           st = pcxo::md::dynamic_storage<float, basis>(nx, ny, nz);
        expect(st.extent<x>() == nx && st.extent<z>() == nz && st.row_stride() == 2000, "md storage extents / padding");
        std::vector<std::vector<cd>> rows;
        for (unsigned k = 0; k < nz; ++k) {
            for (unsigned j = 0; j < ny; ++j) {
                auto row = st.slice<z>(k).slice<y>(j);
                std::vector<cd> r(nx);
                for (unsigned i = 0; i < nx; ++i) {
                    r[i]   = cd(u(rng), u(rng));
                    row[i] = r[i];
                }
                rows.push_back(r);
            }
        }
        // nx = 1000 is not a power of two: use the first 512 points of every row via a 512-point storage
        auto st2 = pcxo::md::dynamic_storage<float, basis>(512u, ny, nz);
        std::vector<std::vector<cd>> want;
        for (unsigned k = 0, q = 0; k < nz; ++k) {
            for (unsigned j = 0; j < ny; ++j, ++q) {
                auto row = st2.slice<z>(k).slice<y>(j);
                std::vector<cd> r(rows[q].begin(), rows[q].begin() + 512);
                for (unsigned i = 0; i < 512; ++i) row[i] = r[i];
                want.push_back(dft(r, -1));
            }
        }
        pcxo::fft_unit<float> unit(512);
        pcxo::md::fft_rows(unit, st2);
        double worst = 0;
        for (unsigned k = 0, q = 0; k < nz; ++k) {
            for (unsigned j = 0; j < ny; ++j, ++q) {
                auto row = st2.slice<z>(k).slice<y>(j);
                worst    = std::max(worst, rel_err(row, want[q]));
            }
        }
        expect(worst < 2e-6, "md::fft_rows over 15 rows", worst);
        auto one = st2.slice<z>(2).slice<y>(1);
        unit.ifft(one);    // a single row through the vector interface
        std::vector<cd> back(rows[2 * ny + 1].begin(), rows[2 * ny + 1].begin() + 512);
        expect(rel_err(one, back) < 2e-6, "fft_unit on an md row slice", rel_err(one, back));
    }
    {    // fft_unit_par (fft.hpp:2167): the reference test's pattern, tests/test_fft.cpp:700-754
        for (std::size_t size: {64u, 512u, 4096u}) {
            std::vector<pcxo::vector<float>> st_par(size), out(size);
            std::vector<cd>                  col(size);
            for (std::size_t i = 0; i < size; ++i) {
                st_par[i] = pcxo::vector<float>(128);
                out[i]    = pcxo::vector<float>(128);
                auto val  = std::exp(std::complex<float>(0, 2 * pi * i / size * 13.37f));
                for (std::size_t p = 0; p < 128; ++p) st_par[i][p] = val * float(1 + p % 3);
                col[i] = cd(val);
            }
            pcxo::fft_unit_par<float> par_unit(size);
            par_unit(out, st_par);
            const auto      X = dft(col, -1);
            double          worst = 0;
            for (std::size_t p: {0u, 1u, 2u, 127u}) {
                std::vector<std::complex<float>> got(size);
                std::vector<cd>                  want(size);
                for (std::size_t i = 0; i < size; ++i) {
                    got[i]  = out[i][p].value();
                    want[i] = X[i] * double(1 + p % 3);
                }
                worst = std::max(worst, rel_err(got, want));
            }
            char what[64];
            std::snprintf(what, sizeof what, "fft_unit_par size %zu x 128", size);
            expect(worst < 2e-6, what, worst);
        }
    }
    {    // vector expressions on the device (vector_arithm.hpp; tests/test_op.cpp:116-131 table)
        const std::size_t   n = 1000;
        pcxo::vector<float> a(n), b(n), c(n), out(n);
        std::vector<cd>     za(n), zb(n), zc(n);
        for (std::size_t i = 0; i < n; ++i) {
            za[i] = cd(u(rng), u(rng));
            zb[i] = cd(2 + u(rng), u(rng));
            zc[i] = cd(u(rng), u(rng));
            a[i]  = std::complex<float>(za[i]);
            b[i]  = std::complex<float>(zb[i]);
            c[i]  = std::complex<float>(zc[i]);
        }
        const std::complex<float> s(0.5f, -1.5f);
        const cd                  sd(0.5, -1.5);
        auto check = [&](const char* what, auto&& make_want) {
            std::vector<cd> want(n);
            for (std::size_t i = 0; i < n; ++i) want[i] = make_want(i);
            expect(rel_err(out, want) < 2e-6, what, rel_err(out, want));
        };
        out = a + b;
        check("expr a + b", [&](std::size_t i) { return za[i] + zb[i]; });
        out = a * pcxo::conj(b);
        check("expr a * conj(b)", [&](std::size_t i) { return za[i] * std::conj(zb[i]); });
        out = pcxo::conj(a) / b - c;
        check("expr conj(a) / b - c", [&](std::size_t i) { return std::conj(za[i]) / zb[i] - zc[i]; });
        out = s * a + 2.f / c;
        check("expr s * a + 2 / c", [&](std::size_t i) { return sd * za[i] + 2.0 / zc[i]; });
        a = a * a;
        std::vector<cd> sq(n);
        for (std::size_t i = 0; i < n; ++i) sq[i] = za[i] * za[i];
        expect(rel_err(a, sq) < 2e-6, "expr a = a * a (in place)", rel_err(a, sq));
    }
    {    // tensor-core form (pcx_tc_fft_exec): forward in each precision, inverse round trip
        const std::size_t n = 4096, batch = 4;
        pcxo::fft_unit<float> unit(n);
        std::vector<cd>       x(n * batch);
        for (auto& v: x) v = cd(u(rng), u(rng));
        std::vector<float> h(2 * n * batch);
        for (std::size_t b = 0; b < batch; ++b) {
            for (std::size_t i = 0; i < n; ++i) {
                h[2 * n * b + pcxo::pidx<8>(i)]     = float(x[b * n + i].real());
                h[2 * n * b + pcxo::pidx<8>(i) + 8] = float(x[b * n + i].imag());
                x[b * n + i] = cd(h[2 * n * b + pcxo::pidx<8>(i)], h[2 * n * b + pcxo::pidx<8>(i) + 8]);
            }
        }
        float *d_x = nullptr, *d_y = nullptr;
        pcxo::detail_::check_cuda(cudaMalloc(&d_x, h.size() * sizeof(float)));
        pcxo::detail_::check_cuda(cudaMalloc(&d_y, h.size() * sizeof(float)));
        pcxo::detail_::check_cuda(cudaMemcpy(d_x, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
        using prec = pcxo::fft_unit<float>::tc_precision;
        auto rel = [&](const float* dev, bool spectrum) {
            std::vector<float> o(h.size());
            pcxo::detail_::check_cuda(cudaMemcpy(o.data(), dev, o.size() * sizeof(float), cudaMemcpyDeviceToHost));
            double worst = 0;
            for (std::size_t b = 0; b < batch; ++b) {
                std::vector<cd> in(x.begin() + b * n, x.begin() + (b + 1) * n), got(n);
                for (std::size_t i = 0; i < n; ++i) {
                    got[i] = cd(o[2 * n * b + pcxo::pidx<8>(i)], o[2 * n * b + pcxo::pidx<8>(i) + 8]);
                }
                worst = std::max(worst, rel_err(got, spectrum ? dft(in, -1) : in));
            }
            return worst;
        };
        unit.fft_batch_tensor_core(d_y, d_x, batch);
        const double e6 = rel(d_y, true);
        expect(e6 < 2e-6, "fft_batch_tensor_core bf16x6", e6);
        unit.fft_batch_tensor_core(d_y, d_x, batch, prec::tf32x3);
        const double et = rel(d_y, true);
        expect(et < 2e-6, "fft_batch_tensor_core tf32x3", et);
        unit.ifft_batch_tensor_core(d_x, d_y, batch, prec::tf32x3);
        const double er = rel(d_x, false);
        expect(er < 2e-6, "ifft_batch_tensor_core round trip", er);
        cudaFree(d_x);
        cudaFree(d_y);
    }
    {    // adjoints (no reference counterpart): fft_unit::vjp is the unnormalised inverse
        const std::size_t n = 1024, batch = 3;
        std::vector<cd>   gy(n * batch);
        for (auto& v: gy) v = cd(u(rng), u(rng));
        pcxo::fft_unit<double> unit(n);
        const std::size_t      row = 2 * n;    // pack 4, no padding
        double*                d_gy = nullptr;
        double*                d_gx = nullptr;
        pcxo::detail_::check_cuda(cudaMalloc(&d_gy, batch * row * sizeof(double)));
        pcxo::detail_::check_cuda(cudaMalloc(&d_gx, batch * row * sizeof(double)));
        std::vector<double> h(batch * row);
        for (std::size_t b = 0; b < batch; ++b) {
            for (std::size_t i = 0; i < n; ++i) {
                h[b * row + pcxo::pidx<4>(i)]     = gy[b * n + i].real();
                h[b * row + pcxo::pidx<4>(i) + 4] = gy[b * n + i].imag();
            }
        }
        pcxo::detail_::check_cuda(cudaMemcpy(d_gy, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
        double worst = 0;
        for (int inverse = 0; inverse < 2; ++inverse) {
            unit.vjp<true, 4>(d_gx, d_gy, batch, inverse != 0);
            pcxo::detail_::check_cuda(cudaMemcpy(h.data(), d_gx, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (std::size_t b = 0; b < batch; ++b) {
                std::vector<cd> in(gy.begin() + b * n, gy.begin() + (b + 1) * n), got(n);
                // adjoint of the forward: F^H g; of the normalised inverse: F g / n
                auto want = dft(in, inverse ? -1 : +1);
                if (inverse) {
                    for (auto& v: want) v /= double(n);
                }
                for (std::size_t i = 0; i < n; ++i) {
                    got[i] = cd(h[b * row + pcxo::pidx<4>(i)], h[b * row + pcxo::pidx<4>(i) + 4]);
                }
                worst = std::max(worst, rel_err(got, want));
            }
        }
        expect(worst < 1e-13, "fft_unit<double>::vjp (forward, inverse)", worst);
        cudaFree(d_gy);
        cudaFree(d_gx);
    }
    {    // fxcorr_unit::vjp: gx = convolution of gy with g, gg = correlation of gy with x
        const std::size_t k = 100, s = 3000, nf = 512;
        std::vector<cd>   gd(k), xd(s), gyd(s);
        for (auto& v: gd) v = cd(u(rng), u(rng));
        for (auto& v: xd) v = cd(u(rng), u(rng));
        for (auto& v: gyd) v = cd(u(rng), u(rng));
        pcxo::vector<float> g(k);
        for (std::size_t i = 0; i < k; ++i) g[i] = std::complex<float>(gd[i]);
        pcxo::fxcorr_unit<float> xc(g, nf);
        pcxo::vector<float>      x(s), gyv(s), gx(s), gg(k);
        for (std::size_t i = 0; i < s; ++i) {
            x[i]   = std::complex<float>(xd[i]);
            gyv[i] = std::complex<float>(gyd[i]);
            xd[i]  = cd(std::complex<float>(x[i]));
            gyd[i] = cd(std::complex<float>(gyv[i]));
        }
        for (std::size_t i = 0; i < k; ++i) gd[i] = cd(std::complex<float>(g[i]));
        xc.vjp(gx.data(), gg.data(), gyv.data(), x.data(), s);
        std::vector<cd> gx_want(s, 0.0), gg_want(k, 0.0);
        for (std::size_t m = 0; m < s; ++m) {
            for (std::size_t j = 0; j < k && m + j < s; ++j) {
                gx_want[m + j] += gd[j] * gyd[m];
                gg_want[j] += xd[m + j] * std::conj(gyd[m]);
            }
        }
        expect(rel_err(gx, gx_want) < 2e-6, "fxcorr_unit::vjp gx (convolution)", rel_err(gx, gx_want));
        expect(rel_err(gg, gg_want) < 2e-6, "fxcorr_unit::vjp gg (correlation)", rel_err(gg, gg_want));
    }
    {    // a bounded device wait that gives up becomes an exception through the drop-in
        pcxo::fft_unit<float> unit(1024);
        pcxo::vector<float>   v(1024);
        pcxo::detail_::check(pcx_selftest_plan_wait(unit.plan(), 1000000ull, nullptr));
        bool thrown = false;
        try {
            unit(v);
        } catch (const std::runtime_error& e) {
            thrown = std::string(e.what()).find("gave up") != std::string::npos;
        }
        expect(thrown, "given-up device wait -> std::runtime_error");
        bool again = true;
        try {
            unit(v);    // the flag was read and cleared: the next call runs normally
        } catch (const std::exception&) {
            again = false;
        }
        expect(again, "next call after a give-up succeeds");
    }
    {    // exceptions keep the reference's types and messages
        bool thrown = false;
        try {
            pcxo::fft_unit<float> bad(1000);
        } catch (const std::invalid_argument& e) {
            thrown = std::string(e.what()).find("power of two") != std::string::npos;
        }
        expect(thrown, "invalid_argument for non power of two");
        thrown = false;
        try {
            pcxo::fft_unit<float> unit(64);
            pcxo::vector<float>   v(32);
            unit(v);
        } catch (const std::invalid_argument& e) {
            thrown = std::string(e.what()).find("is not equal to fft size") != std::string::npos;
        }
        expect(thrown, "invalid_argument for size mismatch");
    }
    std::printf(fails ? "FAILED %d\n" : "ALL OK\n", fails);
    return fails ? 1 : 0;
}
