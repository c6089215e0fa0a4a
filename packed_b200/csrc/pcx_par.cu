// FFT across a set of vectors (reference fft_unit_par, fft.hpp:2167-2572):
// for every element position p < len, the n-point transform of
// src[0][p], src[1][p], ..., src[n-1][p] goes to dst[0][p], ..., dst[n-1][p].
//
// The n vectors are separate allocations, so a tiled transpose gathers them
// into `len` contiguous rows of n points (default pack), the batched FFT of
// the plan transforms those rows in place, and a second tiled transpose
// scatters the rows back into the destination vectors.  Both transposes read
// and write 32 consecutive elements per warp.
#include "pcx_core.cuh"
#include "pcx_host.hpp"

#include <algorithm>
#include <string>

using namespace pcxg;

namespace {

constexpr int TD = 32;    // tile edge
constexpr int TR = 8;     // thread rows

// rows[i][p] (pack 2^lps) -> buf[p][i] (pack 2^lpb, row stride rs reals)
template<class T>
__global__ void k_par_gather(const T* const* __restrict__ rows, int lps, T* __restrict__ buf, int lpb, long long rs,
                             long long n, long long len) {
    __shared__ T re[TD][TD + 1], im[TD][TD + 1];
    const long long i0 = (long long)blockIdx.y * TD, p0 = (long long)blockIdx.x * TD;
    const int       tx = threadIdx.x, ty = threadIdx.y;
    const long long ps = 1LL << lps, pb = 1LL << lpb;
    for (int r = ty; r < TD; r += TR) {
        const long long i = i0 + r, p = p0 + tx;
        if (i < n && p < len) {
            const T*        v = rows[i];
            const long long o = ((p >> lps) << (lps + 1)) + (p & (ps - 1));
            re[r][tx]         = v[o];
            im[r][tx]         = v[o + ps];
        }
    }
    __syncthreads();
    for (int r = ty; r < TD; r += TR) {
        const long long p = p0 + r, i = i0 + tx;
        if (i < n && p < len) {
            const long long o = p * rs + ((i >> lpb) << (lpb + 1)) + (i & (pb - 1));
            buf[o]            = re[tx][r];
            buf[o + pb]       = im[tx][r];
        }
    }
}

// buf[p][i] -> rows[i][p] (pack 2^lpd)
template<class T>
__global__ void k_par_scatter(T* const* __restrict__ rows, int lpd, const T* __restrict__ buf, int lpb, long long rs,
                              long long n, long long len) {
    __shared__ T re[TD][TD + 1], im[TD][TD + 1];
    const long long i0 = (long long)blockIdx.y * TD, p0 = (long long)blockIdx.x * TD;
    const int       tx = threadIdx.x, ty = threadIdx.y;
    const long long pd = 1LL << lpd, pb = 1LL << lpb;
    for (int r = ty; r < TD; r += TR) {
        const long long p = p0 + r, i = i0 + tx;
        if (i < n && p < len) {
            const long long o = p * rs + ((i >> lpb) << (lpb + 1)) + (i & (pb - 1));
            re[r][tx]         = buf[o];
            im[r][tx]         = buf[o + pb];
        }
    }
    __syncthreads();
    for (int r = ty; r < TD; r += TR) {
        const long long i = i0 + r, p = p0 + tx;
        if (i < n && p < len) {
            T*              v = rows[i];
            const long long o = ((p >> lpd) << (lpd + 1)) + (p & (pd - 1));
            v[o]              = re[tx][r];
            v[o + pd]         = im[tx][r];
        }
    }
}

int check_pack(int pack, const char* what) {
    if (pack < 1 || (pack & (pack - 1)) != 0) {
        return pcx_fail(PCX_ERR_INVALID, std::string(what) + " pack size (which is " + std::to_string(pack) +
                                             ") is not a power of two");
    }
    return PCX_OK;
}

}    // namespace

extern "C" int pcx_fft_par_exec(pcx_plan plan, void* const* dst, const void* const* src, size_t count, size_t len,
                                int pack_dst, int pack_src, int direction, int normalize, void* stream) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        pcx_plan_s* p = plan;
        // reference fft.hpp:2197-2211
        if (count != p->n) {
            return pcx_fail(PCX_ERR_INVALID, "destination size (which is " + std::to_string(count) +
                                                 " is not equal to fft size (which is " + std::to_string(p->n) + ")");
        }
        if (int rc = check_pack(pack_dst, "destination")) return rc;
        if (int rc = check_pack(pack_src, "source")) return rc;
        if (direction != PCX_FORWARD && direction != PCX_INVERSE) return pcx_fail(PCX_ERR_INVALID, "unknown direction");
        if (len == 0) return PCX_OK;
        if (!dst || !src) return pcx_fail(PCX_ERR_INVALID, "null vector array");
        for (size_t i = 0; i < count; ++i) {
            if (!dst[i] || !src[i]) return pcx_fail(PCX_ERR_INVALID, "null vector pointer");
        }
        const bool   f64  = p->dtype == PCX_F64;
        const size_t es   = f64 ? sizeof(double) : sizeof(float);
        int          lpb  = f64 ? 2 : 3;    // default pack, at most the row length
        while ((size_t(1) << lpb) > p->n) --lpb;
        const size_t pb   = size_t(1) << lpb;
        const size_t rs   = (p->n + pb - 1) / pb * 2 * pb;    // reals per gathered row
        const size_t need = 2 * count * sizeof(void*) + len * rs * es;
        cudaStream_t st   = static_cast<cudaStream_t>(stream);
        std::lock_guard<std::mutex> g(p->par_mu);
        if (p->par_bytes < need) {
            if (p->par_buf) cudaFree(p->par_buf);
            p->par_buf   = nullptr;
            p->par_bytes = 0;
            PCX_CUDA_TRY(cudaMalloc(&p->par_buf, need));
            p->par_bytes = need;
        }
        void** dptr = static_cast<void**>(p->par_buf);
        void** sptr = dptr + count;
        void*  buf  = sptr + count;
        // the pointer arrays are host memory: the copies return once staged
        PCX_CUDA_TRY(cudaMemcpyAsync(dptr, dst, count * sizeof(void*), cudaMemcpyHostToDevice, st));
        PCX_CUDA_TRY(cudaMemcpyAsync(sptr, src, count * sizeof(void*), cudaMemcpyHostToDevice, st));
        const dim3 blk(TD, TR);
        const dim3 grd((unsigned)((len + TD - 1) / TD), (unsigned)((count + TD - 1) / TD));
        const int  lps = __builtin_ctz(pack_src), lpd = __builtin_ctz(pack_dst);
        if (f64) {
            k_par_gather<double><<<grd, blk, 0, st>>>(reinterpret_cast<const double* const*>(sptr), lps,
                                                      static_cast<double*>(buf), lpb, (long long)rs, (long long)count,
                                                      (long long)len);
        } else {
            k_par_gather<float><<<grd, blk, 0, st>>>(reinterpret_cast<const float* const*>(sptr), lps,
                                                     static_cast<float*>(buf), lpb, (long long)rs, (long long)count,
                                                     (long long)len);
        }
        PCX_CUDA_TRY(cudaGetLastError());
        if (int rc = pcx_fft_run(p, buf, buf, p->n, (int)pb, (int)pb, direction, normalize, len, rs, rs, nullptr, 0,
                                 st, 1.0)) {
            return rc;
        }
        if (f64) {
            k_par_scatter<double><<<grd, blk, 0, st>>>(reinterpret_cast<double* const*>(dptr), lpd,
                                                       static_cast<const double*>(buf), lpb, (long long)rs,
                                                       (long long)count, (long long)len);
        } else {
            k_par_scatter<float><<<grd, blk, 0, st>>>(reinterpret_cast<float* const*>(dptr), lpd,
                                                      static_cast<const float*>(buf), lpb, (long long)rs,
                                                      (long long)count, (long long)len);
        }
        PCX_CUDA_TRY(cudaGetLastError());
        return PCX_OK;
    });
}
