// Host-side state and error plumbing shared by the C ABI translation units.
#pragma once

#include "../../include/pcx_cuda.h"

#include <cuda_runtime.h>
#include <exception>
#include <map>
#include <tuple>
#include <mutex>
#include <string>

namespace pcxg {

// Resident CTAs per SM for (kernel, block size, dynamic smem), queried once per
// device and cached: the occupancy query costs microseconds, which dominates a
// small-batch exec if repeated on every launch.
inline cudaError_t occupancy_cached(const void* kern, int nt, int bytes, int* per_sm) {
    using key_t = std::tuple<int, const void*, int, int>;
    static std::mutex             mu;
    static std::map<key_t, int>   cache;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const key_t k{dev, kern, nt, bytes};
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(k);
        if (it != cache.end()) { *per_sm = it->second; return cudaSuccess; }
    }
    int n = 0;
    e     = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, nt, bytes);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    cache[k] = n;
    *per_sm  = n;
    return cudaSuccess;
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (device, kernel).
inline cudaError_t smem_attr_cached(const void* kern, int bytes) {
    using key_t = std::tuple<int, const void*>;
    static std::mutex           mu;
    static std::map<key_t, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    auto it = done.find(key_t{dev, kern});
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done[key_t{dev, kern}] = bytes;
    return e;
}

struct v2_args;
struct v3_args;

// A variant of the one-launch four-step kernel (k_fourstep): the split
// N = 2^l1 * 2^l2, resident blocks per SM and ring stages.
struct fs_variant {
    int l1 = 0, l2 = 0, minb = 0, st = 0;
    bool operator==(const fs_variant& o) const { return l1 == o.l1 && l2 == o.l2 && minb == o.minb && st == o.st; }
};
// The variants built into the library (FP32 and FP64), in the order the
// autotuner tries them; the first one of a size is its untuned default (the
// fastest one measured on a B200 on 512 MB batches; at 2^15 and 2^17..2^19 an
// uneven split with the longer sub-transform in the row pass is fastest).
constexpr fs_variant kFsVariantsF32[] = {
    {7, 6, 2, 3},  {6, 7, 2, 3},                                      // 2^13 (beside the one-pass form)
    {7, 7, 2, 3},  {7, 7, 1, 3},  {6, 8, 2, 3},                       // 2^14
    {7, 8, 2, 3},  {8, 7, 2, 3},  {6, 9, 2, 3},                       // 2^15
    {8, 8, 2, 3},  {8, 8, 1, 3},  {7, 9, 2, 3},  {9, 7, 2, 3},  {6, 10, 1, 3},    // 2^16
    {8, 9, 2, 3},  {9, 8, 2, 3},  {10, 7, 1, 3}, {9, 8, 1, 3},  {7, 10, 1, 3},    // 2^17
    {8, 10, 1, 3}, {10, 8, 1, 3}, {9, 9, 1, 3},  {9, 9, 2, 3},        // 2^18
    {9, 10, 1, 3}, {9, 10, 1, 2}, {10, 9, 1, 2}, {10, 9, 1, 3},       // 2^19
    {10, 10, 1, 3}, {10, 10, 1, 2},                                   // 2^20
};
constexpr fs_variant kFsVariantsF64[] = {
    {7, 7, 2, 3}, {8, 7, 2, 3}, {8, 8, 2, 3}, {9, 8, 2, 3}, {9, 9, 2, 3}, {10, 9, 1, 2}, {10, 10, 1, 2},
};
}

// Record `msg` as this thread's last error and return `code`.
int pcx_fail(int code, const std::string& msg);

// Run `f`, turning C++ exceptions into PCX_ERR_INVALID (no exception crosses the C ABI).
template<class F>
int pcx_guard(F&& f) {
    try {
        return f();
    } catch (const std::exception& e) {
        return pcx_fail(PCX_ERR_INVALID, e.what());
    } catch (...) {
        return pcx_fail(PCX_ERR_INVALID, "unknown exception");
    }
}

#define PCX_CUDA_TRY(expr)                                                                       \
    do {                                                                                         \
        cudaError_t pcx_e_ = (expr);                                                             \
        if (pcx_e_ != cudaSuccess) {                                                             \
            return pcx_fail(PCX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(pcx_e_)); \
        }                                                                                        \
    } while (0)

struct pcx_plan_s {
    size_t n        = 0;
    int    dtype    = PCX_F32;
    int    order    = PCX_ORDER_NORMAL;
    size_t sub_size = 2048;
    int    log_n    = 0;
    int    two_pass = 0;
    int    log_n1   = 0;
    int    log_n2   = 0;
    int    device   = 0;

    void*  tw       = nullptr;    // one allocation holding every table below
    size_t tw_bytes = 0;
    void*  twL      = nullptr;    // W_N^i, single-pass
    void*  twN1     = nullptr;    // W_N1^i
    void*  twN2     = nullptr;    // W_N2^i
    void*  tw_lo    = nullptr;    // W_N^i, i < N2
    void*  tw_hi    = nullptr;    // W_N^(i*N2), i < N1

    void*  scratch       = nullptr;    // four-step intermediate (plan-owned)
    size_t scratch_bytes = 0;

    // hot-path tables (pcx_fft_v2.cuh)
    void*  stw      = nullptr;    // one allocation: stage twiddles (N | N1, N2) and W_{16*N2}^m
    void*  stwL     = nullptr;    // stage twiddles of the single pass
    void*  stw1     = nullptr;    // stage twiddles of the column pass (N1)
    void*  stw2     = nullptr;    // stage twiddles of the row pass (N2)
    void*  tw_b     = nullptr;    // W_{16*N2}^m, m < 16*N2
    void*  stw_one  = nullptr;    // stage twiddles of a one-pass form of a two-pass size (N = 8192)
    void*  fst      = nullptr;    // one-launch four-step: full stage tables of N1 then N2 (one allocation)
    void*  fst1     = nullptr;
    void*  fst2     = nullptr;
    pcxg::fs_variant fs_var{};    // one-launch four-step: its variant (l1 == 0: none)
    void*  fs_mem   = nullptr;    // tables of fs_var's split (one allocation):
    void*  fs_thi   = nullptr;    //   W_N^(i*N2), i < N1
    void*  fs_tlo   = nullptr;    //   W_N^i, i < N2
    void*  fs_tb    = nullptr;    //   W_{16*N2}^i, i < N2
    void*  fs_st1   = nullptr;    //   full stage tables of the N1- and N2-point sub-transforms
    void*  fs_st2   = nullptr;
    int    fs_tab_l1 = 0;         // split the tables belong to
    int    fs_tc    = 0;          // one-launch four-step: column and row tiles per transform (0: none)
    int    fs_tr    = 0;
    int    fs_per_sm = 1;         // its resident blocks per SM
    int*   fs_ctr   = nullptr;    // its dependency counters, 2 per transform
    size_t fs_ctr_n = 0;
    // form of the plan-owned-scratch path for n > 4096, set by pcx_plan_tune
    int    form        = 0;    // PCX_FORM_*: 0 built-in choice
    int    fs_rounds   = 3;    // one-launch four-step: dependency distance in rounds of tiles
    size_t chunk_bytes = 0;    // chunked four-step: scratch per buffer (0: 24 MB)
    // transforms across vectors (pcx_fft_par_exec): pointer arrays + gathered rows
    void*      par_buf   = nullptr;
    size_t     par_bytes = 0;
    std::mutex par_mu;
    int    sms      = 148;
    int*   err      = nullptr;    // device flag: a bounded wait in a kernel gave up

    // four-step chunk pipeline: column passes on the caller's stream, row
    // passes on `side`, two scratch buffers
    cudaStream_t side = nullptr;
    cudaEvent_t  ev_col[2]{};
    cudaEvent_t  ev_row[2]{};
    cudaEvent_t  ev_fork = nullptr;
    std::mutex   mu;

    size_t elem_bytes() const { return dtype == PCX_F64 ? 16 : 8; }
    size_t chunk_rows(size_t batch) const;
    void   release();
};

// Core of pcx_fft_exec (no exception guard); extra_scale multiplies the output.
// chunk_cap (rows per four-step chunk, 0 = no cap) lets a caller with a
// fixed workspace bound the chunk to it.
int pcx_fft_run(pcx_plan_s* p, void* dst, const void* src, size_t src_len, int pd, int ps, int dir, int norm,
                size_t batch, size_t dstride, size_t sstride, void* ws, size_t ws_bytes, cudaStream_t st,
                double extra_scale, size_t chunk_cap = 0);

// Table W_N^(i*mult), i < count, N = 2^log_n, generated in FP64 and rounded once.
cudaError_t pcx_gen_twiddles(void* out, int count, int log_n, long long mult, bool f64, cudaStream_t st);
// A correlation spectrum K[k1 + N1*k2] (complex64) reordered to [k1*N2 + k2]
// for the in-CTA four-step correlator (pcx_fxcorr.cu).
cudaError_t pcx_xc2_perm_spectrum(const void* ks, void* kp, int log_n1, int log_n2, cudaStream_t st);

namespace pcxg {
// One work item of the persistent tensor-core FFT (pcx_tc.cu): `rows`
// transforms of 2^lg points (8 <= lg <= 12, rows <= 2^(12 - lg)), complex64
// pack 8, each from its own source row to its own destination row.
struct tc_item {
    int          lg;
    int          rows;
    const float* src[16];
    float*       dst[16];
};
}    // namespace pcxg
// The persistent tensor-core FFT over a device list of items (precision 0
// bf16 x3, 1 tf32 x3, 2 bf16 x6): conj = 1 conjugates inputs and outputs (the
// inverse), scale multiplies the outputs; tw = W_M^i (i < M = 2^tw_lg >= every
// item's size).  Resident CTAs, at most one per item.
cudaError_t pcx_tc_list_launch(int precision, const pcxg::tc_item* items, int nitems, int conj, float scale,
                               const void* tw, int tw_lg, int* error, int sms, cudaStream_t st);

// Hot-path launches (pcx_v2_*.cu); cudaErrorNotSupported when no variant exists.
cudaError_t pcx_v2_single(bool f64, int log_n, const pcxg::v2_args& a, cudaStream_t st, bool attr_only);
cudaError_t pcx_v3_single(bool f64, int log_n, const pcxg::v3_args& a, cudaStream_t st, int sms, bool attr_only);
namespace pcxg {
struct fs_args;
}
cudaError_t pcx_fourstep(bool f64, const pcxg::fs_variant& v, const pcxg::fs_args& a, cudaStream_t st, int sms,
                         bool attr_only, int* col_tiles, int* row_tiles, int* blocks_per_sm);
// Full stage tables of an L = 2^log_l point sub-transform of the one-launch
// four-step (entries: their count; out == nullptr only counts).
cudaError_t pcx_fourstep_tables(int log_l, void* out, bool f64, cudaStream_t st, int* entries);
cudaError_t pcx_v2_col(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, cudaStream_t st, int sms,
                       bool attr_only);
cudaError_t pcx_v2_row(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, cudaStream_t st, int sms,
                       bool attr_only);
cudaError_t pcx_v3_col(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, long long total_rows, long long row0,
                       int* err, cudaStream_t st, int sms, bool attr_only);
cudaError_t pcx_v3_row(bool f64, int log_n1, int log_n2, const pcxg::v2_args& a, int* err, cudaStream_t st, int sms,
                       bool attr_only);
// Stage-twiddle table of an L = 2^log_l point transform: *entries complex
// values; generated into `out` unless it is null.
cudaError_t pcx_v2_stage_twiddles(int log_l, void* out, bool f64, cudaStream_t st, int* entries);
