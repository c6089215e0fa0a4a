// Dispatch of the one-launch four-step kernel (k_fourstep) over its variants,
// its stage tables, and the self-tests of its bounded waits.
#include "pcx_fourstep.cuh"
#include "pcx_host.hpp"

// The variant translation units (pcx_fs_part*.cu).
cudaError_t pcx_fs_part0(bool, const pcxg::fs_variant&, const pcxg::fs_args&, cudaStream_t, int, bool, int*, int*, int*);
cudaError_t pcx_fs_part1(bool, const pcxg::fs_variant&, const pcxg::fs_args&, cudaStream_t, int, bool, int*, int*, int*);
cudaError_t pcx_fs_part2(bool, const pcxg::fs_variant&, const pcxg::fs_args&, cudaStream_t, int, bool, int*, int*, int*);
cudaError_t pcx_fs_part3(bool, const pcxg::fs_variant&, const pcxg::fs_args&, cudaStream_t, int, bool, int*, int*, int*);
cudaError_t pcx_fs_part4(bool, const pcxg::fs_variant&, const pcxg::fs_args&, cudaStream_t, int, bool, int*, int*, int*);

cudaError_t pcx_fourstep(bool f64, const pcxg::fs_variant& v, const pcxg::fs_args& a, cudaStream_t st, int sms,
                         bool attr_only, int* col_tiles, int* row_tiles, int* blocks_per_sm) {
    for (auto part: {pcx_fs_part0, pcx_fs_part1, pcx_fs_part2, pcx_fs_part3, pcx_fs_part4}) {
        const cudaError_t e = part(f64, v, a, st, sms, attr_only, col_tiles, row_tiles, blocks_per_sm);
        if (e != cudaErrorNotSupported) return e;
    }
    return cudaErrorNotSupported;
}

namespace {
// One thread runs the kernels' bounded waits on conditions that never come
// true (phase 0 of an mbarrier nobody arrives on, a counter nobody
// increments) and records whether each returned `true`; both must give up.
__global__ void k_wait_probe(const int* ctr, int* out, unsigned long long mbar_limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        pcxg::mbar_init(&bar, 1);
        pcxg::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = pcxg::mbar_wait_bounded(&bar, 0u, mbar_limit_ns) ? 1 : 0;
        out[1] = pcxg::fs_wait(ctr, 1) ? 1 : 0;
        out[2] = 1;    // the kernel got past both waits
    }
}
}    // namespace

namespace {
template<int LOGL, class T>
cudaError_t gen_full_tables(void* out, cudaStream_t st) {
    using P = pcxg::splan<LOGL>;
    for (int s = 1; s < P::NST; ++s) {
        const int n = (1 << P::nsbits(s)) * pcxg::full_tw_row(P::rbits(s));
        auto*     o = static_cast<pcxg::cpx<T>*>(out) + pcxg::fs_full_tw_offset<P>(s);
        pcxg::k_full_twiddles<T><<<(n + 255) / 256, 256, 0, st>>>(o, 1 << P::nsbits(s), P::rbits(s),
                                                                 P::nsbits(s) + P::rbits(s));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
template<int LOGL>
cudaError_t full_tables(void* out, bool f64, cudaStream_t st, int* entries) {
    *entries = pcxg::fs_full_tw_size<pcxg::splan<LOGL>>();
    if (!out) return cudaSuccess;
    return f64 ? gen_full_tables<LOGL, double>(out, st) : gen_full_tables<LOGL, float>(out, st);
}
}    // namespace

cudaError_t pcx_fourstep_tables(int log_l, void* out, bool f64, cudaStream_t st, int* entries) {
    switch (log_l) {
    case 5: return full_tables<5>(out, f64, st, entries);
    case 6: return full_tables<6>(out, f64, st, entries);
    case 7: return full_tables<7>(out, f64, st, entries);
    case 8: return full_tables<8>(out, f64, st, entries);
    case 9: return full_tables<9>(out, f64, st, entries);
    case 10: return full_tables<10>(out, f64, st, entries);
    case 11: return full_tables<11>(out, f64, st, entries);
    case 12: return full_tables<12>(out, f64, st, entries);
    case 13: return full_tables<13>(out, f64, st, entries);
    case 14: return full_tables<14>(out, f64, st, entries);
    default: return cudaErrorNotSupported;
    }
}

namespace {
// One thread waits, bounded by limit_ns, on phase 0 of an mbarrier nobody
// arrives on and, when the wait gives up, records it in the plan's error flag
// exactly as the transform kernels do when their input copy never lands.
__global__ void k_plan_wait_probe(int* err, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        pcxg::mbar_init(&bar, 1);
        pcxg::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !pcxg::mbar_wait_bounded(&bar, 0u, limit_ns)) atomicExch(err, 1);
}
}    // namespace

extern "C" int pcx_selftest_plan_wait(pcx_plan plan, unsigned long long limit_ns, void* stream) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        if (limit_ns > 2000000000ull) return pcx_fail(PCX_ERR_INVALID, "wait limit above 2 s");
        k_plan_wait_probe<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(plan->err, limit_ns);
        PCX_CUDA_TRY(cudaGetLastError());
        return PCX_OK;
    });
}

extern "C" int pcx_selftest_waits(unsigned long long mbar_limit_ns, int* mbar_satisfied, int* counter_satisfied) {
    return pcx_guard([&]() -> int {
        if (!mbar_satisfied || !counter_satisfied) return pcx_fail(PCX_ERR_INVALID, "null result pointer");
        int* d = nullptr;
        PCX_CUDA_TRY(cudaMalloc(&d, 4 * sizeof(int)));
        int         h[4] = {-1, -1, -1, 0};
        cudaError_t e    = cudaMemset(d, 0, 4 * sizeof(int));
        if (e == cudaSuccess) {
            k_wait_probe<<<1, 32>>>(d + 3, d, mbar_limit_ns);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(h, d, 3 * sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(d);
        PCX_CUDA_TRY(e);
        if (h[2] != 1) return pcx_fail(PCX_ERR_CUDA, "wait probe did not finish");
        *mbar_satisfied    = h[0];
        *counter_satisfied = h[1];
        return PCX_OK;
    });
}
