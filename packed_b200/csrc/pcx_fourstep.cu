// Instantiations and launch of the one-launch four-step kernel (k_fourstep).
#include "pcx_fourstep.cuh"
#include "pcx_v2_launch.cuh"

namespace pcxg {

template<class T, int LOGN1, int LOGN2>
static cudaError_t launch_fs(const fs_args& a, cudaStream_t st, int sms, bool attr_only, int* tc, int* tr,
                             int* per_sm) {
    using F = fs_cfg<T, LOGN1, LOGN2>;
    static_assert(F::SMEM <= 232448, "shared memory per block");
    static_assert(F::MINB * (F::SMEM + 1024 + 256) <= 233472, "blocks per SM fit the shared memory");
    static_assert(F::STAGE % 128 == 0, "TMA destinations stay 128-byte aligned");
    auto kern = k_fourstep<T, LOGN1, LOGN2>;
    if (tc) *tc = F::TC;
    if (tr) *tr = F::TR;
    if (attr_only) {
        cudaError_t e = set_smem(kern, F::SMEM);
        if (e == cudaSuccess && per_sm) e = occupancy_cached(reinterpret_cast<const void*>(kern), F::NT + 32, F::SMEM, per_sm);
        return e;
    }
    const long long items = a.batch * (F::TC + F::TR);
    if (items == 0) return cudaSuccess;
    // 3-D view of the source: [transform][n1][2*N2 reals], box = 64 bytes x min(N1, 256) rows
    CUtensorMap      map;
    const cuuint64_t dims[3]    = {(cuuint64_t)2 << LOGN2, (cuuint64_t)1 << LOGN1, (cuuint64_t)a.batch};
    const long long  ss         = a.batch > 1 ? a.src_stride : (2LL << (LOGN1 + LOGN2));    // unused when 1 row
    const cuuint64_t strides[2] = {((cuuint64_t)2 << LOGN2) * sizeof(T), (cuuint64_t)ss * sizeof(T)};
    const cuuint32_t box[3]     = {(cuuint32_t)(2 * F::C), (cuuint32_t)F::BOXY, 1};
    const cuuint32_t estr[3]    = {1, 1, 1};
    cudaError_t      e = encode_tensor_map(&map, sizeof(T) == 8, 3, const_cast<void*>(a.src), dims, strides, box, estr);
    if (e != cudaSuccess) return e;
    unsigned grid = 0;
    e             = persistent_grid(kern, F::NT + 32, F::SMEM, items, sms, &grid);
    if (e != cudaSuccess) return e;
    kern<<<grid, F::NT + 32, F::SMEM, st>>>(map, a);
    return cudaGetLastError();
}

template<class T>
static cudaError_t dispatch_fs(int l1, int l2, const fs_args& a, cudaStream_t st, int sms, bool attr_only, int* tc,
                               int* tr, int* per_sm) {
    switch (l1 * 32 + l2) {
    case 7 * 32 + 7: return launch_fs<T, 7, 7>(a, st, sms, attr_only, tc, tr, per_sm);
    case 8 * 32 + 7: return launch_fs<T, 8, 7>(a, st, sms, attr_only, tc, tr, per_sm);
    case 8 * 32 + 8: return launch_fs<T, 8, 8>(a, st, sms, attr_only, tc, tr, per_sm);
    case 9 * 32 + 8: return launch_fs<T, 9, 8>(a, st, sms, attr_only, tc, tr, per_sm);
    case 9 * 32 + 9: return launch_fs<T, 9, 9>(a, st, sms, attr_only, tc, tr, per_sm);
    case 10 * 32 + 9: return launch_fs<T, 10, 9>(a, st, sms, attr_only, tc, tr, per_sm);
    case 10 * 32 + 10: return launch_fs<T, 10, 10>(a, st, sms, attr_only, tc, tr, per_sm);
    default: return cudaErrorNotSupported;
    }
}

}    // namespace pcxg

cudaError_t pcx_fourstep(bool f64, int log_n1, int log_n2, const pcxg::fs_args& a, cudaStream_t st, int sms,
                         bool attr_only, int* col_tiles, int* row_tiles, int* blocks_per_sm) {
    return f64 ? pcxg::dispatch_fs<double>(log_n1, log_n2, a, st, sms, attr_only, col_tiles, row_tiles, blocks_per_sm)
               : pcxg::dispatch_fs<float>(log_n1, log_n2, a, st, sms, attr_only, col_tiles, row_tiles, blocks_per_sm);
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
