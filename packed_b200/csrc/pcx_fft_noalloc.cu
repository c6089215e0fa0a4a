// Allocation-free variant of the batched FFT (pcx_fft_exec_noalloc).
//
// Some callers cannot allocate device memory once they are running: a
// real-time signal-processing loop that owns a fixed memory budget set at
// start-up, an embedding whose device memory is handed out only by its own
// pool, or a deployment whose rules forbid device allocation after
// initialisation.  pcx_fft_exec allocates the four-step scratch on first use
// for sizes above 4096; this entry point instead uses one file-scope device
// array of PCX_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library
// holds until the process exits.
//
// The array's name in host code is a host-side stand-in, not a device
// address, so its device address is looked up with cudaGetSymbolAddress, with
// the device current, on the first call on that device (set-up) and passed to
// the kernels.  That lookup also makes the CUDA runtime load the array's
// module (with lazy module loading, the default, the 8 MiB are committed
// then, by the loader), so the first call on each device belongs in the
// caller's initialisation and should come before any stream capture.  The
// address is cached per device together with the context it was looked up
// in, and looked up again when the device's context has changed (after a
// reset the module is loaded anew and may sit elsewhere).  Calls share the
// array and it keeps the last call's contents; the four-step passes write
// every scratch element before reading it, so nothing needs clearing.  Calls
// whose GPU work overlaps (different streams, other threads) race on the
// array.
#include "pcx_host.hpp"

#include <mutex>
#include <string>

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[PCX_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
struct scratch_entry {
    void* ctx;    // CUcontext current when the address was looked up
    void* ptr;
};
scratch_entry g_scratch[MAX_DEVICES];
std::mutex    g_scratch_mutex;

// cuCtxGetCurrent through the runtime's driver entry point (no -lcuda).
using ctx_get_fn = int (*)(void**);
ctx_get_fn ctx_get() {
    static ctx_get_fn f = []() -> ctx_get_fn {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            return nullptr;
        }
        return reinterpret_cast<ctx_get_fn>(p);
    }();
    return f;
}
void* current_ctx() {
    void* c = nullptr;
    if (ctx_get_fn f = ctx_get()) {
        if (f(&c) != 0) c = nullptr;
    }
    return c;
}

// Device address of g_noalloc_scratch on the current device.
int scratch_address(void** out) {
    int dev = 0;
    PCX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return pcx_fail(PCX_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    scratch_entry&              e   = g_scratch[dev];
    void*                       ctx = current_ctx();
    if (!e.ptr || !ctx || e.ctx != ctx) {
        void*       p  = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (rc != cudaSuccess || !p) {
            return pcx_fail(PCX_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(rc));
        }
        e.ptr = p;
        e.ctx = current_ctx();    // the lookup has made the primary context current
    }
    *out = e.ptr;
    return PCX_OK;
}

}    // namespace

extern "C" int pcx_fft_exec_noalloc(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst,
                                    int pack_src, int direction, int normalize, size_t batch, size_t dst_stride,
                                    size_t src_stride, void* stream) {
    return pcx_guard([&]() -> int {
        if (!plan) return pcx_fail(PCX_ERR_INVALID, "plan is null");
        if (plan->two_pass) {
            // one chunk of the four-step must fit: at least one whole transform
            const size_t one = plan->n * plan->elem_bytes();
            if (one > (size_t)PCX_NOALLOC_SCRATCH_BYTES) {
                return pcx_fail(PCX_ERR_UNSUPPORTED,
                                "fft_size (which is " + std::to_string(plan->n) + ") needs " + std::to_string(one) +
                                    " bytes of scratch per transform; pcx_fft_exec_noalloc has " +
                                    std::to_string((size_t)PCX_NOALLOC_SCRATCH_BYTES));
            }
        }
        void* scratch = nullptr;
        if (plan->two_pass) {
            if (int rc = scratch_address(&scratch)) return rc;
        }
        // pcx_fft_run uses the given workspace (chunking the batch to fit it)
        // and allocates nothing when one is supplied.
        const size_t cap = plan->two_pass ? (size_t)PCX_NOALLOC_SCRATCH_BYTES / (plan->n * plan->elem_bytes()) : 0;
        return pcx_fft_run(plan, dst, src, src_len, pack_dst, pack_src, direction, normalize, batch, dst_stride,
                           src_stride, scratch, plan->two_pass ? (size_t)PCX_NOALLOC_SCRATCH_BYTES : 0,
                           static_cast<cudaStream_t>(stream), 1.0, cap);
    });
}
