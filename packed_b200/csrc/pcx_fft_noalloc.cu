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
// address, so its device address is looked up with cudaGetSymbolAddress once
// per device (with that device current) on the first call on that device and
// passed to the kernels.  That first call should therefore come before any
// stream capture.  Calls share the array and it keeps the last call's
// contents; the four-step passes write every scratch element before reading
// it, so nothing needs clearing.  Calls whose GPU work overlaps (different
// streams, other threads) race on the array.
#include "pcx_host.hpp"

#include <mutex>
#include <string>

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[PCX_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
void*         g_scratch_ptr[MAX_DEVICES];
std::mutex    g_scratch_mutex;

// Device address of g_noalloc_scratch on the current device (looked up once).
int scratch_address(void** out) {
    int dev = 0;
    PCX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return pcx_fail(PCX_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void*       p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            return pcx_fail(PCX_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
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
