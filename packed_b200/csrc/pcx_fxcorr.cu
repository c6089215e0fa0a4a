// Overlap-save correlation (fxcorr_unit).  Placeholder until the fused kernel lands.
#include "pcx_host.hpp"

struct pcx_fxcorr_s {};

extern "C" int pcx_fxcorr_create(pcx_fxcorr* h, const void*, size_t, int, size_t, int) {
    if (h) *h = nullptr;
    return pcx_fail(PCX_ERR_UNSUPPORTED, "fxcorr not built yet");
}
extern "C" int pcx_fxcorr_destroy(pcx_fxcorr) { return PCX_OK; }
extern "C" int pcx_fxcorr_exec(pcx_fxcorr, void*, const void*, size_t, int, size_t, size_t, size_t, void*) {
    return pcx_fail(PCX_ERR_UNSUPPORTED, "fxcorr not built yet");
}
extern "C" int pcx_fxcorr_vjp(pcx_fxcorr, void*, void*, const void*, const void*, size_t, int, size_t, size_t,
                              void*) {
    return pcx_fail(PCX_ERR_UNSUPPORTED, "fxcorr not built yet");
}
