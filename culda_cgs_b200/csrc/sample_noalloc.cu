// sample_noalloc.cu — culda_sample_noalloc: the kernel-level sampler with its
// scratch memory in a fixed device array instead of a caller workspace.
//
// Who needs it: a serving process whose own pool allocator reserved all
// device memory up front and lets no library call cudaMalloc cannot hand
// culda_sample a workspace allocated for this purpose.  This entry point
// allocates nothing: the sampler's scratch (work-queue head, error word,
// per-item log terms, rows of hot words) lives in `g_sample_scratch`, a
// file-scope device array that every GPU which loads the library holds until
// the process exits.  Each call still reads culda_sample's theta range check
// back to the host, so it returns only once its stream has drained.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/culda_b200.h"
#include "internal.h"

namespace {

static_assert(CULDA_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size must keep 256-byte alignment");

// The scratch itself.  Host code may not use this name as an address (on the
// host it is a stand-in symbol, not device memory): the device address comes
// from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_sample_scratch[CULDA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (the lookup loads the library's device code on that device if it is
// not loaded yet) and kept for the life of the process: a cudaDeviceReset
// unloads the module, after which the kept address is stale.
int scratch_address(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        culda::set_global_error("culda_sample_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return CULDA_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        culda::set_global_error("culda_sample_noalloc: device %d beyond the %d devices it supports", dev, kMaxDevices);
        return CULDA_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sample_scratch);
        if (e != cudaSuccess || !p) {
            culda::set_global_error("culda_sample_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return CULDA_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CULDA_OK;
}

}  // namespace

extern "C" int culda_sample_noalloc(const culda_sample_args *a, void *stream) {
    if (!a) {
        culda::set_global_error("culda_sample_noalloc: null arguments");
        return CULDA_ERR_INVALID_ARG;
    }
    // reject malformed sizes before they reach the size arithmetic below
    if (a->k < 32 || a->k > 4096 || (a->k % 32) != 0 || a->num_items <= 0 || a->num_hot < 0) {
        culda::set_global_error("culda_sample_noalloc: invalid argument (k %d, num_items %d, num_hot %d)", a->k,
                                a->num_items, a->num_hot);
        return CULDA_ERR_INVALID_ARG;
    }
    const size_t need = culda_sample_workspace(a->k, a->num_items, a->num_hot);
    if (need > (size_t)CULDA_NOALLOC_SCRATCH_BYTES) {
        culda::set_global_error(
            "culda_sample_noalloc: this work list needs %zu bytes of scratch but the fixed device array holds %zu "
            "(use fewer work items or fewer hot words, or culda_sample with a workspace)",
            need, (size_t)CULDA_NOALLOC_SCRATCH_BYTES);
        return CULDA_ERR_UNSUPPORTED;
    }
    void *scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != CULDA_OK) return rc;
    // culda_sample clears the parts of the workspace that must start at zero
    // (work-queue head, error word, hot rows) on every call and writes every
    // per-item slot it later reads.
    return culda_sample(a, scratch, (size_t)CULDA_NOALLOC_SCRATCH_BYTES, stream);
}
