// noalloc.cu -- pxb_cloths_gather_positions_device: the position gather of
// pxb_cloths_read_positions into a caller-provided device buffer, with no allocation at all.
//
// Who needs it: callers that may not allocate device memory while they run -- a renderer or
// recorder that reads cloth positions every frame from inside a fixed device memory budget,
// or code running where cudaMalloc / cudaFree would stall the device (they synchronise it) or
// is not allowed at all. pxb_cloths_read_positions grows internal device buffers on demand;
// this entry point never does.
//
// Its only scratch, the per-call cloth list (registry slot and output offset of each cloth),
// lives in a fixed-size array compiled into the library: kMaxCloths entries, 48 KB, present on
// every GPU that loads the library until the process exits. Host code gets the array's device
// address with cudaGetSymbolAddress once per context, on the context's first call (the set-up),
// and keeps it on the context: a context made after a device reset, or in another CUDA context
// of the device, looks the address up again. Every call overwrites the entries it uses before its kernel reads them, so
// nothing has to start at zero; but all calls share the one array, so calls that can run at the
// same time on the GPU (from different contexts or streams of one device) race, and must be
// serialised by the caller. Calls on one context are ordered on its stream.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "pxb_kernels.h"
#include "runtime_internal.h"

using namespace pxb;

namespace {

constexpr uint32_t kMaxCloths = 4096;
constexpr size_t kOrderBytes = 4 * kMaxCloths;   // int32 registry slot per cloth
constexpr size_t kOffsetBytes = 8 * kMaxCloths;  // int64 first output float per cloth

static __device__ __align__(256) unsigned char g_gather_scratch[kOrderBytes + kOffsetBytes];

constexpr int kMaxDevices = 64;

// The per-call cloth list is assembled in host memory that is also static (no allocation and no
// 48 KB on the caller's stack, which render and worker threads may not have): one buffer for the
// process, filled and uploaded under this mutex. Its upload is a pageable copy, so the buffer is
// free again when cudaMemcpyAsync returns.
std::mutex g_list_mutex;
int32_t g_order[kMaxCloths];
int64_t g_offs[kMaxCloths];

// The device address of g_gather_scratch in the context's device (which must be current),
// looked up at the context's first call.
cudaError_t scratch_of(pxb_context* ctx, unsigned char** out) {
    if (!ctx->gather_scratch) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_gather_scratch);
        if (e != cudaSuccess) return e;
        ctx->gather_scratch = static_cast<unsigned char*>(p);
    }
    *out = ctx->gather_scratch;
    return cudaSuccess;
}

}  // namespace

extern "C" {

pxb_status pxb_cloths_gather_positions_device(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                              float* out_device, size_t capacity) {
    if (!ctx || (n && (!cloths || !out_device))) return PXB_ERR_INVALID_ARGUMENT;
    if (n > kMaxCloths)
        return ctx->fail(PXB_ERR_TOO_LARGE, "%u cloths in one call; this entry point takes at most %u", n, kMaxCloths);
    if (n == 0) return PXB_OK;
    if (ctx->registry_dirty)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT,
                         "cloths were added, removed or changed since the last step: step them (or call "
                         "pxb_cloths_read_positions) once before gathering without allocation");
    int device = -1;
    if (pxb_status s = ctx->cuda(cudaGetDevice(&device), "current device")) return s;
    if (device != ctx->device || device < 0 || device >= kMaxDevices)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "the context's device (%d) is not the current device (%d)",
                         ctx->device, device);
    unsigned char* scratch = nullptr;
    if (pxb_status s = ctx->cuda(scratch_of(ctx, &scratch), "look up the gather scratch")) return s;
    {
        std::lock_guard<std::mutex> lock(g_list_mutex);
        int64_t total = 0;
        for (uint32_t k = 0; k < n; ++k) {
            ClothEntry* e = ctx->lookup(cloths[k]);
            if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
            g_order[k] = static_cast<int32_t>(e - ctx->cloths.data());
            g_offs[k] = total;
            total += 3 * static_cast<int64_t>(e->n_particles);
        }
        if (static_cast<size_t>(total) > capacity) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "output too small");
        // Pageable host sources: each copy has left the host buffers when cudaMemcpyAsync
        // returns, and runs in stream order before the kernel.
        if (pxb_status s = ctx->cuda(cudaMemcpyAsync(scratch, g_order, 4 * static_cast<size_t>(n),
                                                     cudaMemcpyHostToDevice, ctx->stream), "upload gather order"))
            return s;
        if (pxb_status s = ctx->cuda(cudaMemcpyAsync(scratch + kOrderBytes, g_offs, 8 * static_cast<size_t>(n),
                                                     cudaMemcpyHostToDevice, ctx->stream), "upload gather offsets"))
            return s;
    }
    cudaError_t le = launch_gather_positions(static_cast<const PxbClothDev*>(ctx->d_registry.p),
                                             reinterpret_cast<const int32_t*>(scratch),
                                             reinterpret_cast<const int64_t*>(scratch + kOrderBytes),
                                             static_cast<int>(n), out_device, ctx->stream);
    if (le != cudaSuccess) return ctx->cuda(le, "launch gather");
    ++ctx->launches;
    return PXB_OK;
}

}  // extern "C"
