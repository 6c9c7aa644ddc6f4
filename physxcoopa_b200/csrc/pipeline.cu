// pipeline.cu -- pipelined read-back of cloth positions for callers that render frame k while
// frame k + 1 is simulated (what an engine's render thread does with the previous frame).
//
// pxb_cloths_read_positions_async snapshots the listed cloths' positions, in the caller's order,
// into one of two device buffers with the gather kernel on the step stream (so the snapshot is
// the state after every step enqueued before it), then copies the snapshot to the caller's host
// buffer on a separate copy stream that waits for the gather. The next step, enqueued right after
// on the step stream, runs while the copy engine moves the snapshot. pxb_cloths_wait_positions
// blocks until every pending copy has landed. Two snapshots may be in flight; a third call waits
// for the older one first. pxb_cloths_read_results_async does the same for the last step's
// per-cloth results (bounds, largest speed, time), gathered into the caller's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"
#include "pxb_kernels.h"
#include "runtime_internal.h"

using namespace pxb;

namespace {

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// The last step's per-cloth results in the caller's order: record k comes from launch slot
// slot[k], with the cloth's time after the step.
__global__ void gather_results_kernel(const PxbFrameResult* __restrict__ results, const int32_t* __restrict__ slot,
                                      const float* __restrict__ time, int n, PxbFrameResult* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        PxbFrameResult r = results[__ldg(&slot[k])];
        r.time = __ldg(&time[k]);
        out[k] = r;
    }
}

pxb_status ensure_pipeline(pxb_context* ctx) {
    if (ctx->copy_stream) return PXB_OK;
    if (pxb_status s = ctx->cuda(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream"))
        return s;
    for (int k = 0; k < 2; ++k)
        for (cudaEvent_t* ev : {&ctx->snap_ready[k], &ctx->snap_copied[k], &ctx->res_ready[k], &ctx->res_copied[k]})
            if (pxb_status s = ctx->cuda(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "event")) return s;
    return PXB_OK;
}

}  // namespace

extern "C" {

pxb_status pxb_cloths_read_positions_async(pxb_context* ctx, const uint64_t* cloths, uint32_t n, float* out,
                                           size_t capacity) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    std::vector<int32_t> order(n);
    std::vector<int64_t> offs(n);
    int64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        order[k] = static_cast<int32_t>(e - ctx->cloths.data());
        offs[k] = total;
        total += 3 * static_cast<int64_t>(e->n_particles);
    }
    if (static_cast<size_t>(total) > capacity) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "output too small");
    if (n == 0) return PXB_OK;
    if (pxb_status s = ensure_pipeline(ctx)) return s;
    if (pxb_status s = ctx->sync_registry()) return s;
    const int r = ctx->snap_next;
    // this snapshot buffer's previous copy must have landed before it is gathered into again
    if (ctx->snap_busy[r]) {
        if (pxb_status s = ctx->cuda(cudaEventSynchronize(ctx->snap_copied[r]), "wait for a snapshot copy")) return s;
        ctx->snap_busy[r] = false;
    }
    const size_t o_offs = align256(4 * static_cast<size_t>(n));
    if (pxb_status s = ctx->grow(ctx->d_snap_meta[r], o_offs + 8 * static_cast<size_t>(n), "snapshot meta")) return s;
    if (pxb_status s = ctx->grow(ctx->d_snap[r], 4 * static_cast<size_t>(total), "snapshot")) return s;
    char* meta = static_cast<char*>(ctx->d_snap_meta[r].p);
    pxb_status s = ctx->cuda(cudaMemcpyAsync(meta, order.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), "snapshot order");
    if (!s) s = ctx->cuda(cudaMemcpyAsync(meta + o_offs, offs.data(), 8 * n, cudaMemcpyHostToDevice, ctx->stream),
                          "snapshot offsets");
    if (s) return s;
    cudaError_t le = launch_gather_positions(static_cast<const PxbClothDev*>(ctx->d_registry.p),
                                             reinterpret_cast<const int32_t*>(meta),
                                             reinterpret_cast<const int64_t*>(meta + o_offs), static_cast<int>(n),
                                             static_cast<float*>(ctx->d_snap[r].p), ctx->stream);
    if (le != cudaSuccess) return ctx->cuda(le, "launch snapshot gather");
    ++ctx->launches;
    if ((s = ctx->cuda(cudaEventRecord(ctx->snap_ready[r], ctx->stream), "record snapshot"))) return s;
    if ((s = ctx->cuda(cudaStreamWaitEvent(ctx->copy_stream, ctx->snap_ready[r], 0), "copy waits for snapshot"))) return s;
    // in 4 MB pieces: a small device-to-host read on the step stream (the step's results, the
    // error word) then waits for one piece, not for the whole snapshot
    constexpr size_t kPiece = size_t(4) << 20;
    const size_t bytes = 4 * static_cast<size_t>(total);
    for (size_t o = 0; o < bytes; o += kPiece)
        if ((s = ctx->cuda(cudaMemcpyAsync(reinterpret_cast<char*>(out) + o, static_cast<char*>(ctx->d_snap[r].p) + o,
                                           std::min(kPiece, bytes - o), cudaMemcpyDeviceToHost, ctx->copy_stream),
                           "copy snapshot")))
            return s;
    if ((s = ctx->cuda(cudaEventRecord(ctx->snap_copied[r], ctx->copy_stream), "record snapshot copy"))) return s;
    ctx->snap_busy[r] = true;
    ctx->snap_next = r ^ 1;
    return PXB_OK;
}

pxb_status pxb_cloths_read_results_async(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                         pxb_cloth_frame_result* out) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    if (n == 0) return PXB_OK;
    if (ctx->last_step_warm) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "the last step was a warm-start step");
    // launch slot of every cloth of the last step
    std::vector<int32_t> slot(n);
    std::vector<float> time(n);
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        const int32_t q = e->last_slot;
        if (q < 0 || static_cast<size_t>(q) >= ctx->last_step.size() || ctx->last_step[q] != cloths[k])
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "cloth %llu was not in the last step",
                             (unsigned long long)cloths[k]);
        slot[k] = q;
        time[k] = e->time;
    }
    if (pxb_status s = ensure_pipeline(ctx)) return s;
    const int r = ctx->res_next;
    if (ctx->res_busy[r]) {
        if (pxb_status s = ctx->cuda(cudaEventSynchronize(ctx->res_copied[r]), "wait for a results copy")) return s;
        ctx->res_busy[r] = false;
    }
    const size_t o_time = align256(4 * static_cast<size_t>(n)), o_out = o_time + align256(4 * static_cast<size_t>(n));
    if (pxb_status s = ctx->grow(ctx->d_res_snap[r], o_out + sizeof(PxbFrameResult) * n, "results snapshot")) return s;
    char* b = static_cast<char*>(ctx->d_res_snap[r].p);
    pxb_status s = ctx->cuda(cudaMemcpyAsync(b, slot.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), "results slots");
    if (!s) s = ctx->cuda(cudaMemcpyAsync(b + o_time, time.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), "results times");
    if (s) return s;
    gather_results_kernel<<<static_cast<int>(std::min<uint32_t>((n + 255) / 256, 1024)), 256, 0, ctx->stream>>>(
        static_cast<const PxbFrameResult*>(ctx->d_results.p), reinterpret_cast<const int32_t*>(b),
        reinterpret_cast<const float*>(b + o_time), static_cast<int>(n), reinterpret_cast<PxbFrameResult*>(b + o_out));
    if ((s = ctx->cuda(cudaGetLastError(), "launch results gather"))) return s;
    ++ctx->launches;
    if ((s = ctx->cuda(cudaEventRecord(ctx->res_ready[r], ctx->stream), "record results"))) return s;
    if ((s = ctx->cuda(cudaStreamWaitEvent(ctx->copy_stream, ctx->res_ready[r], 0), "copy waits for results"))) return s;
    static_assert(sizeof(pxb_cloth_frame_result) == sizeof(PxbFrameResult), "result layout");
    if ((s = ctx->cuda(cudaMemcpyAsync(out, b + o_out, sizeof(PxbFrameResult) * n, cudaMemcpyDeviceToHost,
                                       ctx->copy_stream),
                       "copy results")))
        return s;
    if ((s = ctx->cuda(cudaEventRecord(ctx->res_copied[r], ctx->copy_stream), "record results copy"))) return s;
    ctx->res_busy[r] = true;
    ctx->res_next = r ^ 1;
    return PXB_OK;
}

pxb_status pxb_cloths_wait_positions(pxb_context* ctx) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 2; ++k) {
        if (ctx->snap_busy[k]) {
            if (pxb_status s = ctx->cuda(cudaEventSynchronize(ctx->snap_copied[k]), "wait for a snapshot copy")) return s;
            ctx->snap_busy[k] = false;
        }
        if (ctx->res_busy[k]) {
            if (pxb_status s = ctx->cuda(cudaEventSynchronize(ctx->res_copied[k]), "wait for a results copy")) return s;
            ctx->res_busy[k] = false;
        }
    }
    return ctx->check_device_error();
}

}  // extern "C"
