// runtime_mlp.cu -- C-ABI of the warm-start network: weights in and out, batch inference.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "pxb_kernels.h"
#include "pxb_mlp.cuh"
#include "runtime_internal.h"

using namespace pxb;

namespace {

bool finite_weights(const pxb_mlp_weights& w) {
    const float* f = reinterpret_cast<const float*>(&w);
    for (size_t i = 0; i < sizeof(w) / sizeof(float); ++i)
        if (!std::isfinite(f[i])) return false;
    return true;
}

}  // namespace

pxb_status pxb_context::upload_mlp() {
    std::vector<unsigned char> blob(kMlpBlobBytes);
    mlp_pack_blob(mlp, blob.data());
    if (pxb_status s = grow(d_mlp, kMlpBlobBytes, "network weights")) return s;
    if (pxb_status s = cuda(cudaMemcpyAsync(d_mlp.p, blob.data(), kMlpBlobBytes, cudaMemcpyHostToDevice, stream),
                            "upload network"))
        return s;
    return cuda(cudaStreamSynchronize(stream), "upload network");
}

extern "C" {

pxb_status pxb_mlp_set_weights(pxb_context* ctx, const pxb_mlp_weights* weights) {
    if (!ctx || !weights) return PXB_ERR_INVALID_ARGUMENT;
    if (!finite_weights(*weights)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "network weights are not all finite");
    ctx->mlp = *weights;
    ctx->has_mlp = true;
    return ctx->upload_mlp();
}

pxb_status pxb_mlp_get_weights(pxb_context* ctx, pxb_mlp_weights* out) {
    if (!ctx || !out) return PXB_ERR_INVALID_ARGUMENT;
    if (!ctx->has_mlp) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "no network installed");
    *out = ctx->mlp;
    return PXB_OK;
}

pxb_status pxb_mlp_infer(pxb_context* ctx, const float* features, uint32_t n, float* out) {
    if (!ctx || (n && (!features || !out))) return PXB_ERR_INVALID_ARGUMENT;
    if (!ctx->has_mlp) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "no network installed");
    if (n == 0) return PXB_OK;
    const size_t in_b = sizeof(float) * kMlpIn * static_cast<size_t>(n);
    const size_t out_b = sizeof(float) * kMlpOut * static_cast<size_t>(n);
    const size_t o_out = (in_b + 255) & ~static_cast<size_t>(255);
    if (pxb_status s = ctx->grow(ctx->d_mlp_io, o_out + out_b, "network batch")) return s;
    char* base = static_cast<char*>(ctx->d_mlp_io.p);
    if (pxb_status s = ctx->cuda(cudaMemcpyAsync(base, features, in_b, cudaMemcpyHostToDevice, ctx->stream),
                                 "upload features"))
        return s;
    cudaError_t le = launch_mlp_infer(reinterpret_cast<const float*>(base), static_cast<int>(n),
                                      static_cast<const unsigned char*>(ctx->d_mlp.p),
                                      reinterpret_cast<float*>(base + o_out), ctx->d_err, ctx->n_sms, ctx->stream);
    if (le != cudaSuccess) return ctx->cuda(le, "launch network");
    ++ctx->launches;
    if (pxb_status s = ctx->cuda(cudaMemcpyAsync(out, base + o_out, out_b, cudaMemcpyDeviceToHost, ctx->stream),
                                 "read network output"))
        return s;
    return ctx->check_device_error();
}

pxb_status pxb_cloths_step_warm(pxb_context* ctx, const pxb_cloth_step_desc* step, const pxb_warm_start_desc* warm) {
    if (!ctx || !step || !warm) return PXB_ERR_INVALID_ARGUMENT;
    pxb_context::WarmCfg cfg;
    cfg.warm_iters = static_cast<int>(warm->warm_iterations);
    cfg.tau = warm->residual_threshold;
    cfg.taus = warm->thresholds;
    return ctx->step_cloths(step, &cfg);
}

pxb_status pxb_cloths_read_warm_results(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                        pxb_cloth_warm_result* out) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    if (pxb_status s = ctx->fetch_warm_results()) return s;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        if (!e->has_warm_result) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "cloth has no warm-start step");
        out[k].residual = e->warm_result.residual;
        out[k].fallbacks = static_cast<uint32_t>(e->warm_result.fallbacks);
        out[k].substeps = static_cast<uint32_t>(e->warm_result.substeps);
    }
    return PXB_OK;
}

pxb_status pxb_cloths_record(pxb_context* ctx, const pxb_cloth_step_desc* step, uint32_t substep,
                             float* features, float* targets, uint64_t capacity, uint64_t* rows_out) {
    if (!ctx || !step || !rows_out || (capacity && (!features || !targets))) return PXB_ERR_INVALID_ARGUMENT;
    *rows_out = 0;
    if (step->n_cloths && !step->cloths) return PXB_ERR_INVALID_ARGUMENT;
    std::vector<int64_t> row0(step->n_cloths);
    int64_t rows = 0;
    for (uint32_t k = 0; k < step->n_cloths; ++k) {
        ClothEntry* e = ctx->lookup(step->cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        row0[k] = rows;
        rows += e->n_layout;
    }
    const size_t bytes = sizeof(float) * static_cast<size_t>(rows) * (kMlpIn + 4);
    if (pxb_status s = ctx->grow(ctx->d_rec, std::max<size_t>(bytes, 16), "recording buffer")) return s;
    pxb_context::WarmCfg cfg;
    cfg.record = 1;
    cfg.record_substep = static_cast<int>(substep);
    cfg.rec_x = static_cast<float*>(ctx->d_rec.p);
    cfg.rec_y = cfg.rec_x + static_cast<size_t>(rows) * kMlpIn;
    cfg.rec_row0 = row0.data();
    if (pxb_status s = ctx->step_cloths(step, &cfg)) return s;
    std::vector<float> h(static_cast<size_t>(rows) * (kMlpIn + 4));
    if (rows) {
        if (pxb_status s = ctx->cuda(cudaMemcpyAsync(h.data(), ctx->d_rec.p, bytes, cudaMemcpyDeviceToHost, ctx->stream),
                                     "read recording"))
            return s;
    }
    if (pxb_status s = ctx->check_device_error()) return s;
    const float* hx = h.data();
    const float* hy = hx + static_cast<size_t>(rows) * kMlpIn;
    uint64_t w = 0;
    for (int64_t r = 0; r < rows && w < capacity; ++r) {
        if (hy[4 * r + 3] == 0.0f) continue;  // pinned, anchored or ghost slot
        std::memcpy(features + w * kMlpIn, hx + r * kMlpIn, sizeof(float) * kMlpIn);
        std::memcpy(targets + w * 3, hy + 4 * r, sizeof(float) * 3);
        ++w;
    }
    *rows_out = w;
    return PXB_OK;
}

}  // extern "C"
