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

}  // extern "C"
