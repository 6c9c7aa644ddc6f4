// runtime_mlp.cu -- C-ABI of the warm-start network: weights in and out, batch inference.
#include <cuda_runtime.h>

#include <algorithm>
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

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return static_cast<double>(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }
double normal01(uint64_t& s) {
    const double u1 = std::max(uniform01(s), 1e-300), u2 = uniform01(s);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// Normalisation from the data: feature mean and inverse standard deviation, target root mean
// square (floors keep constant columns finite).
void fit_normalisation(const float* X, const float* Y, uint64_t n, pxb_mlp_weights& w) {
    double mx[kMlpIn] = {}, sx[kMlpIn] = {}, sy[kMlpOut] = {};
    for (uint64_t r = 0; r < n; ++r)
        for (int k = 0; k < kMlpIn; ++k) mx[k] += X[r * kMlpIn + k];
    for (int k = 0; k < kMlpIn; ++k) mx[k] /= static_cast<double>(n);
    for (uint64_t r = 0; r < n; ++r) {
        for (int k = 0; k < kMlpIn; ++k) {
            const double d = X[r * kMlpIn + k] - mx[k];
            sx[k] += d * d;
        }
        for (int j = 0; j < kMlpOut; ++j) sy[j] += static_cast<double>(Y[r * 3 + j]) * Y[r * 3 + j];
    }
    for (int k = 0; k < kMlpIn; ++k) {
        const double sd = std::sqrt(sx[k] / static_cast<double>(n));
        w.in_mean[k] = static_cast<float>(mx[k]);
        w.in_scale[k] = static_cast<float>(1.0 / std::max(sd, 1e-12));
    }
    for (int j = 0; j < kMlpOut; ++j)
        w.out_scale[j] = static_cast<float>(std::max(std::sqrt(sy[j] / static_cast<double>(n)), 1e-12));
}

size_t al256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

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

pxb_status pxb_mlp_train(pxb_context* ctx, const float* features, const float* targets, uint64_t n,
                         const pxb_mlp_train_desc* desc, float* final_loss) {
    if (!ctx || !desc || !features || !targets || n == 0) return PXB_ERR_INVALID_ARGUMENT;
    if (n > 0x7FFFFFFFull) return ctx->fail(PXB_ERR_TOO_LARGE, "more than 2^31 training rows");
    const uint32_t batch = std::max<uint32_t>(desc->batch, 1);
    // initial weights: N(0, 1 / fan_in), the last layer scaled down by 10
    pxb_mlp_weights w{};
    uint64_t seed = desc->seed;
    for (int o = 0; o < kMlpHidden; ++o)
        for (int i = 0; i < kMlpIn; ++i) w.w1[o][i] = static_cast<float>(normal01(seed) / std::sqrt(double(kMlpIn)));
    for (int o = 0; o < kMlpHidden; ++o)
        for (int i = 0; i < kMlpHidden; ++i)
            w.w2[o][i] = static_cast<float>(normal01(seed) / std::sqrt(double(kMlpHidden)));
    for (int o = 0; o < kMlpOut; ++o)
        for (int i = 0; i < kMlpHidden; ++i)
            w.w3[o][i] = static_cast<float>(0.1 * normal01(seed) / std::sqrt(double(kMlpHidden)));
    fit_normalisation(features, targets, n, w);

    // device: X | Y | row order | W | M | V | loss | gradient partials (one block per CTA)
    const size_t bx = sizeof(float) * kMlpIn * n, by = sizeof(float) * 3 * n, bi = sizeof(uint32_t) * n;
    const size_t bw = sizeof(pxb_mlp_weights), bp = sizeof(float) * mlp_partial_floats(ctx->n_sms);
    const size_t oy = al256(bx), oi = oy + al256(by), ow = oi + al256(bi), om = ow + al256(bw), ov = om + al256(bw),
                 ol = ov + al256(bw), op = ol + 256, total = op + al256(bp);
    DevBuf buf;
    if (pxb_status s = ctx->grow(buf, total, "training buffers")) return s;
    char* b = static_cast<char*>(buf.p);
    auto* X = reinterpret_cast<float*>(b);
    auto* Y = reinterpret_cast<float*>(b + oy);
    auto* I = reinterpret_cast<uint32_t*>(b + oi);
    auto* W = reinterpret_cast<pxb_mlp_weights*>(b + ow);
    auto* M = reinterpret_cast<pxb_mlp_weights*>(b + om);
    auto* V = reinterpret_cast<pxb_mlp_weights*>(b + ov);
    auto* L = reinterpret_cast<float*>(b + ol);
    auto* part = reinterpret_cast<float*>(b + op);
    cudaStream_t st = ctx->stream;
    pxb_status s = PXB_OK;
    auto chk = [&](cudaError_t e, const char* what) {
        if (!s && e != cudaSuccess) s = ctx->cuda(e, what);
    };
    chk(cudaMemcpyAsync(X, features, bx, cudaMemcpyHostToDevice, st), "upload training features");
    chk(cudaMemcpyAsync(Y, targets, by, cudaMemcpyHostToDevice, st), "upload training targets");
    chk(cudaMemcpyAsync(W, &w, bw, cudaMemcpyHostToDevice, st), "upload initial weights");
    chk(cudaMemsetAsync(M, 0, ov + al256(bw) - om, st), "zero optimiser state");
    std::vector<uint32_t> order(n);
    for (uint64_t r = 0; r < n; ++r) order[r] = static_cast<uint32_t>(r);
    float epoch_loss = 0.0f;
    uint64_t t = 0;
    const uint32_t epochs = std::max<uint32_t>(desc->epochs, 1);
    for (uint32_t ep = 0; ep < epochs && !s; ++ep) {
        for (uint64_t r = n - 1; r > 0; --r) std::swap(order[r], order[splitmix(seed) % (r + 1)]);
        chk(cudaMemcpyAsync(I, order.data(), bi, cudaMemcpyHostToDevice, st), "upload batch order");
        chk(cudaMemsetAsync(L, 0, sizeof(float), st), "zero loss");
        // cosine learning-rate schedule over the epochs
        const float lr = desc->learning_rate * 0.5f * (1.0f + std::cos(3.14159265f * ep / epochs));
        for (uint64_t r0 = 0; r0 < n && !s; r0 += batch) {
            const int rows = static_cast<int>(std::min<uint64_t>(batch, n - r0));
            ++t;
            cudaError_t ge = cudaSuccess;
            const int parts = launch_mlp_grad(X, Y, I + r0, rows, rows, W, part, ctx->d_err, ctx->n_sms, st, &ge);
            chk(ge, "launch gradients");
            chk(launch_mlp_adam(part, parts, ctx->n_sms, W, M, V, lr, std::pow(0.9f, float(t)),
                                std::pow(0.999f, float(t)), L, st),
                "launch adam");
            ctx->launches += 2;
        }
        float lsum = 0.0f;
        chk(cudaMemcpyAsync(&lsum, L, sizeof(float), cudaMemcpyDeviceToHost, st), "read loss");
        chk(cudaStreamSynchronize(st), "training epoch");
        // every batch added the squared errors of its rows: the epoch's mean over rows and outputs
        epoch_loss = lsum / (3.0f * static_cast<float>(n));
    }
    pxb_mlp_weights out{};
    chk(cudaMemcpyAsync(&out, W, bw, cudaMemcpyDeviceToHost, st), "read trained weights");
    chk(cudaStreamSynchronize(st), "training");
    cudaFree(buf.p);
    if (s) return s;
    if (pxb_status e = ctx->check_device_error()) return e;
    if (!finite_weights(out)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "training diverged (non-finite weights)");
    if (final_loss) *final_loss = epoch_loss;
    ctx->mlp = out;
    ctx->has_mlp = true;
    return ctx->upload_mlp();
}

pxb_status pxb_mlp_loss_gradients(pxb_context* ctx, const float* features, const float* targets, uint64_t n,
                                  float* loss, pxb_mlp_weights* grads) {
    if (!ctx || !features || !targets || !loss || !grads || n == 0) return PXB_ERR_INVALID_ARGUMENT;
    if (!ctx->has_mlp) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "no network installed");
    if (n > 0x7FFFFFFFull) return ctx->fail(PXB_ERR_TOO_LARGE, "too many rows");
    const size_t bx = sizeof(float) * kMlpIn * n, by = sizeof(float) * 3 * n, bi = sizeof(uint32_t) * n;
    const size_t bw = sizeof(pxb_mlp_weights), bp = sizeof(float) * mlp_partial_floats(ctx->n_sms);
    const size_t oy = al256(bx), oi = oy + al256(by), ow = oi + al256(bi), og = ow + al256(bw), ol = og + al256(bw),
                 op = ol + 256, total = op + al256(bp);
    DevBuf buf;
    if (pxb_status s = ctx->grow(buf, total, "gradient buffers")) return s;
    char* b = static_cast<char*>(buf.p);
    std::vector<uint32_t> order(n);
    for (uint64_t r = 0; r < n; ++r) order[r] = static_cast<uint32_t>(r);
    cudaStream_t st = ctx->stream;
    pxb_status s = PXB_OK;
    auto chk = [&](cudaError_t e, const char* what) {
        if (!s && e != cudaSuccess) s = ctx->cuda(e, what);
    };
    chk(cudaMemcpyAsync(b, features, bx, cudaMemcpyHostToDevice, st), "upload features");
    chk(cudaMemcpyAsync(b + oy, targets, by, cudaMemcpyHostToDevice, st), "upload targets");
    chk(cudaMemcpyAsync(b + oi, order.data(), bi, cudaMemcpyHostToDevice, st), "upload rows");
    chk(cudaMemcpyAsync(b + ow, &ctx->mlp, bw, cudaMemcpyHostToDevice, st), "upload weights");
    chk(cudaMemsetAsync(b + og, 0, bw, st), "zero gradients");
    chk(cudaMemsetAsync(b + ol, 0, sizeof(float), st), "zero loss");
    cudaError_t ge = cudaSuccess;
    auto* part = reinterpret_cast<float*>(b + op);
    const int parts = launch_mlp_grad(reinterpret_cast<float*>(b), reinterpret_cast<float*>(b + oy),
                                      reinterpret_cast<uint32_t*>(b + oi), static_cast<int>(n), static_cast<int>(n),
                                      reinterpret_cast<pxb_mlp_weights*>(b + ow), part, ctx->d_err, ctx->n_sms, st, &ge);
    chk(ge, "launch gradients");
    chk(launch_mlp_reduce(part, parts, ctx->n_sms, reinterpret_cast<pxb_mlp_weights*>(b + og),
                          reinterpret_cast<float*>(b + ol), st),
        "launch gradient sum");
    ctx->launches += 2;
    float lsum = 0.0f;
    chk(cudaMemcpyAsync(grads, b + og, bw, cudaMemcpyDeviceToHost, st), "read gradients");
    chk(cudaMemcpyAsync(&lsum, b + ol, sizeof(float), cudaMemcpyDeviceToHost, st), "read loss");
    chk(cudaStreamSynchronize(st), "gradients");
    cudaFree(buf.p);
    if (s) return s;
    if (pxb_status e = ctx->check_device_error()) return e;
    *loss = lsum / (3.0f * static_cast<float>(n));
    return PXB_OK;
}

pxb_status pxb_cloths_step_warm(pxb_context* ctx, const pxb_cloth_step_desc* step, const pxb_warm_start_desc* warm) {
    if (!ctx || !step || !warm) return PXB_ERR_INVALID_ARGUMENT;
    pxb_context::WarmCfg cfg;
    cfg.warm_iters = static_cast<int>(warm->warm_iterations);
    cfg.tau = warm->residual_threshold;
    cfg.taus = warm->thresholds;
    cfg.continue_iters = warm->continue_iterations ? 1 : 0;
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
        out[k].extra_iterations = static_cast<uint32_t>(e->warm_result.extra_iterations);
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
