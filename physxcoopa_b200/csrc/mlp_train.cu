// mlp_train.cu -- fitting the warm-start network: mean squared error in normalised units, FP32
// gradients, Adam. Training is offline (once per scene family, before stepping), so it runs on
// the FP32 CUDA cores with the weights kept in FP32; the installed network is rounded to bf16
// for the tensor-core inference.
//
// Loss over a batch of B rows: L = 1 / (3B) * sum_r sum_j (y_rj - t_rj / out_scale_j)^2, with
// y = W3 h2 + b3, h2 = silu(W2 h1 + b2), h1 = silu(W1 xn + b1), xn = (x - in_mean) * in_scale.
#include <cuda_runtime.h>

#include <cstddef>

#include "pxb_kernels.h"

namespace pxb {

namespace {

constexpr int kRows = 128;          // rows per CTA, one per thread
constexpr int kXs = 25, kHs = 65;   // padded row strides (bank-conflict free)
// float block of the staged parameters: b1 64 | b2 64 | b3 3 (+1) | mean 24 | scale 24 | out_scale 3 (+1)
constexpr int kPb2 = 64, kPb3 = 128, kPmean = 132, kPscale = 156, kPout = 180, kPfloats = 184;

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Gradients over the rows idx[0 .. rows) accumulated into G (one atomic per weight per CTA),
// the summed squared error into *loss.
__global__ void __launch_bounds__(kRows) mlp_grad_kernel(const float* __restrict__ X, const float* __restrict__ T,
                                                          const uint32_t* __restrict__ idx, int rows,
                                                          const pxb_mlp_weights* __restrict__ W,
                                                          pxb_mlp_weights* __restrict__ G, float* __restrict__ loss) {
    extern __shared__ float sm[];
    float* sW1 = sm;                       // 64 x 24
    float* sW2 = sW1 + 64 * 24;            // 64 x 64
    float* sW3 = sW2 + 64 * 64;            // 3 x 64
    float* sB = sW3 + 3 * 64;              // kPfloats
    float* sx = sB + kPfloats;             // kRows x kXs normalised inputs
    float* sz1 = sx + kRows * kXs;         // kRows x kHs pre-activations, then their gradients
    float* sh1 = sz1 + kRows * kHs;
    float* sz2 = sh1 + kRows * kHs;
    float* sh2 = sz2 + kRows * kHs;
    __shared__ float s_dy[kRows][3];
    __shared__ float s_loss[kRows / 32];
    const int tid = threadIdx.x;
    for (int i = tid; i < 64 * 24; i += kRows) sW1[i] = (&W->w1[0][0])[i];
    for (int i = tid; i < 64 * 64; i += kRows) sW2[i] = (&W->w2[0][0])[i];
    for (int i = tid; i < 3 * 64; i += kRows) sW3[i] = (&W->w3[0][0])[i];
    if (tid < 64) {
        sB[tid] = W->b1[tid];
        sB[kPb2 + tid] = W->b2[tid];
    }
    if (tid < 3) {
        sB[kPb3 + tid] = W->b3[tid];
        sB[kPout + tid] = W->out_scale[tid];
    }
    if (tid < 24) {
        sB[kPmean + tid] = W->in_mean[tid];
        sB[kPscale + tid] = W->in_scale[tid];
    }
    const int r0 = blockIdx.x * kRows;
    const int r = r0 + tid;
    const bool live = r < rows;
    const uint32_t row = live ? idx[r] : 0u;
    __syncthreads();
    float* x = sx + tid * kXs;
    for (int k = 0; k < 24; ++k)
        x[k] = live ? (X[static_cast<size_t>(row) * 24 + k] - sB[kPmean + k]) * sB[kPscale + k] : 0.0f;
    // forward, one row per thread
    float* z1 = sz1 + tid * kHs;
    float* h1 = sh1 + tid * kHs;
    for (int j = 0; j < 64; ++j) {
        float a = sB[j];
        for (int k = 0; k < 24; ++k) a += sW1[j * 24 + k] * x[k];
        z1[j] = a;
        h1[j] = silu_f(a);
    }
    float* z2 = sz2 + tid * kHs;
    float* h2 = sh2 + tid * kHs;
    for (int j = 0; j < 64; ++j) {
        float a = sB[kPb2 + j];
        for (int k = 0; k < 64; ++k) a += sW2[j * 64 + k] * h1[k];
        z2[j] = a;
        h2[j] = silu_f(a);
    }
    float err2 = 0.0f;
    const float inv = 1.0f / (3.0f * static_cast<float>(rows));
    for (int o = 0; o < 3; ++o) {
        float y = sB[kPb3 + o];
        for (int k = 0; k < 64; ++k) y += sW3[o * 64 + k] * h2[k];
        const float t = live ? T[static_cast<size_t>(row) * 3 + o] / sB[kPout + o] : 0.0f;
        const float e = live ? y - t : 0.0f;
        err2 += e * e;
        s_dy[tid][o] = 2.0f * e * inv;
    }
    // backward through the row: dz2 (into z2), then dz1 (into z1)
    for (int k = 0; k < 64; ++k) {
        float g = 0.0f;
        for (int o = 0; o < 3; ++o) g += sW3[o * 64 + k] * s_dy[tid][o];
        z2[k] = g * silu_grad(z2[k]);
    }
    for (int k = 0; k < 64; ++k) {
        float g = 0.0f;
        for (int j = 0; j < 64; ++j) g += sW2[j * 64 + k] * z2[j];
        z1[k] = g * silu_grad(z1[k]);
    }
    for (int o = 16; o > 0; o >>= 1) err2 += __shfl_xor_sync(0xffffffffu, err2, o);
    if ((tid & 31) == 0) s_loss[tid >> 5] = err2;
    __syncthreads();
    if (tid == 0) atomicAdd(loss, s_loss[0] + s_loss[1] + s_loss[2] + s_loss[3]);
    // weight gradients: sums over this CTA's rows
    const int nr = rows - r0 < kRows ? rows - r0 : kRows;
    for (int e = tid; e < 64 * 64; e += kRows) {
        const int j = e >> 6, k = e & 63;
        float g = 0.0f;
        for (int q = 0; q < nr; ++q) g += sz2[q * kHs + j] * sh1[q * kHs + k];
        atomicAdd(&G->w2[j][k], g);
    }
    for (int e = tid; e < 64 * 24; e += kRows) {
        const int j = e / 24, k = e - j * 24;
        float g = 0.0f;
        for (int q = 0; q < nr; ++q) g += sz1[q * kHs + j] * sx[q * kXs + k];
        atomicAdd(&G->w1[j][k], g);
    }
    for (int e = tid; e < 3 * 64; e += kRows) {
        const int o = e >> 6, k = e & 63;
        float g = 0.0f;
        for (int q = 0; q < nr; ++q) g += s_dy[q][o] * sh2[q * kHs + k];
        atomicAdd(&G->w3[o][k], g);
    }
    if (tid < 64) {
        float g1 = 0.0f, g2 = 0.0f;
        for (int q = 0; q < nr; ++q) {
            g1 += sz1[q * kHs + tid];
            g2 += sz2[q * kHs + tid];
        }
        atomicAdd(&G->b1[tid], g1);
        atomicAdd(&G->b2[tid], g2);
    }
    if (tid < 3) {
        float g = 0.0f;
        for (int q = 0; q < nr; ++q) g += s_dy[q][tid];
        atomicAdd(&G->b3[tid], g);
    }
}

// Adam over the weight and bias fields (the normalisation fields are not trained).
__global__ void mlp_adam_kernel(pxb_mlp_weights* W, const pxb_mlp_weights* G, pxb_mlp_weights* M,
                                pxb_mlp_weights* V, float lr, float b1t, float b2t) {
    constexpr int n = static_cast<int>(offsetof(pxb_mlp_weights, in_mean) / sizeof(float));
    float* w = reinterpret_cast<float*>(W);
    const float* g = reinterpret_cast<const float*>(G);
    float* m = reinterpret_cast<float*>(M);
    float* v = reinterpret_cast<float*>(V);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        m[i] = 0.9f * m[i] + 0.1f * gi;
        v[i] = 0.999f * v[i] + 0.001f * gi * gi;
        const float mh = m[i] / (1.0f - b1t), vh = v[i] / (1.0f - b2t);
        w[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
    }
}

}  // namespace

int mlp_grad_smem_bytes() {
    return 4 * (64 * 24 + 64 * 64 + 3 * 64 + kPfloats + kRows * kXs + 4 * kRows * kHs);
}

cudaError_t launch_mlp_grad(const float* X, const float* T, const uint32_t* idx, int rows, const pxb_mlp_weights* W,
                            pxb_mlp_weights* G, float* loss, cudaStream_t stream) {
    if (rows <= 0) return cudaSuccess;
    static bool configured = false;
    const int smem = mlp_grad_smem_bytes();
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    mlp_grad_kernel<<<(rows + kRows - 1) / kRows, kRows, smem, stream>>>(X, T, idx, rows, W, G, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(pxb_mlp_weights* W, const pxb_mlp_weights* G, pxb_mlp_weights* M, pxb_mlp_weights* V,
                            float lr, float b1t, float b2t, cudaStream_t stream) {
    mlp_adam_kernel<<<8, 256, 0, stream>>>(W, G, M, V, lr, b1t, b2t);
    return cudaGetLastError();
}

}  // namespace pxb
