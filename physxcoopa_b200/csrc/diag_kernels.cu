// diag_kernels.cu -- measurement kernels behind pxb_measure_smem_bandwidth.
//
// The cloth kernel is bound by shared-memory bandwidth, a figure no vendor table states for
// this part under its power cap. This kernel measures it the way STREAM measures HBM: every
// CTA (one per SM, 1024 threads) copies a float4 array between two shared-memory buffers,
// conflict-free, many times over; bytes read + written / elapsed is the achievable figure.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/physxcoopa_b200.h"
#include "runtime_internal.h"

namespace {

constexpr int kSmemFloat4 = 6144;  // 96 KB per buffer, two buffers

__global__ void __launch_bounds__(1024, 1) smem_copy_kernel(int rounds, float* sink) {
    extern __shared__ __align__(16) float4 buf[];
    float4* a = buf;
    float4* b = buf + kSmemFloat4;
    for (int i = threadIdx.x; i < kSmemFloat4; i += blockDim.x) {
        a[i] = make_float4(i, i + 1, i + 2, i + 3);
        b[i] = a[i];
    }
    __syncthreads();
    for (int r = 0; r < rounds; ++r) {
#pragma unroll 6
        for (int i = threadIdx.x; i < kSmemFloat4; i += blockDim.x) {
            float4 v = a[i];
            v.x += 1.0f;
            b[i] = v;
        }
        __syncthreads();
        float4* t = a;
        a = b;
        b = t;
    }
    if (threadIdx.x == 0) sink[blockIdx.x] = a[blockIdx.x % kSmemFloat4].x;
}

}  // namespace

extern "C" pxb_status pxb_measure_smem_bandwidth(pxb_context* ctx, double* bytes_per_second) {
    if (!ctx || !bytes_per_second) return PXB_ERR_INVALID_ARGUMENT;
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e != cudaSuccess) return ctx->cuda(e, "device attribute");
    const int smem = 2 * kSmemFloat4 * 16;
    e = cudaFuncSetAttribute(smem_copy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return ctx->cuda(e, "smem attribute");
    if (pxb_status s = ctx->grow(ctx->d_scratch, 4 * static_cast<size_t>(sms), "smem probe")) return s;
    float* sink = static_cast<float*>(ctx->d_scratch.p);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const int rounds = 4000;
    smem_copy_kernel<<<sms, 1024, smem, ctx->stream>>>(50, sink);  // warm-up
    cudaEventRecord(t0, ctx->stream);
    smem_copy_kernel<<<sms, 1024, smem, ctx->stream>>>(rounds, sink);
    cudaEventRecord(t1, ctx->stream);
    e = cudaEventSynchronize(t1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return ctx->cuda(e, "smem probe");
    ctx->launches += 2;
    const double bytes = static_cast<double>(sms) * rounds * kSmemFloat4 * 32.0;
    *bytes_per_second = bytes / (ms * 1e-3);
    return PXB_OK;
}
