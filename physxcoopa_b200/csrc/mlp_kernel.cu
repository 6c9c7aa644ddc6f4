// mlp_kernel.cu -- the warm-start network over a batch of feature rows (tensor cores), and the
// host packing of its weights into the device blob.
//
// The cloth solver runs the same network inside its own kernel (pxb_mlp.cuh); this standalone
// form serves pxb_mlp_infer, the reference-free check of the tensor-core path, and training.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "pxb_kernels.h"
#include "pxb_mlp.cuh"

namespace pxb {

namespace {

// One warpgroup per CTA; persistent over 128-row tiles.
__global__ void __launch_bounds__(128) mlp_infer_kernel(const float* __restrict__ X, int n,
                                                        const unsigned char* __restrict__ blob,
                                                        float* __restrict__ Y, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpBlobBytes / 16; i += 128)
        reinterpret_cast<uint4*>(sm)[i] = reinterpret_cast<const uint4*>(blob)[i];
    if (tid < 32) tc::tmem_alloc(&tslot, kMlpTmemCols);
    if (tid == 0) tc::mbar_init(&bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    MlpSmem S;
    S.w = sm;
    S.f = reinterpret_cast<const float*>(sm + kMlpWBytes);
    S.a = sm + ((kMlpBlobBytes + 127) & ~127);
    S.h = S.a;  // the first layer consumes the inputs before the activations are written
    S.bar = &bar;
    S.tmem = tslot;
    uint32_t phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; ok && tile * 128 < n; tile += gridDim.x) {
        const int row = tile * 128 + tid;
        float x[kMlpIn];
        for (int k = 0; k < kMlpIn; ++k) x[k] = row < n ? X[static_cast<size_t>(row) * kMlpIn + k] : 0.0f;
        mlp_put_input(S, tid, x);
        float y[kMlpOut];
        ok = mlp_tile(S, tid, tid >> 5, 1, phase, y);
        // every thread learns whether any MMA wait expired before the next tile
        ok = __syncthreads_and(ok) != 0;
        if (ok && row < n)
            for (int j = 0; j < kMlpOut; ++j) Y[static_cast<size_t>(row) * kMlpOut + j] = y[j];
    }
    if (!ok && tid == 0) atomicOr(err, PXB_DEVERR_MMA_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(S.tmem, kMlpTmemCols);
}

}  // namespace

int mlp_infer_smem_bytes() { return ((kMlpBlobBytes + 127) & ~127) + kMlpTileH; }

cudaError_t launch_mlp_infer(const float* X, int n, const unsigned char* blob, float* Y, uint32_t* err,
                             int n_sms, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    static bool configured = false;
    const int smem = mlp_infer_smem_bytes();
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int tiles = (n + 127) / 128;
    // At most 8 CTAs per SM share its 512 TMEM columns (64 each), so allocation never waits.
    const int grid = tiles < 4 * n_sms ? tiles : 4 * n_sms;
    mlp_infer_kernel<<<grid, 128, smem, stream>>>(X, n, blob, Y, err);
    return cudaGetLastError();
}

// Float weights (row-major, out x in) -> the device blob: bf16 K-major operands + float block.
void mlp_pack_blob(const pxb_mlp_weights& m, unsigned char* out) {
    std::memset(out, 0, kMlpBlobBytes);
    auto put = [&](unsigned char* base, int r, int k, int K, float v) {
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        std::memcpy(base + tc::kmajor_offset(r, k, K), &b, 2);
    };
    for (int o = 0; o < kMlpHidden; ++o)
        for (int i = 0; i < kMlpIn; ++i) put(out, o, i, kMlpInPad, m.w1[o][i]);
    for (int o = 0; o < kMlpHidden; ++o)
        for (int i = 0; i < kMlpHidden; ++i) put(out + kMlpW1Bytes, o, i, kMlpHidden, m.w2[o][i]);
    for (int o = 0; o < kMlpOut; ++o)
        for (int i = 0; i < kMlpHidden; ++i) put(out + kMlpW1Bytes + kMlpW2Bytes, o, i, kMlpHidden, m.w3[o][i]);
    float f[kMlpFloats] = {};
    for (int i = 0; i < kMlpHidden; ++i) {
        f[kMlpB1 + i] = m.b1[i];
        f[kMlpB2 + i] = m.b2[i];
    }
    for (int i = 0; i < kMlpOut; ++i) {
        f[kMlpB3 + i] = m.b3[i];
        f[kMlpOutScale + i] = m.out_scale[i];
    }
    for (int i = 0; i < kMlpIn; ++i) {
        f[kMlpMean + i] = m.in_mean[i];
        f[kMlpScale + i] = m.in_scale[i];
    }
    std::memcpy(out + kMlpWBytes, f, sizeof(f));
}

}  // namespace pxb
