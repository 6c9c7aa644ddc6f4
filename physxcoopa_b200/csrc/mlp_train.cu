// mlp_train.cu -- fitting the warm-start network on the tensor cores: mean squared error in
// normalised units, forward and backward passes as BF16 tcgen05 MMAs accumulating in FP32 (TMEM),
// Adam on FP32 master weights.
//
// Loss over a batch of B rows: L = 1 / (3B) * sum_r sum_j (y_rj - t_rj / out_scale_j)^2, with
// y = W3 h2 + b3, h2 = silu(z2), z2 = W2 h1 + b2, h1 = silu(z1), z1 = W1 xn + b1,
// xn = (x - in_mean) * in_scale.
//
// One CTA is one warpgroup (128 threads); it takes 128-row tiles of the batch in turn, thread r
// owning row r of the tile. Per tile, each GEMM is one group of MMAs issued by thread 0:
//   forward   Z1 = Xn W1^T, Z2 = H1 W2^T, Y = H2 W3^T          (M = 128 rows, K = features)
//   backward  dH2 = dY W3, dH1 = dZ2 W2                        (B operands: W3^T, W2^T)
//   weights   [dZ2^T; dZ1^T] [H1^T; Xn^T; 1]^T   -> dW2, db2 (rows 0..63), dW1, db1 (rows 64..127)
//             [dY^T; ...]    [H2^T; 1]^T         -> dW3, db3 (rows 0..2)
// The weight-gradient MMAs take the batch as their K dimension and stack two gradients into one
// M = 128 operand; their accumulators stay in TMEM across all of the CTA's tiles, so a CTA
// writes its partial gradients once. Bias gradients come from the ones row of the B operand.
// Partials are summed in a fixed order by the Adam (or reduce) kernel: training is
// deterministic for a given batch order.
//
// Precision: inputs, activations and back-propagated errors are rounded to bf16 as MMA operands;
// every product is accumulated in FP32; the pre-activations z1, z2 stay in FP32 in TMEM for the
// SiLU derivatives; Adam keeps FP32 master weights, re-rounded to bf16 operands at the start of
// every gradient launch.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

#include "pxb_kernels.h"
#include "pxb_mlp.cuh"

namespace pxb {

namespace {

constexpr int kRows = 128;
// trained parameters: the pxb_mlp_weights fields before in_mean, in declaration order
constexpr int kTrain = static_cast<int>(offsetof(pxb_mlp_weights, in_mean) / sizeof(float));  // 5955
constexpr int kPartStride = 6016;  // floats per CTA partial (kTrain rounded up to 64)
constexpr int kOffB1 = static_cast<int>(offsetof(pxb_mlp_weights, b1) / sizeof(float));
constexpr int kOffW2 = static_cast<int>(offsetof(pxb_mlp_weights, w2) / sizeof(float));
constexpr int kOffB2 = static_cast<int>(offsetof(pxb_mlp_weights, b2) / sizeof(float));
constexpr int kOffW3 = static_cast<int>(offsetof(pxb_mlp_weights, w3) / sizeof(float));
constexpr int kOffB3 = static_cast<int>(offsetof(pxb_mlp_weights, b3) / sizeof(float));
static_assert(kTrain == 64 * 24 + 64 + 64 * 64 + 64 + 3 * 64 + 3, "trained parameter count");
static_assert(kTrain <= kPartStride, "partial stride");

// Shared memory (bytes). All operands are K-major, no swizzle (pxb_tcgen05.cuh).
constexpr int kSW1 = 0;                    // W1    64 x 32
constexpr int kSW2 = kSW1 + 64 * 32 * 2;   // W2    64 x 64
constexpr int kSW3 = kSW2 + 64 * 64 * 2;   // W3    16 x 64 (rows 3..15 zero)
constexpr int kSW2T = kSW3 + 16 * 64 * 2;  // W2^T  64 x 64
constexpr int kSW3T = kSW2T + 64 * 64 * 2; // W3^T  64 x 16 (columns 3..15 zero)
constexpr int kSF = kSW3T + 64 * 16 * 2;   // floats: b1 64 | b2 64 | b3 4 | mean 32 | scale 32 | out_scale 4
constexpr int kSAX = kSF + 256 * 4;        // Xn    128 x 32; later dY 128 x 16
constexpr int kSH1 = kSAX + 128 * 32 * 2;  // H1    128 x 64; later dZ2
constexpr int kSH2 = kSH1 + 128 * 64 * 2;  // H2    128 x 64
constexpr int kSAG = kSH2 + 128 * 64 * 2;  // [dY^T (16 rows); dZ2^T (64); dZ1^T (64)]  144 x 128
constexpr int kSBG1 = kSAG + 144 * 128 * 2;  // [H1^T (64); Xn^T (32); ones (16)]        112 x 128
constexpr int kSBG2 = kSBG1 + 112 * 128 * 2; // [H2^T (64); ones (16)]                    80 x 128
constexpr int kSmemBytes = kSBG2 + 80 * 128 * 2;  // 152576
constexpr int kFb1 = 0, kFb2 = 64, kFb3 = 128, kFmean = 132, kFscale = 164, kFout = 196;

// TMEM columns (lane = row of the tile)
constexpr uint32_t kTZ1 = 0, kTZ2 = 64, kTS = 128, kTG1 = 256, kTG2 = 384, kTCols = 512;

__device__ __forceinline__ float sig(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sig(z);
    return s * (1.0f + z * (1.0f - s));
}

// Row r of an R x K K-major operand, columns c0 .. c0 + 15, from FP32 values.
__device__ __forceinline__ void put_row16(unsigned char* base, int r, int K, int c0, const float (&v)[16]) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        __align__(16) __nv_bfloat162 p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = __floats2bfloat162_rn(v[8 * half + 2 * j], v[8 * half + 2 * j + 1]);
        *reinterpret_cast<uint4*>(base + tc::kmajor_offset(r, c0 + 8 * half, K)) = *reinterpret_cast<uint4*>(p);
    }
}

// Column r (a sample) of the transposed operand rows f0 .. f0 + F - 1 (features) of an R x 128
// K-major operand. Lanes r and r ^ 1 swap halves so that each stores one 4-byte word holding
// samples (r & ~1, r | 1) of one feature: the even lane feature f, the odd lane feature f + 1.
template <int F>
__device__ __forceinline__ void put_col(unsigned char* base, int r, int f0, const float* v) {
    const bool odd = (r & 1) != 0;
#pragma unroll
    for (int f = 0; f < F; f += 2) {
        const float a = v[f], b = v[f + 1];
        const float got = __shfl_xor_sync(0xffffffffu, odd ? a : b, 1);
        const __nv_bfloat162 w = odd ? __floats2bfloat162_rn(got, b) : __floats2bfloat162_rn(a, got);
        const int feat = f0 + f + (odd ? 1 : 0);
        *reinterpret_cast<__nv_bfloat162*>(base + tc::kmajor_offset(feat, r & ~1, 128)) = w;
    }
}

// K = 16 slices of an MMA group: D (+)= A B^T with A, B K-major of K columns.
__device__ __forceinline__ void mma_group(uint32_t d, uint32_t a, uint32_t b, int K, uint32_t idesc, bool acc0) {
    const uint32_t sbo = static_cast<uint32_t>(K / 8 * 128);
    for (int kk = 0; kk < K / 16; ++kk)
        tc::mma_bf16(d, tc::smem_desc(a + 256 * kk, 128, sbo), tc::smem_desc(b + 256 * kk, 128, sbo), idesc,
                     acc0 || kk > 0);
}

// The FP32 master weights rounded to the CTA's bf16 operands, and the float block.
__device__ void load_weights(unsigned char* sm, const pxb_mlp_weights* __restrict__ W, int tid) {
    float* F = reinterpret_cast<float*>(sm + kSF);
    auto bf = [](float v) { return __float2bfloat16_rn(v); };
    for (int e = tid; e < 64 * 32; e += kRows) {  // W1 (inputs 24..31 zero)
        const int o = e >> 5, i = e & 31;
        *reinterpret_cast<__nv_bfloat16*>(sm + kSW1 + tc::kmajor_offset(o, i, 32)) = bf(i < 24 ? W->w1[o][i] : 0.0f);
    }
    for (int e = tid; e < 64 * 64; e += kRows) {  // W2 and its transpose
        const int o = e >> 6, i = e & 63;
        const __nv_bfloat16 v = bf(W->w2[o][i]);
        *reinterpret_cast<__nv_bfloat16*>(sm + kSW2 + tc::kmajor_offset(o, i, 64)) = v;
        *reinterpret_cast<__nv_bfloat16*>(sm + kSW2T + tc::kmajor_offset(i, o, 64)) = v;
    }
    for (int e = tid; e < 16 * 64; e += kRows) {  // W3 (outputs 3..15 zero) and its transpose
        const int o = e >> 6, i = e & 63;
        const __nv_bfloat16 v = bf(o < 3 ? W->w3[o][i] : 0.0f);
        *reinterpret_cast<__nv_bfloat16*>(sm + kSW3 + tc::kmajor_offset(o, i, 64)) = v;
        *reinterpret_cast<__nv_bfloat16*>(sm + kSW3T + tc::kmajor_offset(i, o, 16)) = v;
    }
    if (tid < 64) {
        F[kFb1 + tid] = W->b1[tid];
        F[kFb2 + tid] = W->b2[tid];
    }
    if (tid < 32) {
        F[kFmean + tid] = tid < 24 ? W->in_mean[tid] : 0.0f;
        F[kFscale + tid] = tid < 24 ? W->in_scale[tid] : 0.0f;
    }
    if (tid < 4) {
        F[kFb3 + tid] = tid < 3 ? W->b3[tid] : 0.0f;
        F[kFout + tid] = tid < 3 ? W->out_scale[tid] : 1.0f;
    }
}

// Loss and gradient partials of rows idx[0 .. rows) for this CTA's tiles (tile = blockIdx.x,
// blockIdx.x + gridDim.x, ...). inv = 1 / (3 B) with B the rows of the whole optimiser batch.
// part: gridDim.x x kPartStride floats, part_loss: gridDim.x floats (summed squared errors).
__global__ void __launch_bounds__(kRows, 1) mlp_grad_tc_kernel(const float* __restrict__ X, const float* __restrict__ T,
                                                               const uint32_t* __restrict__ idx, int rows, float inv,
                                                               const pxb_mlp_weights* __restrict__ W,
                                                               float* __restrict__ part, float* __restrict__ part_loss,
                                                               uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    __shared__ float s_loss[kRows / 32];
    const int tid = threadIdx.x, warp = tid >> 5;
    const float* F = reinterpret_cast<const float*>(sm + kSF);

    // zero every operand (padding rows and columns must hold finite values), then the weights
    for (int i = tid; i < kSmemBytes / 16; i += kRows) reinterpret_cast<uint4*>(sm)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    load_weights(sm, W, tid);
    {   // the ones rows of the weight-gradient B operands (bias gradients)
        const __nv_bfloat16 one = __float2bfloat16_rn(1.0f);
        *reinterpret_cast<__nv_bfloat16*>(sm + kSBG1 + tc::kmajor_offset(96, tid, 128)) = one;
        *reinterpret_cast<__nv_bfloat16*>(sm + kSBG2 + tc::kmajor_offset(64, tid, 128)) = one;
    }
    if (warp == 0) tc::tmem_alloc(&tslot, kTCols);
    if (tid == 0) tc::mbar_init(&bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tslot;
    const uint32_t lane = tm + (static_cast<uint32_t>(warp * 32) << 16);
    const uint32_t s0 = tc::smem_u32(sm);
    uint32_t phase = 0;
    bool ok = true;
    float err2 = 0.0f;
    const int tiles = (rows + kRows - 1) / kRows;

    // one MMA group by thread 0, then every thread waits for its completion
    auto issue_and_wait = [&](auto&& body) {
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc::fence_after_sync();
            body();
            tc::mma_commit(&bar);
        }
        bool done = ok ? tc::mbar_wait(&bar, phase, kMlpWaitLimit) : false;
        ok = __syncthreads_and(ok && done) != 0;
        phase ^= 1u;
        tc::fence_after_sync();
    };

    bool first = true;
    for (int tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const int r = tile * kRows + tid;
        const bool live = r < rows;
        const size_t row = live ? idx[r] : 0u;
        float x[32], t[3];
#pragma unroll
        for (int k = 0; k < 32; ++k)
            x[k] = (live && k < 24) ? (X[row * 24 + k] - F[kFmean + k]) * F[kFscale + k] : 0.0f;
#pragma unroll
        for (int j = 0; j < 3; ++j) t[j] = live ? T[row * 3 + j] / F[kFout + j] : 0.0f;
        {
            float v[16];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int k = 0; k < 16; ++k) v[k] = x[16 * h + k];
                put_row16(sm + kSAX, tid, 32, 16 * h, v);
            }
            put_col<24>(sm + kSBG1, tid, 64, x);
        }
        // Z1 = Xn W1^T
        issue_and_wait([&] { mma_group(tm + kTZ1, s0 + kSAX, s0 + kSW1, 32, tc::idesc_bf16_f32(128, 64), false); });
        if (!ok) break;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc::tmem_ld16(lane + kTZ1 + c0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float z = v[j] + F[kFb1 + c0 + j];
                v[j] = z * sig(z);
            }
            put_row16(sm + kSH1, tid, 64, c0, v);
            put_col<16>(sm + kSBG1, tid, c0, v);
        }
        // Z2 = H1 W2^T
        issue_and_wait([&] { mma_group(tm + kTZ2, s0 + kSH1, s0 + kSW2, 64, tc::idesc_bf16_f32(128, 64), false); });
        if (!ok) break;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc::tmem_ld16(lane + kTZ2 + c0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float z = v[j] + F[kFb2 + c0 + j];
                v[j] = z * sig(z);
            }
            put_row16(sm + kSH2, tid, 64, c0, v);
            put_col<16>(sm + kSBG2, tid, c0, v);
        }
        // Y = H2 W3^T (16 columns, 3 used)
        issue_and_wait([&] { mma_group(tm + kTS, s0 + kSH2, s0 + kSW3, 64, tc::idesc_bf16_f32(128, 16), false); });
        if (!ok) break;
        {
            float v[16];
            tc::tmem_ld16(lane + kTS, v);
            float dy[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) dy[j] = 0.0f;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float e = live ? v[j] + F[kFb3 + j] - t[j] : 0.0f;
                err2 += e * e;
                dy[j] = 2.0f * e * inv;
            }
            put_row16(sm + kSAX, tid, 16, 0, dy);  // dY, 128 x 16
            put_col<4>(sm + kSAG, tid, 0, dy);     // dY^T rows 0..3
        }
        // dH2 = dY W3 (B operand W3^T)
        issue_and_wait([&] { mma_group(tm + kTS, s0 + kSAX, s0 + kSW3T, 16, tc::idesc_bf16_f32(128, 64), false); });
        if (!ok) break;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float g[16], z[16];
            tc::tmem_ld16(lane + kTS + c0, g);
            tc::tmem_ld16(lane + kTZ2 + c0, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) g[j] *= dsilu(z[j] + F[kFb2 + c0 + j]);
            put_row16(sm + kSH1, tid, 64, c0, g);      // dZ2 (H1 is no longer read)
            put_col<16>(sm + kSAG, tid, 16 + c0, g);   // dZ2^T rows 16..79
        }
        // dH1 = dZ2 W2 (B operand W2^T)
        issue_and_wait([&] { mma_group(tm + kTS, s0 + kSH1, s0 + kSW2T, 64, tc::idesc_bf16_f32(128, 64), false); });
        if (!ok) break;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float g[16], z[16];
            tc::tmem_ld16(lane + kTS + c0, g);
            tc::tmem_ld16(lane + kTZ1 + c0, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) g[j] *= dsilu(z[j] + F[kFb1 + c0 + j]);
            put_col<16>(sm + kSAG, tid, 80 + c0, g);   // dZ1^T rows 80..143
        }
        // weight gradients, accumulated over the CTA's tiles
        const bool acc = !first;
        issue_and_wait([&] {
            mma_group(tm + kTG1, s0 + kSAG + 2 * 2048, s0 + kSBG1, 128, tc::idesc_bf16_f32(128, 112), acc);
            mma_group(tm + kTG2, s0 + kSAG, s0 + kSBG2, 128, tc::idesc_bf16_f32(128, 80), acc);
        });
        first = false;
    }

    // partials: this CTA's accumulated gradients and squared errors
    for (int o = 16; o > 0; o >>= 1) err2 += __shfl_xor_sync(0xffffffffu, err2, o);
    if ((tid & 31) == 0) s_loss[warp] = err2;
    __syncthreads();
    float* P = part + static_cast<size_t>(blockIdx.x) * kPartStride;
    if (tid == 0) part_loss[blockIdx.x] = s_loss[0] + s_loss[1] + s_loss[2] + s_loss[3];
    if (ok && !first) {
        float v[16];
        if (warp < 2) {  // rows 0..63 of the first group: dW2 (columns 0..63), db2 (column 96)
            const int j = tid;
            for (int c0 = 0; c0 < 64; c0 += 16) {
                tc::tmem_ld16(lane + kTG1 + c0, v);
#pragma unroll
                for (int k = 0; k < 16; ++k) P[kOffW2 + j * 64 + c0 + k] = v[k];
            }
            tc::tmem_ld16(lane + kTG1 + 96, v);
            P[kOffB2 + j] = v[0];
        } else {         // rows 64..127: dW1 (columns 64..87), db1 (column 96)
            const int j = tid - 64;
            tc::tmem_ld16(lane + kTG1 + 64, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) P[j * 24 + k] = v[k];
            tc::tmem_ld16(lane + kTG1 + 80, v);
#pragma unroll
            for (int k = 0; k < 8; ++k) P[j * 24 + 16 + k] = v[k];
            tc::tmem_ld16(lane + kTG1 + 96, v);
            P[kOffB1 + j] = v[0];
        }
        if (warp == 0) { // rows 0..2 of the second group: dW3 (columns 0..63), db3 (column 64)
            for (int c0 = 0; c0 < 64; c0 += 16) {
                tc::tmem_ld16(lane + kTG2 + c0, v);
                if (tid < 3)
#pragma unroll
                    for (int k = 0; k < 16; ++k) P[kOffW3 + tid * 64 + c0 + k] = v[k];
            }
            tc::tmem_ld16(lane + kTG2 + 64, v);
            if (tid < 3) P[kOffB3 + tid] = v[0];
        }
    } else {
        for (int i = tid; i < kTrain; i += kRows) P[i] = 0.0f;
    }
    if (!ok && tid == 0) atomicOr(err, PXB_DEVERR_MMA_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tm, kTCols);
}

// Sum of parameter i's partials over the gradient launch's CTAs, in CTA order.
__device__ __forceinline__ float sum_partials(const float* __restrict__ part, int n_parts, int i) {
    float g = 0.0f;
    for (int c = 0; c < n_parts; ++c) g += part[static_cast<size_t>(c) * kPartStride + i];
    return g;
}

__device__ __forceinline__ void add_loss(const float* __restrict__ part_loss, int n_parts, float* loss) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float l = 0.0f;
        for (int c = 0; c < n_parts; ++c) l += part_loss[c];
        *loss += l;
    }
}

// Adam over the trained fields (the normalisation fields are not trained), FP32 master weights.
__global__ void mlp_adam_kernel(const float* __restrict__ part, const float* __restrict__ part_loss, int n_parts,
                                pxb_mlp_weights* W, pxb_mlp_weights* M, pxb_mlp_weights* V, float lr, float b1t,
                                float b2t, float* loss) {
    float* w = reinterpret_cast<float*>(W);
    float* m = reinterpret_cast<float*>(M);
    float* v = reinterpret_cast<float*>(V);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    add_loss(part_loss, n_parts, loss);
    if (i >= kTrain) return;
    const float gi = sum_partials(part, n_parts, i);
    m[i] = 0.9f * m[i] + 0.1f * gi;
    v[i] = 0.999f * v[i] + 0.001f * gi * gi;
    const float mh = m[i] / (1.0f - b1t), vh = v[i] / (1.0f - b2t);
    w[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// The summed gradients into G (trained fields) and the summed squared errors into *loss.
__global__ void mlp_reduce_kernel(const float* __restrict__ part, const float* __restrict__ part_loss, int n_parts,
                                  pxb_mlp_weights* G, float* loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    add_loss(part_loss, n_parts, loss);
    if (i < kTrain) reinterpret_cast<float*>(G)[i] = sum_partials(part, n_parts, i);
}

}  // namespace

size_t mlp_partial_floats(int n_sms) { return static_cast<size_t>(n_sms) * kPartStride + n_sms; }

int launch_mlp_grad(const float* X, const float* T, const uint32_t* idx, int rows, int batch_rows,
                    const pxb_mlp_weights* W, float* part, uint32_t* err, int n_sms, cudaStream_t stream,
                    cudaError_t* status) {
    *status = cudaSuccess;
    if (rows <= 0) return 0;
    static bool configured = false;
    if (!configured) {
        *status = cudaFuncSetAttribute(mlp_grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (*status != cudaSuccess) return 0;
        configured = true;
    }
    const int tiles = (rows + kRows - 1) / kRows;
    // one CTA per SM at most: each holds 512 TMEM columns and ~150 KB of shared memory
    const int grid = tiles < n_sms ? tiles : n_sms;
    const float inv = 1.0f / (3.0f * static_cast<float>(batch_rows));
    mlp_grad_tc_kernel<<<grid, kRows, kSmemBytes, stream>>>(X, T, idx, rows, inv, W, part,
                                                             part + static_cast<size_t>(n_sms) * kPartStride, err);
    *status = cudaGetLastError();
    return grid;
}

cudaError_t launch_mlp_adam(const float* part, int n_parts, int n_sms, pxb_mlp_weights* W, pxb_mlp_weights* M,
                            pxb_mlp_weights* V, float lr, float b1t, float b2t, float* loss, cudaStream_t stream) {
    mlp_adam_kernel<<<(kTrain + 255) / 256, 256, 0, stream>>>(part, part + static_cast<size_t>(n_sms) * kPartStride,
                                                               n_parts, W, M, V, lr, b1t, b2t, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_reduce(const float* part, int n_parts, int n_sms, pxb_mlp_weights* G, float* loss,
                              cudaStream_t stream) {
    mlp_reduce_kernel<<<(kTrain + 255) / 256, 256, 0, stream>>>(part, part + static_cast<size_t>(n_sms) * kPartStride,
                                                                 n_parts, G, loss);
    return cudaGetLastError();
}

}  // namespace pxb
