// pxb_mlp.cuh -- the warm-start network on the tensor cores: 24 -> 64 -> SiLU -> 64 -> SiLU -> 3,
// BF16 weights and activations, FP32 accumulation in TMEM. One warpgroup (128 threads) runs a
// tile of 128 vertices; each thread owns one row (one vertex) from its features to its output.
//
// Model blob (device, built by the host from float weights):
//   [0, 4096)      W1 as a 64 x 32 K-major operand (inputs 24..31 zero)
//   [4096, 12288)  W2, 64 x 64
//   [12288, 14336) W3, 16 x 64 (outputs 3..15 zero)
//   then floats: b1[64] b2[64] b3[16] in_mean[32] in_scale[32] out_scale[4]
#ifndef PXB_MLP_CUH
#define PXB_MLP_CUH

#include "pxb_tcgen05.cuh"

namespace pxb {

constexpr int kMlpIn = 24, kMlpInPad = 32, kMlpHidden = 64, kMlpOut = 3, kMlpOutPad = 16;
constexpr int kMlpW1Bytes = kMlpHidden * kMlpInPad * 2;      // 4096
constexpr int kMlpW2Bytes = kMlpHidden * kMlpHidden * 2;     // 8192
constexpr int kMlpW3Bytes = kMlpOutPad * kMlpHidden * 2;     // 2048
constexpr int kMlpWBytes = kMlpW1Bytes + kMlpW2Bytes + kMlpW3Bytes;
constexpr int kMlpFloats = 64 + 64 + 16 + 32 + 32 + 4;       // 212
constexpr int kMlpBlobBytes = kMlpWBytes + kMlpFloats * 4;   // 15184
constexpr int kMlpTileA = 128 * kMlpInPad * 2;               // 8192: one tile of inputs
constexpr int kMlpTileH = 128 * kMlpHidden * 2;              // 16384: one tile of activations
constexpr int kMlpTmemCols = 64;
constexpr uint32_t kMlpWaitLimit = 1u << 22;

// Offsets of the float block inside the blob (in floats).
constexpr int kMlpB1 = 0, kMlpB2 = 64, kMlpB3 = 128, kMlpMean = 144, kMlpScale = 176, kMlpOutScale = 208;

struct MlpSmem {
    const unsigned char* w;  // kMlpWBytes, K-major operands
    const float* f;          // kMlpFloats
    unsigned char* a;        // this warpgroup's input tile
    unsigned char* h;        // this warpgroup's activation tile (may share the input tile's bytes)
    uint64_t* bar;           // this warpgroup's MMA-completion barrier
    uint32_t tmem;           // this warpgroup's 64 TMEM columns (lane 0)
};

__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// The network needs no IEEE rounding: fast exponential and division.
__device__ __forceinline__ float silu(float x) { return __fdividef(x, 1.0f + __expf(-x)); }

// Writes row r's normalised features (24 floats) into the input tile, bf16, padded with zeros.
__device__ __forceinline__ void mlp_put_input(const MlpSmem& S, int r, const float (&x)[kMlpIn]) {
    for (int c = 0; c < kMlpInPad / 8; ++c) {
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = 8 * c + j;
            const float xn = k < kMlpIn ? (x[k] - S.f[kMlpMean + k]) * S.f[kMlpScale + k] : 0.0f;
            v[j] = __float2bfloat16_rn(xn);
        }
        *reinterpret_cast<uint4*>(S.a + tc::kmajor_offset(r, 8 * c, kMlpInPad)) = *reinterpret_cast<uint4*>(v);
    }
}

// Layer epilogue: TMEM row (64 columns) + bias -> SiLU -> bf16 activation tile row.
__device__ __forceinline__ void mlp_hidden_epilogue(const MlpSmem& S, int r, uint32_t lane_addr, int bias) {
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
        float acc[16];
        tc::tmem_ld16(lane_addr + c0, acc);
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __float2bfloat16_rn(silu(acc[8 * half + j] + S.f[bias + c0 + 8 * half + j]));
            *reinterpret_cast<uint4*>(S.h + tc::kmajor_offset(r, c0 + 8 * half, kMlpHidden)) =
                *reinterpret_cast<uint4*>(v);
        }
    }
}

// Runs the network on the warpgroup's tile (inputs already in S.a). wt = thread index in the
// warpgroup (its row), warp_q = warp index mod 4 (its TMEM lane quarter), bar_id = named
// barrier of the warpgroup, phase = parity of the warpgroup's MMA barrier (advanced here).
// Returns false if an MMA never completed (the caller reports it and stops).
__device__ __forceinline__ bool mlp_tile(const MlpSmem& S, int wt, int warp_q, int bar_id, uint32_t& phase,
                                         float (&out)[kMlpOut]) {
    const uint32_t lane_addr = S.tmem + (static_cast<uint32_t>(warp_q * 32) << 16);
    const uint32_t a0 = tc::smem_u32(S.a), h0 = tc::smem_u32(S.h), w0 = tc::smem_u32(S.w);
    const uint32_t id64 = tc::idesc_bf16_f32(128, 64), id16 = tc::idesc_bf16_f32(128, 16);
    bool ok = true;

    // layer 1: [128 x 32] x W1^T -> 64
    tc::fence_async_smem();
    wg_sync(bar_id);
    if (wt == 0) {
        tc::fence_after_sync();
        for (int kk = 0; kk < kMlpInPad / 16; ++kk)
            tc::mma_bf16(S.tmem, tc::smem_desc(a0 + 256 * kk, 128, kMlpInPad / 8 * 128),
                         tc::smem_desc(w0 + 256 * kk, 128, kMlpInPad / 8 * 128), id64, kk > 0);
        tc::mma_commit(S.bar);
    }
    ok = __all_sync(0xffffffffu, tc::mbar_wait(S.bar, phase, kMlpWaitLimit));
    phase ^= 1u;
    tc::fence_after_sync();
    if (ok) mlp_hidden_epilogue(S, wt, lane_addr, kMlpB1);

    // layer 2: [128 x 64] x W2^T -> 64
    tc::fence_before_sync();
    tc::fence_async_smem();
    wg_sync(bar_id);
    if (wt == 0 && ok) {
        tc::fence_after_sync();
        for (int kk = 0; kk < kMlpHidden / 16; ++kk)
            tc::mma_bf16(S.tmem, tc::smem_desc(h0 + 256 * kk, 128, kMlpHidden / 8 * 128),
                         tc::smem_desc(w0 + kMlpW1Bytes + 256 * kk, 128, kMlpHidden / 8 * 128), id64, kk > 0);
        tc::mma_commit(S.bar);
    }
    if (ok) {
        ok = __all_sync(0xffffffffu, tc::mbar_wait(S.bar, phase, kMlpWaitLimit));
        phase ^= 1u;
    }
    tc::fence_after_sync();
    // Every thread's layer-2 MMA wait has returned before any thread overwrites the tile.
    wg_sync(bar_id);
    if (ok) mlp_hidden_epilogue(S, wt, lane_addr, kMlpB2);

    // layer 3: [128 x 64] x W3^T -> 16 (3 used)
    tc::fence_before_sync();
    tc::fence_async_smem();
    wg_sync(bar_id);
    if (wt == 0 && ok) {
        tc::fence_after_sync();
        for (int kk = 0; kk < kMlpHidden / 16; ++kk)
            tc::mma_bf16(S.tmem, tc::smem_desc(h0 + 256 * kk, 128, kMlpHidden / 8 * 128),
                         tc::smem_desc(w0 + kMlpW1Bytes + kMlpW2Bytes + 256 * kk, 128, kMlpHidden / 8 * 128),
                         id16, kk > 0);
        tc::mma_commit(S.bar);
    }
    if (ok) {
        ok = __all_sync(0xffffffffu, tc::mbar_wait(S.bar, phase, kMlpWaitLimit));
        phase ^= 1u;
    }
    tc::fence_after_sync();
    out[0] = out[1] = out[2] = 0.0f;
    if (ok) {
        float acc[16];
        tc::tmem_ld16(lane_addr, acc);
#pragma unroll
        for (int j = 0; j < kMlpOut; ++j) out[j] = (acc[j] + S.f[kMlpB3 + j]) * S.f[kMlpOutScale + j];
    }
    tc::fence_before_sync();
    return ok;
}

}  // namespace pxb

#endif  // PXB_MLP_CUH
