// diag_kernels.cu -- measurement and self-check kernels: pxb_measure_smem_bandwidth and
// pxb_check_quotients.
//
// The cloth kernel is bound by shared-memory bandwidth, a figure no vendor table states for
// this part under its power cap. This kernel measures it the way STREAM measures HBM: every
// CTA (one per SM, 1024 threads) copies a float4 array between two shared-memory buffers,
// conflict-free, many times over; bytes read + written / elapsed is the achievable figure.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/physxcoopa_b200.h"
#include "pxb_device_math.cuh"
#include "pxb_quotient.cuh"
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

// ------------------------------------------------------------------------------------------
// pxb_check_quotients: the solver's quotients against IEEE division on this device
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// counts[0]: significands m (and three exponents) where the refined reciprocal of the scaled
// divisor differs from the correctly rounded reciprocal.
__global__ void check_reciprocal_kernel(unsigned long long* counts) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= (1u << 23)) return;
    uint32_t bad = 0;
    const uint32_t exps[3] = {131u, 191u, 250u};  // 2^4, 2^64, 2^123: the scaled divisors' range
    for (int k = 0; k < 3; ++k) {
        const float B = __uint_as_float((exps[k] << 23) | m);
        bad += __float_as_uint(pxb::rcp_refined(B)) != __float_as_uint(__frcp_rn(B));
    }
    if (bad) atomicAdd(&counts[0], bad);
}

// counts[1]: components where unit3 differs from IEEE division, over seeded random
// constraints: a length l (log-uniform over [2^-24, 2^24], with random significands, plus every
// tenth one anywhere in [2^-70, 2^70]) and numerators of |a| <= l drawn four ways -- components
// of a random direction times l, random bit patterns below l (subnormals and quotients below
// 2^-100 included), numerators just below l, and signed zeros, +-l and subnormals.
__global__ void check_quotient_kernel(uint64_t seed, uint64_t n, unsigned long long* counts) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long bad = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t r0 = mix64(seed ^ (i * 0xD1B54A32D192ED03ull));
        const uint64_t r1 = mix64(r0);
        const uint64_t r2 = mix64(r1);
        const uint32_t lexp = (i % 10 == 9) ? 57u + static_cast<uint32_t>(r0 % 140u) : 103u + static_cast<uint32_t>(r0 % 48u);
        const float l = __uint_as_float((lexp << 23) | static_cast<uint32_t>((r0 >> 8) & 0x7fffffu));
        float a[3];
        const int mode = static_cast<int>((r0 >> 40) % 4u);
        for (int k = 0; k < 3; ++k) {
            const uint64_t rk = k == 0 ? r1 : (k == 1 ? r2 : mix64(r2));
            const uint32_t sign = static_cast<uint32_t>(rk >> 63) << 31;
            if (mode == 0) {  // a component of a random direction
                const float u = static_cast<float>((rk >> 40) & 0xffffffu) * (1.0f / 16777216.0f);
                a[k] = __uint_as_float(__float_as_uint(u * l) | sign);
            } else if (mode == 1) {  // a random bit pattern at or below l, subnormals included
                const uint32_t lb = __float_as_uint(l);
                a[k] = __uint_as_float(static_cast<uint32_t>(rk % (static_cast<uint64_t>(lb) + 1u)) | sign);
            } else if (mode == 2) {  // near l: the quotient just below 1
                const uint32_t lb = __float_as_uint(l);
                const uint32_t back = static_cast<uint32_t>(rk % 64u);
                a[k] = __uint_as_float((lb > back ? lb - back : 0u) | sign);
            } else {  // zeros, +-l, and a tiny subnormal
                const uint32_t pick = static_cast<uint32_t>(rk % 4u);
                a[k] = __uint_as_float((pick == 0 ? 0u : pick == 1 ? __float_as_uint(l) : pick == 2 ? 1u : 0x00400000u) | sign);
            }
        }
        float q[3];
        pxb::unit3(a[0], a[1], a[2], l, q[0], q[1], q[2]);
        for (int k = 0; k < 3; ++k) bad += __float_as_uint(q[k]) != __float_as_uint(__fdiv_rn(a[k], l));
    }
    if (bad) atomicAdd(&counts[1], bad);
}

// counts[2]: for divisor significands [b_first, b_first + gridDim.y) (b in [1, 2)) and every
// numerator significand (a in [1, 2)), quotients that differ from IEEE division. The method's
// rounding depends on the significands alone once the operands are scaled into range, so the
// whole 2^23 x 2^23 square is every case there is.
__global__ void check_significands_kernel(uint32_t b_first, unsigned long long* counts) {
    const uint32_t am = blockIdx.x * blockDim.x + threadIdx.x;
    if (am >= (1u << 23)) return;
    const float a = __uint_as_float((127u << 23) | am);
    const float na = a * -0x1p64f;
    uint32_t bad = 0;
    for (uint32_t k = 0; k < 64; ++k) {
        const uint32_t bm = b_first + blockIdx.y * 64u + k;
        if (bm >= (1u << 23)) break;
        const float b = __uint_as_float((127u << 23) | bm);
        const float B = b * 0x1p64f;
        const float q = pxb::quotient_scaled(na, B, -pxb::rcp_refined(B));
        bad += __float_as_uint(q) != __float_as_uint(__fdiv_rn(a, b));
    }
    if (bad) atomicAdd(&counts[2], bad);
}

// The projection as the reference writes it, scalar IEEE operations throughout (the check for
// distance_core's packed and reciprocal-sharing form).
__device__ __noinline__ bool distance_scalar(float4& pa, float4& pb, float rest, float lam, float alpha, float& dlambda) {
    const float w = pa.w + pb.w;
    const float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    const float l = sqrtf(dx * dx + dy * dy + dz * dz);
    const bool ok = !(w <= 0.0f) && !(l < PXB_EPSILON);
    const float nx = __fdiv_rn(dx, l), ny = __fdiv_rn(dy, l), nz = __fdiv_rn(dz, l);
    const float c = l - rest;
    dlambda = __fdiv_rn(-c - alpha * lam, w + alpha);
    const float cx = dlambda * nx, cy = dlambda * ny, cz = dlambda * nz;
    pa.x = pa.x + pa.w * cx;
    pa.y = pa.y + pa.w * cy;
    pa.z = pa.z + pa.w * cz;
    pb.x = pb.x - pb.w * cx;
    pb.y = pb.y - pb.w * cy;
    pb.z = pb.z - pb.w * cz;
    return ok;
}

__device__ __forceinline__ float rnd_coord(uint64_t r, int mode) {
    // positions around the origin: ordinary values, values near zero, exact zeros
    const uint32_t sign = static_cast<uint32_t>(r >> 63) << 31;
    if (mode == 0) return __uint_as_float(sign | ((118u + static_cast<uint32_t>(r % 12u)) << 23) | static_cast<uint32_t>((r >> 8) & 0x7fffffu));
    if (mode == 1) return __uint_as_float(sign | static_cast<uint32_t>((r >> 8) % 0x3f800000u));
    return (r & 1) ? 0.0f : -0.0f;
}

// counts[3]: projections where distance_core differs from distance_scalar in any output bit
// (positions, dlambda, the early-return flag), over seeded random endpoint pairs: ordinary
// coordinates, coordinates anywhere below 1 (subnormals included) and signed zeros, inverse masses
// of 0 or random, compliances 0 or random, lambdas 0 or random. The first differing input goes to
// first_bad (8 floats: pa, pb).
__global__ void check_projection_kernel(uint64_t seed, uint64_t n, unsigned long long* counts, float* first_bad) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long bad = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t r = mix64(seed ^ (i * 0x9E3779B97F4A7C15ull));
        float v[8];
        const int mode = static_cast<int>(r % 8u);
        for (int k = 0; k < 8; ++k) {
            r = mix64(r);
            if (k == 3 || k == 7) {
                v[k] = (r % 5u == 0) ? 0.0f : static_cast<float>((r >> 20) & 0xffffu) * (1.0f / 64.0f);
            } else {
                const int m = mode < 5 ? 0 : (mode < 7 ? 1 : (r % 3u == 0 ? 2 : 0));
                v[k] = rnd_coord(r, m);
                if (mode < 3 && k >= 4) v[k] = v[k - 4] + __uint_as_float(((100u + static_cast<uint32_t>(r % 24u)) << 23)) * ((r >> 40) & 1 ? 1.0f : -1.0f);
            }
        }
        r = mix64(r);
        const float rest = static_cast<float>((r >> 16) & 0xffffu) * (1.0f / 32768.0f);
        const float lam = (r & 3) ? 0.0f : static_cast<float>((r >> 40) & 0xffffu) * (1.0f / 65536.0f) - 0.5f;
        const float alpha = (r & 12) ? 0.0f : static_cast<float>((r >> 32) & 0xffu) * 0.25f;
        float4 a1 = make_float4(v[0], v[1], v[2], v[3]), b1 = make_float4(v[4], v[5], v[6], v[7]);
        float4 a2 = a1, b2 = b1;
        float d1 = 0.0f, d2 = 0.0f;
        const bool ok1 = pxb::distance_core<true>(a1, b1, rest, lam, alpha, d1);
        const bool ok2 = distance_scalar(a2, b2, rest, lam, alpha, d2);
        bool same = ok1 == ok2;
        if (ok2) {
            same = same && __float_as_uint(a1.x) == __float_as_uint(a2.x) && __float_as_uint(a1.y) == __float_as_uint(a2.y) &&
                   __float_as_uint(a1.z) == __float_as_uint(a2.z) && __float_as_uint(b1.x) == __float_as_uint(b2.x) &&
                   __float_as_uint(b1.y) == __float_as_uint(b2.y) && __float_as_uint(b1.z) == __float_as_uint(b2.z) &&
                   __float_as_uint(d1) == __float_as_uint(d2);
        }
        if (!same) {
            if (atomicAdd(&counts[4], 1ull) == 0)
                for (int k = 0; k < 8; ++k) first_bad[k] = v[k];
            ++bad;
        }
    }
    if (bad) atomicAdd(&counts[3], bad);
}

}  // namespace

extern "C" pxb_status pxb_check_projections(pxb_context* ctx, uint64_t samples, uint64_t seed, uint64_t* mismatches,
                                            float* first_bad) {
    if (!ctx || !mismatches) return PXB_ERR_INVALID_ARGUMENT;
    if (pxb_status s = ctx->grow(ctx->d_scratch, 64 + 32, "projection check")) return s;
    auto* counts = static_cast<unsigned long long*>(ctx->d_scratch.p);
    float* fb = reinterpret_cast<float*>(static_cast<char*>(ctx->d_scratch.p) + 64);
    cudaError_t e = cudaMemsetAsync(counts, 0, 64 + 32, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "clear counts");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    check_projection_kernel<<<sms * 8, 256, 0, ctx->stream>>>(seed, samples, counts, fb);
    ++ctx->launches;
    unsigned long long host[5] = {0, 0, 0, 0, 0};
    float hfb[8] = {0};
    e = cudaMemcpyAsync(host, counts, 40, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hfb, fb, 32, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "projection check");
    *mismatches = host[3];
    if (first_bad) for (int k = 0; k < 8; ++k) first_bad[k] = hfb[k];
    return PXB_OK;
}

extern "C" pxb_status pxb_check_quotient_significands(pxb_context* ctx, uint32_t b_first, uint32_t b_count,
                                                      uint64_t* mismatches) {
    if (!ctx || !mismatches) return PXB_ERR_INVALID_ARGUMENT;
    if (b_first >= (1u << 23) || b_count > (1u << 23) - b_first) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "divisor significands out of range");
    if (pxb_status s = ctx->grow(ctx->d_scratch, 24, "quotient check")) return s;
    auto* counts = static_cast<unsigned long long*>(ctx->d_scratch.p);
    cudaError_t e = cudaMemsetAsync(counts, 0, 24, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "clear counts");
    // launches of at most 2^9 x 64 divisors each (2^38 quotients, about a second)
    for (uint32_t b = b_first; b < b_first + b_count; b += 512u * 64u) {
        const uint32_t n = std::min<uint32_t>(512u * 64u, b_first + b_count - b);
        check_significands_kernel<<<dim3((1u << 23) / 256, (n + 63) / 64), 256, 0, ctx->stream>>>(b, counts);
        ++ctx->launches;
    }
    unsigned long long host[3] = {0, 0, 0};
    e = cudaMemcpyAsync(host, counts, 24, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "quotient check");
    *mismatches = host[2];
    return PXB_OK;
}

extern "C" pxb_status pxb_check_quotients(pxb_context* ctx, uint64_t samples, uint64_t seed, uint64_t* mismatches) {
    if (!ctx || !mismatches) return PXB_ERR_INVALID_ARGUMENT;
    if (pxb_status s = ctx->grow(ctx->d_scratch, 16, "quotient check")) return s;
    auto* counts = static_cast<unsigned long long*>(ctx->d_scratch.p);
    cudaError_t e = cudaMemsetAsync(counts, 0, 16, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "clear counts");
    check_reciprocal_kernel<<<(1u << 23) / 256, 256, 0, ctx->stream>>>(counts);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    check_quotient_kernel<<<sms * 8, 256, 0, ctx->stream>>>(seed, samples, counts);
    ctx->launches += 2;
    unsigned long long host[2] = {0, 0};
    e = cudaMemcpyAsync(host, counts, 16, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda(e, "quotient check");
    mismatches[0] = host[0];
    mismatches[1] = host[1];
    return PXB_OK;
}

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
