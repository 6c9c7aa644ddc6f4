// consumers.cu -- what the cloth's readers take from it each frame, produced from the device state:
//   * the bytes PhysicsWorld::world_state_hash mixes for the cloths (world.h:1334-1359): every
//     particle's position then velocity, cloth after cloth, through FNV-1a 64. The hash is a
//     serial byte chain, so the device gathers the bytes in that order (one launch for every
//     cloth) and the host runs the chain;
//   * a renderer's vertex buffer over Cloth::triangles (cloth.h:293-299): per particle its
//     position and unit vertex normal, the normal being the sum of cross(b - a, c - a) over the
//     particle's triangles in ascending triangle order (a grid cloth's from make_grid_cloth's two
//     per cell, any other cloth's from its triangle index), normalized.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"
#include "runtime_internal.h"

namespace {

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

__device__ __forceinline__ int slot(int x, int y, int Q, int S) { return y * S + (x & 3) * Q + (x >> 2); }

// 6 floats per particle in index order: position xyz, velocity xyz.
__global__ void gather_state_kernel(const PxbClothDev* __restrict__ cloths, const int32_t* __restrict__ order,
                                    const int64_t* __restrict__ offsets, float* __restrict__ out) {
    const PxbClothDev* C = &cloths[__ldg(&order[blockIdx.y])];
    const int cols = C->columns, n = C->n_real, Q = C->Q, S = C->S;
    float* dst = out + __ldg(&offsets[blockIdx.y]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / cols, x = i - y * cols;
        const int l = slot(x, y, Q, S);
        const float4 p = C->pos[l], v = C->vel[l];
        dst[6 * i] = p.x; dst[6 * i + 1] = p.y; dst[6 * i + 2] = p.z;
        dst[6 * i + 3] = v.x; dst[6 * i + 4] = v.y; dst[6 * i + 5] = v.z;
    }
}

struct P3 {
    float x, y, z;
};
__device__ __forceinline__ P3 ld(const float4* pos, int x, int y, int Q, int S) {
    const float4 p = pos[slot(x, y, Q, S)];
    return P3{p.x, p.y, p.z};
}
// n += cross(b - a, c - a)
__device__ __forceinline__ void face(P3 a, P3 b, P3 c, P3& n) {
    const float ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const float vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
    n.x = n.x + (uy * vz - vy * uz);
    n.y = n.y + (uz * vx - vz * ux);
    n.z = n.z + (ux * vy - vx * uy);
}

// 6 floats per particle in index order: position xyz, unit normal xyz. The faces of cell (x, y)
// are (i00, i10, i11) and (i00, i11, i01) (cloth_builder.h:200-207); a particle sums the faces it
// belongs to in ascending triangle order; a zero sum gives a zero normal.
__global__ void render_buffer_kernel(const PxbClothDev* __restrict__ cloths, const int32_t* __restrict__ order,
                                     const int64_t* __restrict__ offsets, float* __restrict__ out) {
    const PxbClothDev* C = &cloths[__ldg(&order[blockIdx.y])];
    const int cols = C->columns, rows = C->rows, n = C->n_real, Q = C->Q, S = C->S;
    const float4* pos = C->pos;
    float* dst = out + __ldg(&offsets[blockIdx.y]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / cols, x = i - y * cols;
        const P3 p = ld(pos, x, y, Q, S);
        P3 nm{0.0f, 0.0f, 0.0f};
        if (C->topology != 0) {
            // general topology: the particle's triangles from the triangle index, ascending
            const int l = slot(x, y, Q, S);
            for (int k = C->tri_off[l]; k < C->tri_off[l + 1]; ++k) {
                const int4 t = C->tri_ent[k];
                const float4 a = pos[t.x], b = pos[t.y], c = pos[t.z];
                face(P3{a.x, a.y, a.z}, P3{b.x, b.y, b.z}, P3{c.x, c.y, c.z}, nm);
            }
            const float l2 = nm.x * nm.x + nm.y * nm.y + nm.z * nm.z;
            const float s = l2 > 0.0f ? 1.0f / sqrtf(l2) : 0.0f;
            dst[6 * i] = p.x; dst[6 * i + 1] = p.y; dst[6 * i + 2] = p.z;
            dst[6 * i + 3] = nm.x * s; dst[6 * i + 4] = nm.y * s; dst[6 * i + 5] = nm.z * s;
            continue;
        }
        const bool xm = x >= 1, xp = x + 1 < cols, ym = y >= 1, yp = y + 1 < rows;
        if (xm && ym) {  // cell (x-1, y-1): both faces
            const P3 a = ld(pos, x - 1, y - 1, Q, S), b = ld(pos, x, y - 1, Q, S), d = ld(pos, x - 1, y, Q, S);
            face(a, b, p, nm);
            face(a, p, d, nm);
        }
        if (xp && ym) face(ld(pos, x, y - 1, Q, S), ld(pos, x + 1, y, Q, S), p, nm);  // cell (x, y-1): second face
        if (xm && yp) face(ld(pos, x - 1, y, Q, S), p, ld(pos, x, y + 1, Q, S), nm);  // cell (x-1, y): first face
        if (xp && yp) {  // cell (x, y): both faces
            const P3 b = ld(pos, x + 1, y, Q, S), c = ld(pos, x + 1, y + 1, Q, S), d = ld(pos, x, y + 1, Q, S);
            face(p, b, c, nm);
            face(p, c, d, nm);
        }
        const float l2 = nm.x * nm.x + nm.y * nm.y + nm.z * nm.z;
        const float s = l2 > 0.0f ? 1.0f / sqrtf(l2) : 0.0f;
        dst[6 * i] = p.x; dst[6 * i + 1] = p.y; dst[6 * i + 2] = p.z;
        dst[6 * i + 3] = nm.x * s; dst[6 * i + 4] = nm.y * s; dst[6 * i + 5] = nm.z * s;
    }
}

// The listed cloths' 6-float-per-particle records, gathered by `kernel` into host `out`.
template <typename Kernel>
pxb_status gather6(pxb_context* ctx, const uint64_t* cloths, uint32_t n, float* out, size_t capacity, bool need_tris,
                   Kernel kernel, const char* what) {
    std::vector<int32_t> order(n);
    std::vector<int64_t> offs(n);
    int64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id %llu is not live", (unsigned long long)cloths[k]);
        if (need_tris && e->n_triangle_indices == 0)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "cloth %llu has no triangle list to render",
                             (unsigned long long)cloths[k]);
        order[k] = static_cast<int32_t>(e - ctx->cloths.data());
        offs[k] = total;
        total += 6 * static_cast<int64_t>(e->n_particles);
    }
    if (static_cast<size_t>(total) > capacity) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "output too small");
    if (n == 0) return PXB_OK;
    if (pxb_status s = ctx->sync_registry()) return s;
    const size_t o_offs = align256(4 * static_cast<size_t>(n));
    if (pxb_status s = ctx->grow(ctx->d_gather_meta, o_offs + 8 * static_cast<size_t>(n), "gather meta")) return s;
    if (pxb_status s = ctx->grow(ctx->d_gather, 4 * static_cast<size_t>(total), "gather")) return s;
    char* meta = static_cast<char*>(ctx->d_gather_meta.p);
    pxb_status s = ctx->cuda(cudaMemcpyAsync(meta, order.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), what);
    if (!s) s = ctx->cuda(cudaMemcpyAsync(meta + o_offs, offs.data(), 8 * n, cudaMemcpyHostToDevice, ctx->stream), what);
    if (s) return s;
    kernel<<<dim3(8, n), 256, 0, ctx->stream>>>(static_cast<const PxbClothDev*>(ctx->d_registry.p),
                                                reinterpret_cast<const int32_t*>(meta),
                                                reinterpret_cast<const int64_t*>(meta + o_offs),
                                                static_cast<float*>(ctx->d_gather.p));
    if ((s = ctx->cuda(cudaGetLastError(), what))) return s;
    ++ctx->launches;
    s = ctx->cuda(cudaMemcpyAsync(out, ctx->d_gather.p, 4 * static_cast<size_t>(total), cudaMemcpyDeviceToHost,
                                  ctx->stream), what);
    if (!s) s = ctx->cuda(cudaStreamSynchronize(ctx->stream), what);
    if (s) return s;
    return ctx->check_device_error();
}

}  // namespace

extern "C" {

pxb_status pxb_cloths_state_hash(pxb_context* ctx, const uint64_t* cloths, uint32_t n, uint64_t seed,
                                 uint64_t* hash_out) {
    if (!ctx || !hash_out || (n && !cloths)) return PXB_ERR_INVALID_ARGUMENT;
    size_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id %llu is not live", (unsigned long long)cloths[k]);
        total += 6 * static_cast<size_t>(e->n_particles);
    }
    std::vector<float> state(total);
    if (pxb_status s = gather6(ctx, cloths, n, state.data(), total, false, gather_state_kernel, "state hash")) return s;
    // FNV-1a 64 over the bytes, as world.h:1336-1341 mixes them
    uint64_t h = seed;
    const unsigned char* bytes = reinterpret_cast<const unsigned char*>(state.data());
    for (size_t i = 0, nb = total * sizeof(float); i < nb; ++i) {
        h ^= bytes[i];
        h *= 1099511628211ull;
    }
    *hash_out = h;
    return PXB_OK;
}

pxb_status pxb_cloths_read_render_buffer(pxb_context* ctx, const uint64_t* cloths, uint32_t n, float* out,
                                         size_t capacity) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    return gather6(ctx, cloths, n, out, capacity, true, render_buffer_kernel, "render buffer");
}

}  // extern "C"
