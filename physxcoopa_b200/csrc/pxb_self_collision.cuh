// pxb_self_collision.cuh -- stage 6 of cloth::solve_cloth, self-collision
// (physxcoopa/cloth/cloth_solver.h:291-366), for a cloth held by one CTA.
//
// The reference pass is serial: particle i in index order scans the 27 hash cells around its
// CURRENT position and pushes every later, non-neighbouring particle closer than self_distance
// apart, each push moving both particles before the next test. Its result depends on that order,
// so the device keeps it exactly:
//   * the spatial hash (detail::hash_cell, counting sort into bucket-major order, ascending index
//     within a bucket) is built by the whole CTA: atomic bucket counts, a block-wide exclusive
//     scan, and a stable scatter by one warp in index order (lanes of a chunk that share a bucket
//     take consecutive places in lane order);
//   * one warp then walks the particles in index order. For particle i the 27 cells are hashed by
//     27 lanes at once and their candidates numbered in the reference's scan order (dz, dy, dx,
//     then bucket position); 32 candidates are tested at a time against i's current position,
//     the first one that pushes is applied, and only the candidates after it are tested again
//     with the moved positions. The pushes, and the positions every test sees, are the
//     reference's, in its order.
// Tables (PXB_SELF_WORDS words of dynamic shared memory at `tab`): bucket ends [buckets + 1],
// sorted particle indices [n], scan scratch [32], candidate table [64].
#ifndef PXB_SELF_COLLISION_CUH
#define PXB_SELF_COLLISION_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "pxb_internal.h"

namespace pxb {
namespace {

// detail::hash_cell (cloth_solver.h:100-105): Teschner's three primes, masked to `buckets`.
__device__ __forceinline__ uint32_t self_hash(int32_t x, int32_t y, int32_t z, uint32_t buckets) {
    const uint32_t h = static_cast<uint32_t>(x) * 73856093u ^ static_cast<uint32_t>(y) * 19349663u ^
                       static_cast<uint32_t>(z) * 83492791u;
    return h & (buckets - 1u);
}

__device__ __forceinline__ int self_slot(int i, int cols, int Q, int S) {
    const int y = i / cols, x = i - y * cols;
    return y * S + (x & 3) * Q + (x >> 2);
}

__device__ __forceinline__ uint32_t self_cell_of(float4 p, float inv_cell, uint32_t buckets) {
    return self_hash(static_cast<int32_t>(floorf(p.x * inv_cell)), static_cast<int32_t>(floorf(p.y * inv_cell)),
                     static_cast<int32_t>(floorf(p.z * inv_cell)), buckets);
}

// The counting sort of cloth_solver.h:300-323. On return ends[b] is the end of bucket b (bucket b
// spans [b ? ends[b-1] : 0, ends[b])) and sorted[] lists indices bucket by bucket, ascending.
// Called by every thread of the CTA; T must be a multiple of 32.
__device__ void self_build_hash(const float4* pos, uint32_t* tab, int n, int cols, int Q, int S,
                                uint32_t buckets, float inv_cell, int tid, int T) {
    uint32_t* ends = tab;
    uint32_t* sorted = tab + buckets + 1;
    uint32_t* scan = sorted + n;
    const int lane = tid & 31, warp = tid >> 5;
    for (uint32_t b = tid; b <= buckets; b += T) ends[b] = 0u;
    __syncthreads();
    for (int i = tid; i < n; i += T) atomicAdd(&ends[self_cell_of(pos[self_slot(i, cols, Q, S)], inv_cell, buckets)], 1u);
    __syncthreads();
    // exclusive scan of the counts: a contiguous run of buckets per thread
    const uint32_t per = (buckets + T - 1) / T;
    const uint32_t b0 = per * tid < buckets ? per * tid : buckets;
    const uint32_t b1 = b0 + per < buckets ? b0 + per : buckets;
    uint32_t local = 0;
    for (uint32_t b = b0; b < b1; ++b) local += ends[b];
    uint32_t x = local;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scan[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = lane < (T >> 5) ? scan[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        scan[lane] = v;
    }
    __syncthreads();
    uint32_t run = (warp > 0 ? scan[warp - 1] : 0u) + x - local;
    for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t c = ends[b];
        ends[b] = run;
        run += c;
    }
    if (tid == 0) ends[buckets] = static_cast<uint32_t>(n);
    __syncthreads();
    // stable scatter in index order, 32 particles at a time (ends[b] advances to the bucket's end)
    if (warp == 0) {
        for (int i0 = 0; i0 < n; i0 += 32) {
            const int i = i0 + lane;
            const bool v = i < n;
            const uint32_t cell = v ? self_cell_of(pos[self_slot(i, cols, Q, S)], inv_cell, buckets) : 0xffffffffu;
            const uint32_t peers = __match_any_sync(0xffffffffu, cell);
            const uint32_t before = __popc(peers & ((1u << lane) - 1u));
            const uint32_t start = v ? ends[cell] : 0u;
            __syncwarp();
            if (v) {
                sorted[start + before] = static_cast<uint32_t>(i);
                if (before == 0) ends[cell] = start + __popc(peers);
            }
            __syncwarp();
        }
    }
    __syncthreads();
}

// The pair pass of cloth_solver.h:325-365, by warp 0 (the caller's other warps wait at the
// barrier after it). `pos` holds xyz + inverse mass in layout order.
// The candidate table is rewritten for every particle, so `tab` is a plain pointer: no const or
// restrict promise that would let the compiler keep an earlier particle's table.
__device__ void self_pair_pass(float4* pos, uint32_t* tab, int n, int cols, int Q, int S, uint32_t buckets,
                               float d_min, float inv_cell, int lane) {
    const uint32_t* ends = tab;
    const uint32_t* sorted = tab + buckets + 1;
    uint32_t* cell_first = tab + buckets + 1 + n + 32;
    uint32_t* cell_excl = cell_first + 32;
    const float d2_min = d_min * d_min;
    for (int i = 0; i < n; ++i) {
        const int yi = i / cols, xi = i - yi * cols;
        const int li = yi * S + (xi & 3) * Q + (xi >> 2);
        float4 pi = pos[li];
        if (pi.w == 0.0f) continue;
        const int32_t cx = static_cast<int32_t>(floorf(pi.x * inv_cell));
        const int32_t cy = static_cast<int32_t>(floorf(pi.y * inv_cell));
        const int32_t cz = static_cast<int32_t>(floorf(pi.z * inv_cell));
        // lane k < 27 is cell (dx, dy, dz) = (k % 3, k / 3 % 3, k / 9) - 1: the reference's loop
        // order, dz outermost
        uint32_t first = 0u, cnt = 0u;
        if (lane < 27) {
            const uint32_t b = self_hash(cx + lane % 3 - 1, cy + lane / 3 % 3 - 1, cz + lane / 9 - 1, buckets);
            first = b ? ends[b - 1] : 0u;
            cnt = ends[b] - first;
        }
        uint32_t inc = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
        if (total == 0u) continue;
        cell_first[lane] = first;
        cell_excl[lane] = inc - cnt;
        __syncwarp();
        for (uint32_t c0 = 0; c0 < total; c0 += 32u) {
            const uint32_t c = c0 + static_cast<uint32_t>(lane);
            int j = -1, lj = 0;
            if (c < total) {
                // the last cell whose first candidate number is <= c holds candidate c
                int lo = 0, hi = 26;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (cell_excl[mid] <= c) lo = mid;
                    else hi = mid - 1;
                }
                j = static_cast<int>(sorted[cell_first[lo] + (c - cell_excl[lo])]);
                const int yj = j / cols, xj = j - yj * cols;
                // each pair once; the 1-ring (Chebyshev distance 1 on the grid) is exempt
                if (j <= i || (abs(xi - xj) <= 1 && abs(yi - yj) <= 1)) j = -1;
                else lj = yj * S + (xj & 3) * Q + (xj >> 2);
            }
            uint32_t done = 0u;  // lanes at or before the last push of this chunk
            for (;;) {
                bool push = false;
                float4 pj = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                float dx = 0.0f, dy = 0.0f, dz = 0.0f, len2 = 0.0f, w = 0.0f;
                if (j >= 0 && !((done >> lane) & 1u)) {
                    pj = pos[lj];
                    w = pi.w + pj.w;
                    if (w > 0.0f) {
                        dx = pi.x - pj.x;
                        dy = pi.y - pj.y;
                        dz = pi.z - pj.z;
                        len2 = dx * dx + dy * dy + dz * dz;
                        push = !(len2 >= d2_min || len2 < PXB_EPSILON);
                    }
                }
                const uint32_t m = __ballot_sync(0xffffffffu, push);
                if (!m) break;
                const int k0 = __ffs(m) - 1;
                if (lane == k0) {
                    const float len = sqrtf(len2);
                    const float s = (d_min - len) / w;
                    const float px = (dx / len) * s, py = (dy / len) * s, pz = (dz / len) * s;
                    pi.x = pi.x + px * pi.w;
                    pi.y = pi.y + py * pi.w;
                    pi.z = pi.z + pz * pi.w;
                    pj.x = pj.x - px * pj.w;
                    pj.y = pj.y - py * pj.w;
                    pj.z = pj.z - pz * pj.w;
                    pos[lj] = pj;
                    pos[li] = pi;
                }
                __syncwarp();
                pi = pos[li];
                done = k0 == 31 ? 0xffffffffu : ((2u << k0) - 1u);
            }
        }
        __syncwarp();
    }
}

}  // namespace
}  // namespace pxb

#endif  // PXB_SELF_COLLISION_CUH
