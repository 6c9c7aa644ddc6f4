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
//   * one warp then walks the particles in index order. For particle i, 27 lanes each own one of
//     the 27 cells (in the reference's scan order) and scan their bucket for the first candidate
//     that pushes; the first such candidate in the reference's order is applied and the cells
//     after it are scanned again against the moved particle. The pushes, and the positions every
//     test sees, are the reference's, in its order.
// Tables (PXB_SELF_WORDS words of dynamic shared memory at `tab`): bucket ends [buckets + 1],
// sorted particle indices [n], block-scan scratch [32].
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

// One particle of the pair pass (cloth_solver.h:325-365), exactly, by the whole warp. Lane k < 27
// owns cell k of the reference's scan order (dx, dy, dz) = (k % 3, k / 3 % 3, k / 9) - 1, dz
// outermost, and a cursor into that cell's bucket. Each round every lane scans from its cursor to
// its first candidate that pushes against the current positions; the lowest such lane holds the
// first pushing candidate in the reference's order, applies it and moves its cursor past it. The
// lanes before it have tested all their candidates and are done; the lanes after it scan again
// from where they were, against the moved particle. Returns whether any push ran.
// The 1-ring exemption (cloth_solver.h:346-352) reads the cloth's own `columns` (ex_cols, 0: no
// exemption, row by multiply-high with ex_magic); the layout's columns (cols) only place particles.
// On a grid cloth the two are the same.
__device__ bool self_exact_particle(float4* pos, const uint32_t* tab, int i, int n, int cols, uint32_t col_magic,
                                   int ex_cols, uint32_t ex_magic, int Q, int S, uint32_t buckets, float d_min,
                                   float d2_min, float inv_cell, int lane) {
    const uint32_t* ends = tab;
    const uint32_t* sorted = tab + buckets + 1;
    const int yi = static_cast<int>(__umulhi(static_cast<uint32_t>(i), col_magic)), xi = i - yi * cols;
    const int li = yi * S + (xi & 3) * Q + (xi >> 2);
    const bool ex_same = ex_cols == cols;
    const int eyi = ex_same ? yi : (ex_cols ? static_cast<int>(__umulhi(static_cast<uint32_t>(i), ex_magic)) : 0);
    const int exi = ex_same ? xi : i - eyi * ex_cols;
    float4 pi = pos[li];
    if (pi.w == 0.0f) return false;
    const int32_t cx = static_cast<int32_t>(floorf(pi.x * inv_cell));
    const int32_t cy = static_cast<int32_t>(floorf(pi.y * inv_cell));
    const int32_t cz = static_cast<int32_t>(floorf(pi.z * inv_cell));
    uint32_t cur = 0u, last = 0u;
    if (lane < 27) {
        const uint32_t b = self_hash(cx + lane % 3 - 1, cy + lane / 3 % 3 - 1, cz + lane / 9 - 1, buckets);
        cur = b ? ends[b - 1] : 0u;
        last = ends[b];
    }
    bool any = false;
    for (;;) {
        bool hit = false;
        uint32_t hs = 0u;
        int lj = 0;
        float4 pj = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float dx = 0.0f, dy = 0.0f, dz = 0.0f, len2 = 0.0f, w = 0.0f;
        for (uint32_t s = cur; s < last; ++s) {
            const int j = static_cast<int>(sorted[s]);
            if (j <= i) continue;  // each pair once
            const int yj = static_cast<int>(__umulhi(static_cast<uint32_t>(j), col_magic)), xj = j - yj * cols;
            if (ex_cols) {  // the 1-ring is exempt
                int exj = xj, eyj = yj;
                if (!ex_same) {
                    eyj = static_cast<int>(__umulhi(static_cast<uint32_t>(j), ex_magic));
                    exj = j - eyj * ex_cols;
                }
                if (abs(exi - exj) <= 1 && abs(eyi - eyj) <= 1) continue;
            }
            const int l = yj * S + (xj & 3) * Q + (xj >> 2);
            const float4 q = pos[l];
            const float ww = pi.w + q.w;
            if (ww <= 0.0f) continue;
            const float ex = pi.x - q.x, ey = pi.y - q.y, ez = pi.z - q.z;
            const float e2 = ex * ex + ey * ey + ez * ez;
            if (e2 >= d2_min || e2 < PXB_EPSILON) continue;
            hit = true;
            hs = s;
            lj = l;
            pj = q;
            dx = ex; dy = ey; dz = ez; len2 = e2; w = ww;
            break;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (!m) break;
        any = true;
        const int k0 = __ffs(m) - 1;
        if (lane == k0) {
            const float len = sqrtf(len2);
            const float sc = (d_min - len) / w;
            const float px = (dx / len) * sc, py = (dy / len) * sc, pz = (dz / len) * sc;
            pi.x = pi.x + px * pi.w;
            pi.y = pi.y + py * pi.w;
            pi.z = pi.z + pz * pi.w;
            pj.x = pj.x - px * pj.w;
            pj.y = pj.y - py * pj.w;
            pj.z = pj.z - pz * pj.w;
            pos[lj] = pj;
            pos[li] = pi;
            cur = hs + 1u;
        } else if (lane < k0) {
            cur = last;
        }
        __syncwarp();
        pi = pos[li];
    }
    return any;
}

// The pair pass of cloth_solver.h:325-365, by warp 0 (the caller's other warps wait at the
// barrier after it): every particle in index order, each exactly. `pos` holds xyz + inverse mass
// in layout order; it is written as the pass goes, so it carries no restrict promise.
__device__ void self_pair_pass(float4* pos, const uint32_t* tab, int n, int cols, int ex_cols, int Q, int S,
                               uint32_t buckets, float d_min, float inv_cell, int lane) {
    const float d2_min = d_min * d_min;
    // row of index j = umulhi(j, ceil(2^32 / cols)), checked exact on the host for every j < n,
    // and the same for ex_cols
    const uint32_t col_magic = static_cast<uint32_t>((0x100000000ull + static_cast<uint32_t>(cols) - 1u) /
                                                     static_cast<uint32_t>(cols));
    const uint32_t ex_magic = ex_cols > 0 ? static_cast<uint32_t>((0x100000000ull + static_cast<uint32_t>(ex_cols) - 1u) /
                                                                  static_cast<uint32_t>(ex_cols))
                                          : 0u;
    for (int i = 0; i < n; ++i)
        self_exact_particle(pos, tab, i, n, cols, col_magic, ex_cols, ex_magic, Q, S, buckets, d_min, d2_min, inv_cell,
                            lane);
    __syncwarp();
}

}  // namespace
}  // namespace pxb

#endif  // PXB_SELF_COLLISION_CUH
