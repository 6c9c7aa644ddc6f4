// tethers.cu -- cloth::build_tethers (physxcoopa/cloth/cloth_builder.h:308-358) on the device.
//
// The reference runs Dijkstra over the stretch graph from every anchored particle at once and
// tethers each free particle to the anchor it reached first, at its float path length times
// tether_scale. With non-negative float edge lengths and round-to-nearest additions, its
// distances satisfy dist[v] = min over neighbours u of fl(dist[u] + |p_v - p_u|), and when no
// edge vanishes in such a sum (fl(dist[u] + w) > dist[u] for distinct u, v) that fixpoint is
// unique, so a parallel relaxation reaches the same floats. Its priority queue then settles
// vertices in (dist, index) order, and the relaxation that fixed dist[v] came from the first
// settled neighbour reaching it: the smallest (dist[u], u) among the neighbours with
// fl(dist[u] + w) == dist[v]. Following those predecessors to their anchor gives the reference's
// source. A vanishing edge breaks both facts; the device detects it and refuses.
//
// Steps: adjacency (degrees, one-block scan, scatter), rounds of frontier relaxation with
// atomicMin on the distances' bit patterns (non-negative floats order as their bits) until no
// distance moves, the predecessor pass (which also checks for vanishing edges), pointer jumping
// to the anchors, then the tether list in particle order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "runtime_internal.h"

namespace {

constexpr uint32_t kInfBits = 0x7f7fffffu;  // std::numeric_limits<float>::max(): "not reached"
constexpr uint32_t kIdle = 0xffffffffu;     // relaxation round stamp of a particle nobody moved

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// glm::length(p_v - p_u): sqrt of x*x + y*y + z*z, left to right
__device__ __forceinline__ float edge_len(const pxb_particle* __restrict__ p, uint32_t u, uint32_t v) {
    const float dx = p[v].position[0] - p[u].position[0];
    const float dy = p[v].position[1] - p[u].position[1];
    const float dz = p[v].position[2] - p[u].position[2];
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

__global__ void degree_kernel(const pxb_constraint* __restrict__ e, uint32_t m, uint32_t* __restrict__ deg) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = e[k].a, b = e[k].b;
        if (a == b) continue;  // a self-edge relaxes nothing (candidate >= dist)
        atomicAdd(&deg[a], 1u);
        atomicAdd(&deg[b], 1u);
    }
}

// Exclusive scan of deg[0, n) into off[0, n] by one block: each thread sums a contiguous chunk,
// the block scans the chunk sums, each thread writes its chunk's prefixes.
__global__ void scan_kernel(const uint32_t* __restrict__ deg, uint32_t n, uint32_t* __restrict__ off) {
    __shared__ uint32_t s[1024];
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const uint32_t chunk = (n + T - 1) / T;
    const uint32_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; ++i) sum += deg[i];
    s[t] = sum;
    __syncthreads();
    for (uint32_t d = 1; d < T; d <<= 1) {
        const uint32_t v = t >= d ? s[t - d] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    uint32_t run = s[t] - sum;
    for (uint32_t i = lo; i < hi; ++i) {
        off[i] = run;
        run += deg[i];
    }
    if (t == T - 1) off[n] = s[t];
}

__global__ void scatter_kernel(const pxb_constraint* __restrict__ e, uint32_t m, uint32_t* __restrict__ cursor,
                               uint32_t* __restrict__ adj) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = e[k].a, b = e[k].b;
        if (a == b) continue;
        adj[atomicAdd(&cursor[a], 1u)] = b;
        adj[atomicAdd(&cursor[b], 1u)] = a;
    }
}

__global__ void seed_kernel(uint32_t n, uint32_t* __restrict__ dist, uint32_t* __restrict__ stamp,
                            uint8_t* __restrict__ anchor) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        dist[i] = kInfBits;
        stamp[i] = kIdle;
        anchor[i] = 0;
    }
}

__global__ void seed_anchors_kernel(const pxb_anchor* __restrict__ a, uint32_t na, uint32_t* __restrict__ dist,
                                    uint32_t* __restrict__ stamp, uint8_t* __restrict__ anchor) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < na; k += gridDim.x * blockDim.x) {
        const uint32_t p = a[k].particle;
        dist[p] = 0u;  // +0.0f
        stamp[p] = 0u;
        anchor[p] = 1;
    }
}

// One round: every particle moved in the previous round offers dist + edge to its neighbours.
__global__ void relax_kernel(const pxb_particle* __restrict__ p, const uint32_t* __restrict__ off,
                             const uint32_t* __restrict__ adj, uint32_t n, uint32_t round, uint32_t* dist,
                             uint32_t* stamp, uint32_t* __restrict__ moved) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        if (stamp[u] != round) continue;
        const float du = __uint_as_float(dist[u]);
        for (uint32_t k = off[u]; k < off[u + 1]; ++k) {
            const uint32_t v = adj[k];
            const uint32_t cb = __float_as_uint(du + edge_len(p, u, v));
            if (cb >= dist[v]) continue;  // candidate >= dist[next]: no improvement
            if (cb < atomicMin(&dist[v], cb)) {
                stamp[v] = round + 1;
                *moved = 1u;
            }
        }
    }
}

// The neighbour the reference's queue settles first among those reaching dist[v]; flags a
// vanishing edge or a particle no neighbour explains.
__global__ void pred_kernel(const pxb_particle* __restrict__ p, const uint32_t* __restrict__ off,
                            const uint32_t* __restrict__ adj, uint32_t n, const uint32_t* __restrict__ dist,
                            const uint8_t* __restrict__ anchor, int32_t* __restrict__ jump,
                            uint32_t* __restrict__ flags) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t dv = dist[v];
        bool vanish = false;
        unsigned long long best = ~0ull;
        for (uint32_t k = off[v]; k < off[v + 1]; ++k) {
            const uint32_t u = adj[k];
            const uint32_t du = dist[u];
            if (du == kInfBits) continue;
            const float cand = __uint_as_float(du) + edge_len(p, u, v);
            if (cand == __uint_as_float(du)) vanish = true;
            if (__float_as_uint(cand) == dv) best = min(best, (static_cast<unsigned long long>(du) << 32) | u);
        }
        if (vanish) atomicOr(flags, 1u);
        if (dv == kInfBits) {
            jump[v] = -1;  // no anchor reaches it
        } else if (anchor[v]) {
            jump[v] = static_cast<int32_t>(v);
        } else if (best == ~0ull) {
            jump[v] = -1;
            atomicOr(flags, 2u);
        } else {
            jump[v] = static_cast<int32_t>(best & 0xffffffffu);
        }
    }
}

__global__ void jump_kernel(uint32_t n, int32_t* jump, uint32_t* __restrict__ moved) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int32_t j = jump[v];
        if (j < 0) continue;
        const int32_t jj = jump[j];
        if (jj != j) {
            jump[v] = jj;
            *moved = 1u;
        }
    }
}

// Per particle: max_length (dist x scale) and its anchor, or anchor -1 when it gets no tether.
__global__ void emit_kernel(const pxb_particle* __restrict__ p, uint32_t n, const uint32_t* __restrict__ dist,
                            const int32_t* __restrict__ jump, float scale, float* __restrict__ len,
                            int32_t* __restrict__ src) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool tether = p[i].inv_mass != 0.0f && dist[i] < kInfBits && jump[i] >= 0;
        len[i] = __uint_as_float(dist[i]) * scale;
        src[i] = tether ? jump[i] : -1;
    }
}

}  // namespace

extern "C" {

pxb_status pxb_build_tethers_device(pxb_context* ctx, const pxb_particle* particles, uint32_t n,
                                    const pxb_constraint* stretch, uint32_t m, const pxb_anchor* anchors,
                                    uint32_t na, float tether_scale, pxb_tether* out, uint32_t capacity,
                                    uint32_t* n_out) {
    if (!ctx || !n_out || (n && !particles) || (m && !stretch) || (na && !anchors)) return PXB_ERR_INVALID_ARGUMENT;
    *n_out = 0;
    for (uint32_t k = 0; k < m; ++k)
        if (stretch[k].a >= n || stretch[k].b >= n)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "stretch constraint %u indexes past the particles", k);
    for (uint32_t k = 0; k < na; ++k)
        if (anchors[k].particle >= n)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "anchor %u indexes past the particles", k);
    if (n == 0 || na == 0) return PXB_OK;  // cloth_builder.h:310: no anchors, no tethers
    if (capacity && !out) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null output");

    // --- one allocation: particles | constraints | anchors | offsets | cursor | adjacency |
    //     dist | stamp | jump | len | src | anchor flags | two counters ---
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align256(std::max<size_t>(bytes, 16));
        return o;
    };
    const size_t N = n;
    const size_t o_p = take(sizeof(pxb_particle) * N), o_e = take(sizeof(pxb_constraint) * m),
                 o_a = take(sizeof(pxb_anchor) * na), o_off = take(4 * (N + 1)), o_cur = take(4 * (N + 1)),
                 o_adj = take(8 * static_cast<size_t>(m)), o_d = take(4 * N), o_st = take(4 * N),
                 o_j = take(4 * N), o_len = take(4 * N), o_src = take(4 * N), o_anc = take(N),
                 o_flag = take(8);
    void* mem = nullptr;
    if (pxb_status s = ctx->cuda(cudaMalloc(&mem, off), "cudaMalloc(tethers)")) return s;
    char* b = static_cast<char*>(mem);
    auto* dp = reinterpret_cast<pxb_particle*>(b + o_p);
    auto* de = reinterpret_cast<pxb_constraint*>(b + o_e);
    auto* da = reinterpret_cast<pxb_anchor*>(b + o_a);
    auto* doff = reinterpret_cast<uint32_t*>(b + o_off);
    auto* dcur = reinterpret_cast<uint32_t*>(b + o_cur);
    auto* dadj = reinterpret_cast<uint32_t*>(b + o_adj);
    auto* dd = reinterpret_cast<uint32_t*>(b + o_d);
    auto* dst = reinterpret_cast<uint32_t*>(b + o_st);
    auto* dj = reinterpret_cast<int32_t*>(b + o_j);
    auto* dlen = reinterpret_cast<float*>(b + o_len);
    auto* dsrc = reinterpret_cast<int32_t*>(b + o_src);
    auto* danc = reinterpret_cast<uint8_t*>(b + o_anc);
    auto* dflag = reinterpret_cast<uint32_t*>(b + o_flag);
    cudaStream_t st = ctx->stream;
    const int threads = 256;
    const int grid_n = static_cast<int>(std::min<size_t>((N + threads - 1) / threads, 4096));
    const int grid_m = static_cast<int>(std::min<size_t>((m + threads - 1) / threads + 1, 4096));
    const float scale = std::max(1.0f, tether_scale);  // cloth_builder.h:349

    pxb_status s = PXB_OK;
    auto ok = [&](cudaError_t e, const char* what) { return s ? false : !(s = ctx->cuda(e, what)); };
    uint32_t flags[2] = {0, 0};
    std::vector<float> len;
    std::vector<int32_t> src;
    do {
        if (!ok(cudaMemcpyAsync(dp, particles, sizeof(pxb_particle) * N, cudaMemcpyHostToDevice, st), "upload particles"))
            break;
        if (m && !ok(cudaMemcpyAsync(de, stretch, sizeof(pxb_constraint) * m, cudaMemcpyHostToDevice, st),
                     "upload stretch"))
            break;
        if (!ok(cudaMemcpyAsync(da, anchors, sizeof(pxb_anchor) * na, cudaMemcpyHostToDevice, st), "upload anchors"))
            break;
        if (!ok(cudaMemsetAsync(dcur, 0, 4 * (N + 1), st), "zero degrees")) break;
        // adjacency: degrees (into the cursor array), offsets, scatter
        degree_kernel<<<grid_m, threads, 0, st>>>(de, m, dcur);
        scan_kernel<<<1, 1024, 0, st>>>(dcur, n, doff);
        if (!ok(cudaMemcpyAsync(dcur, doff, 4 * (N + 1), cudaMemcpyDeviceToDevice, st), "cursor")) break;
        scatter_kernel<<<grid_m, threads, 0, st>>>(de, m, dcur, dadj);
        seed_kernel<<<grid_n, threads, 0, st>>>(n, dd, dst, danc);
        seed_anchors_kernel<<<std::max(1u, std::min(4096u, (na + threads - 1) / threads)), threads, 0, st>>>(da, na, dd,
                                                                                                            dst, danc);
        ctx->launches += 6;
        if (!ok(cudaGetLastError(), "tether set-up")) break;
        // relaxation rounds: at most n - 1 can still move a distance (Bellman-Ford's bound)
        bool converged = false;
        for (uint32_t round = 0; round <= n && !s; ++round) {
            if (!ok(cudaMemsetAsync(dflag, 0, 4, st), "zero flag")) break;
            relax_kernel<<<grid_n, threads, 0, st>>>(dp, doff, dadj, n, round, dd, dst, dflag);
            ++ctx->launches;
            if (!ok(cudaGetLastError(), "relax")) break;
            if (!ok(cudaMemcpyAsync(flags, dflag, 4, cudaMemcpyDeviceToHost, st), "read flag")) break;
            if (!ok(cudaStreamSynchronize(st), "relax round")) break;
            if (flags[0] == 0) {
                converged = true;
                break;
            }
        }
        if (s) break;
        if (!converged) {
            s = ctx->fail(PXB_ERR_CUDA, "tether distances did not settle");
            break;
        }
        if (!ok(cudaMemsetAsync(dflag, 0, 8, st), "zero flags")) break;
        pred_kernel<<<grid_n, threads, 0, st>>>(dp, doff, dadj, n, dd, danc, dj, dflag + 1);
        ++ctx->launches;
        if (!ok(cudaGetLastError(), "predecessors")) break;
        // pointer jumping: every chain strictly decreases (dist, index), so it ends at an anchor
        converged = false;
        for (int round = 0; round < 64 && !s; ++round) {
            if (!ok(cudaMemsetAsync(dflag, 0, 4, st), "zero flag")) break;
            jump_kernel<<<grid_n, threads, 0, st>>>(n, dj, dflag);
            ++ctx->launches;
            if (!ok(cudaMemcpyAsync(flags, dflag, 8, cudaMemcpyDeviceToHost, st), "read flags")) break;
            if (!ok(cudaStreamSynchronize(st), "jump round")) break;
            if (flags[0] == 0) {
                converged = true;
                break;
            }
        }
        if (s) break;
        if (flags[1] & 1u) {
            s = ctx->fail(PXB_ERR_UNSUPPORTED,
                          "an edge vanishes in its path length (coincident or nearly coincident particles): the "
                          "reference's queue order is not reproducible here; build these tethers on the host");
            break;
        }
        if (!converged || (flags[1] & 2u)) {
            s = ctx->fail(PXB_ERR_CUDA, "tether predecessors are inconsistent");
            break;
        }
        emit_kernel<<<grid_n, threads, 0, st>>>(dp, n, dd, dj, scale, dlen, dsrc);
        ++ctx->launches;
        if (!ok(cudaGetLastError(), "emit")) break;
        len.resize(N);
        src.resize(N);
        if (!ok(cudaMemcpyAsync(len.data(), dlen, 4 * N, cudaMemcpyDeviceToHost, st), "read lengths")) break;
        if (!ok(cudaMemcpyAsync(src.data(), dsrc, 4 * N, cudaMemcpyDeviceToHost, st), "read anchors")) break;
        ok(cudaStreamSynchronize(st), "tethers");
    } while (false);
    cudaStreamSynchronize(st);
    cudaFree(mem);
    if (s) return s;
    if (pxb_status e = ctx->check_device_error()) return e;
    uint32_t count = 0;
    for (uint32_t i = 0; i < n; ++i) count += src[i] >= 0 ? 1u : 0u;
    if (count > capacity || (count && !out)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "output holds %u tethers, %u needed",
                                                              capacity, count);
    uint32_t k = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (src[i] >= 0) out[k++] = pxb_tether{i, static_cast<uint32_t>(src[i]), len[i]};
    *n_out = k;
    return PXB_OK;
}

}  // extern "C"
