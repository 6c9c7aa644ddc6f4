// cloth_kernel.cu -- the launch dispatch of the cloth step (the kernel itself is in
// cloth_step.cuh, its instantiations in cloth_step_*.cu), the whole-GPU path for cloths beyond
// an 8-CTA cluster, and the collider-projection and position-gather kernels.
#include "cloth_step.cuh"

namespace pxb {


// ------------------------------------------------------------------------------------------
// project_particle over a batch of points (the collision primitive on its own)
// ------------------------------------------------------------------------------------------

__global__ void project_points_kernel(const PxbDevCollider* __restrict__ c, float thickness,
                                      const float* __restrict__ pts, const float* __restrict__ starts,
                                      int n, float* __restrict__ out,
                                      float* __restrict__ normals, float* __restrict__ depths,
                                      int32_t* __restrict__ hits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 p = mk(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    f3 nn = mk(0, 0, 0);
    float d = 0.0f;
    const f3 start = starts ? mk(starts[3 * i], starts[3 * i + 1], starts[3 * i + 2]) : p;
    const bool hit = project_particle<true>(c, thickness, p, nn, d, start, starts != nullptr);
    out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
    normals[3 * i] = nn.x; normals[3 * i + 1] = nn.y; normals[3 * i + 2] = nn.z;
    depths[i] = d;
    hits[i] = hit ? 1 : 0;
}

// Positions from layout order to particle order (what a renderer or a state hash reads).
__global__ void gather_positions_kernel(const PxbClothDev* __restrict__ cloths,
                                        const int32_t* __restrict__ order,
                                        const int64_t* __restrict__ out_offsets,
                                        float* __restrict__ out) {
    const PxbClothDev* C = &cloths[__ldg(&order[blockIdx.y])];
    const int cols = C->columns, n = C->n_real, Q = C->Q, S = C->S;
    float* dst = out + __ldg(&out_offsets[blockIdx.y]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / cols, x = i - y * cols;
        const float4 p = C->pos[lay(x, y, Q, S)];
        dst[3 * i] = p.x;
        dst[3 * i + 1] = p.y;
        dst[3 * i + 2] = p.z;
    }
}

cudaError_t launch_gather_positions(const PxbClothDev* cloths, const int32_t* order,
                                    const int64_t* out_offsets, int n_cloths, float* out,
                                    cudaStream_t stream) {
    if (n_cloths <= 0) return cudaSuccess;
    dim3 grid(8, n_cloths);
    gather_positions_kernel<<<grid, 256, 0, stream>>>(cloths, order, out_offsets, out);
    return cudaGetLastError();
}


// ------------------------------------------------------------------------------------------
// Whole-GPU path: one cloth too large for an 8-CTA cluster (e.g. 512 x 512). Every CTA of a
// cooperative launch works on it; positions, rest lengths and lambdas stay in global memory
// (L2-resident at these sizes) and a grid barrier separates colours and stages. Each stage
// evaluates exactly what the shared-memory kernel evaluates, in the same order, so results
// are identical to it and to the reference.
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ unsigned int fkey(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fdecode(unsigned int k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// All CTAs arrive; the last one releases the rest. A wait that runs out (after `polls` polls)
// records the error; from then on no CTA waits at a barrier, so the launch ends after one
// expired wait per CTA (its results are then wrong and the host reports the error word).
// `extra` raises the arrival count a barrier needs (0 in use; a test sets it so that no barrier
// can complete and the expiry path runs).
__device__ __forceinline__ void grid_sync(PxbGridSync* gs, unsigned int& epoch, uint32_t* err, uint32_t polls,
                                          uint32_t extra) {
    __syncthreads();
    if (threadIdx.x == 0) {
        ++epoch;
        __threadfence();
        const unsigned int arrived = atomicAdd(&gs->count, 1u) + 1u;
        if (arrived == epoch * (gridDim.x + extra)) {
            atomicExch(&gs->gen, epoch);
        } else {
            uint32_t spins = 0;
            while (*reinterpret_cast<volatile unsigned int*>(&gs->gen) < epoch) {
                if ((*reinterpret_cast<volatile uint32_t*>(err) & PXB_DEVERR_QUEUE_TIMEOUT) || ++spins > polls) {
                    atomicOr(err, PXB_DEVERR_QUEUE_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int kThreads, bool kExt>
__global__ void __launch_bounds__(kThreads, 1)
cloth_grid_kernel(const PxbClothDev* __restrict__ cloths, const PxbClothStep* __restrict__ stepp,
                  const PxbDevCollider* __restrict__ colliders, const pxb_gravity_source* __restrict__ sources,
                  const int32_t* __restrict__ order, PxbFrameResult* __restrict__ results,
                  uint32_t* __restrict__ err, PxbGridSync* __restrict__ gs, int slot) {
    __shared__ __align__(16) PxbClothDev sC;
    __shared__ PxbClothStep sP;
    __shared__ __align__(16) PxbSeg s_seg[PXB_MAX_SEGS];
    __shared__ float s_red[32][7];
    const int tid = threadIdx.x;
    {
        const int ci = __ldg(&order[slot]);
        const int* srcC = reinterpret_cast<const int*>(&cloths[ci]);
        int* dstC = reinterpret_cast<int*>(&sC);
        for (int i = tid; i < static_cast<int>(sizeof(PxbClothDev) / 4); i += kThreads) dstC[i] = srcC[i];
        const int* srcP = reinterpret_cast<const int*>(&stepp[slot]);
        int* dstP = reinterpret_cast<int*>(&sP);
        for (int i = tid; i < static_cast<int>(sizeof(PxbClothStep) / 4); i += kThreads) dstP[i] = srcP[i];
    }
    __syncthreads();
    {
        const int ns = sC.rank[0].colour_seg[sC.n_colours];
        for (int i = tid; i < ns; i += kThreads) s_seg[i] = sC.segs[sC.rank[0].seg_begin + i];
    }
    const int gt = blockIdx.x * kThreads + tid, GT = gridDim.x * kThreads;
    const int n = sC.n_layout;
    float4* __restrict__ pos = sC.pos;
    float4* __restrict__ gvel = sC.vel;
    float4* __restrict__ gprv = sC.prv;
    const float* rest = sC.rest;
    float* lam = sC.lam_out;
    unsigned int epoch = 0;

    // gravity: uniform, or the source field at the cloth's mean position, summed sequentially
    // in particle order (PhysicsWorld::cloth_centre_ / field_at_, world.h:2048-2076)
    if (blockIdx.x == 0 && tid == 0) {
        float bx = sP.base_accel[0], by = sP.base_accel[1], bz = sP.base_accel[2];
        if (sP.src_count > 0) {
            const int Q = sC.Q, S = sC.S, cols = sC.columns;
            float cx = 0.0f, cy = 0.0f, cz = 0.0f;
            for (int y = 0; y < sC.rows; ++y)
                for (int x = 0; x < cols; ++x) {
                    const float4 p = pos[lay(x, y, Q, S)];
                    cx += p.x; cy += p.y; cz += p.z;
                }
            const float fn = static_cast<float>(sC.n_real);
            const f3 centre = mk(cx / fn, cy / fn, cz / fn);
            float best = 0.0f;
            f3 pull = mk(sP.gravity[0], sP.gravity[1], sP.gravity[2]);
            bool found = false;
            for (int k = 0; k < sP.src_count; ++k) {
                const pxb_gravity_source* g = &sources[sP.src_begin + k];
                const f3 d = sub(ld3(g->centre), centre);
                const float rr = len(d);
                const float range = __ldg(&g->range), radius = __ldg(&g->radius), strength = __ldg(&g->strength);
                if (range > 0.0f && rr > range) continue;
                if (rr < 1e-6f) continue;
                const float a = rr <= radius ? strength : strength * (radius / rr) * (radius / rr);
                if (!found || a > best) {
                    best = a;
                    pull = mul(divs(d, rr), a);
                    found = true;
                }
            }
            const f3 bacc = add(mul(pull, sP.gravity_scale),
                                mk(sP.external_acceleration[0], sP.external_acceleration[1], sP.external_acceleration[2]));
            bx = bacc.x; by = bacc.y; bz = bacc.z;
        }
        gs->base_accel[0] = bx; gs->base_accel[1] = by; gs->base_accel[2] = bz;
        for (int k = 0; k < 3; ++k) {
            gs->keys[k] = 0xFFFFFFFFu;
            gs->keys[3 + k] = 0u;
        }
        gs->keys[6] = 0u;
    }
    grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
    const f3 base_accel = mk(gs->base_accel[0], gs->base_accel[1], gs->base_accel[2]);

    const int steps = sP.steps;
    const int Q = sC.Q, S = sC.S, cols = sC.columns, rows = sC.rows;
    for (int step = 0; step < steps; ++step) {
        const bool aero = sP.aero != 0 && sC.aero_grid != 0;
        // 1. aerodynamics: per-particle gather in ascending triangle order (cloth_solver.h:197-227)
        if (aero) {
            const f3 wind = mk(sP.wind[0], sP.wind[1], sP.wind[2]);
            const float drag = sP.air_drag, lift = sP.air_lift;
            auto P3 = [&](int g) -> f3 { return xyz(pos[g]); };
            auto V3 = [&](int g) -> f3 { return xyz(gvel[g]); };
            for (int gl = gt; gl < n; gl += GT) {
                const int y = gl / S;
                const int j = gl - y * S;
                const int cls = j / Q;
                const int x = 4 * (j - cls * Q) + cls;
                if (x >= cols || y >= rows) continue;
                const bool xm = x >= 1, xp = x + 1 < cols, ym = y >= 1, yp = y + 1 < rows;
                const f3 p00 = P3(gl), v00 = V3(gl);
                f3 a = mk(0.0f, 0.0f, 0.0f);
                if (xm && ym) {
                    const int lmm = lay(x - 1, y - 1, Q, S), l0m = lay(x, y - 1, Q, S), lm0 = lay(x - 1, y, Q, S);
                    tri_share(P3(lmm), P3(l0m), p00, V3(lmm), V3(l0m), v00, wind, drag, lift, a);
                    tri_share(P3(lmm), p00, P3(lm0), V3(lmm), v00, V3(lm0), wind, drag, lift, a);
                }
                if (xp && ym) {
                    const int l0m = lay(x, y - 1, Q, S), lp0 = lay(x + 1, y, Q, S);
                    tri_share(P3(l0m), P3(lp0), p00, V3(l0m), V3(lp0), v00, wind, drag, lift, a);
                }
                if (xm && yp) {
                    const int lm0 = lay(x - 1, y, Q, S), l0p = lay(x, y + 1, Q, S);
                    tri_share(P3(lm0), p00, P3(l0p), V3(lm0), v00, V3(l0p), wind, drag, lift, a);
                }
                if (xp && yp) {
                    const int lp0 = lay(x + 1, y, Q, S), lpp = lay(x + 1, y + 1, Q, S), l0p = lay(x, y + 1, Q, S);
                    tri_share(p00, P3(lp0), P3(lpp), v00, V3(lp0), V3(lpp), wind, drag, lift, a);
                    tri_share(p00, P3(lpp), P3(l0p), v00, V3(lpp), V3(l0p), wind, drag, lift, a);
                }
                gprv[gl] = make_float4(a.x, a.y, a.z, 0.0f);
            }
            grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
        }
        // 4a. lambda reset; 2 + 3. integrate and the anchor lerp (cloth_solver.h:230-254)
        for (int i = gt; i < sC.rank[0].n_lam; i += GT) lam[i] = 0.0f;
        {
            const float alpha_t = static_cast<float>(step + 1) / static_cast<float>(steps);
            const float hs = sP.hs, damping_factor = sP.damping_factor;
            const PxbAnchorRec* anchors = reinterpret_cast<const PxbAnchorRec*>(sC.anchors);
            for (int gl = gt; gl < n; gl += GT) {
                float4 p = pos[gl];
                const f3 acc = aero ? xyz(gprv[gl]) : mk(0.0f, 0.0f, 0.0f);
                gprv[gl] = make_float4(p.x, p.y, p.z, 0.0f);
                if (p.w != 0.0f) {
                    f3 vv = xyz(gvel[gl]);
                    vv = add(vv, mul(add(base_accel, mul(acc, p.w)), hs));
                    vv = mul(vv, damping_factor);
                    p.x = p.x + vv.x * hs;
                    p.y = p.y + vv.y * hs;
                    p.z = p.z + vv.z * hs;
                }
                const int anc = __ldg(&sC.anchor_of[gl]);
                if (anc >= 0) {
                    const PxbAnchorRec& a = anchors[anc];
                    const float om = 1.0f - alpha_t;
                    p.x = a.prev[0] * om + a.world[0] * alpha_t;
                    p.y = a.prev[1] * om + a.world[1] * alpha_t;
                    p.z = a.prev[2] * om + a.world[2] * alpha_t;
                }
                pos[gl] = p;
            }
        }
        grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
        // 4b. colour by colour, a grid barrier after each (cloth_solver.h:256-271)
        {
            const int4* seg4 = reinterpret_cast<const int4*>(s_seg);
            for (int it = 0; it < sP.iters; ++it)
                for (int c = 0; c < sC.n_colours; ++c) {
                    const float alpha = sP.alpha[c];
                    const int se = sC.rank[0].colour_seg[c + 1];
                    for (int sg = sC.rank[0].colour_seg[c]; sg < se; ++sg) {
                        const int4 h0 = seg4[2 * sg], h1 = seg4[2 * sg + 1];
                        int i0 = gt;
                        if (h1.w >= 0)
                            project_segment<1, true, 1>(pos, nullptr, rest + h1.z, lam + h1.w, n, h0, h1, alpha, i0, GT);
                        else
                            project_segment<1, false, 1>(pos, nullptr, rest + h1.z, lam, n, h0, h1, alpha, i0, GT);
                    }
                    grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
                }
        }
        // 5 + 7 + 8. tethers, collisions, velocities (cloth_solver.h:276-451)
        {
            const int col_begin = sP.col_begin, col_count = sP.col_count;
            const float thickness = sP.thickness, inv_hs = sP.inv_hs;
            for (int gl = gt; gl < n; gl += GT) {
                float4 p4 = pos[gl];
                f3 p = xyz(p4);
                bool moved = false;
                f3 nsum = mk(0.0f, 0.0f, 0.0f);
                float dsum = 0.0f;
                if (p4.w != 0.0f) {
                    const int2 teth = __ldg(&sC.tether[gl]);
                    if (teth.x >= 0) {
                        const f3 anchor = xyz(pos[teth.x]);  // a pinned particle: not moved here
                        const f3 d = sub(p, anchor);
                        const float l2 = len(d);
                        const float max_len = __int_as_float(teth.y);
                        if (!(l2 <= max_len || l2 < PXB_EPSILON)) {
                            p = add(anchor, mul(d, max_len / l2));
                            moved = true;
                        }
                    }
                    for (int k = 0; k < col_count; ++k) {
                        const PxbDevCollider* c = &colliders[col_begin + k];
                        if (p.x < __ldg(&c->bmin[0]) - thickness || p.x > __ldg(&c->bmax[0]) + thickness ||
                            p.y < __ldg(&c->bmin[1]) - thickness || p.y > __ldg(&c->bmax[1]) + thickness ||
                            p.z < __ldg(&c->bmin[2]) - thickness || p.z > __ldg(&c->bmax[2]) + thickness) {
                            continue;
                        }
                        f3 nn = mk(0.0f, 0.0f, 0.0f);
                        float depth = 0.0f;
                        const bool mesh = kExt && __ldg(&c->type) == PXB_SHAPE_TRIANGLE_MESH;
                        const f3 start = mesh ? xyz(gprv[gl]) : p;
                        if (!project_particle<kExt>(c, thickness, p, nn, depth, start, mesh)) continue;
                        moved = true;
                        nsum = add(nsum, nn);
                        dsum += depth;
                    }
                }
                if (moved) {
                    p4.x = p.x; p4.y = p.y; p4.z = p.z;
                    pos[gl] = p4;
                }
                const float4 pv = gprv[gl];
                f3 vv = mul(sub(p, xyz(pv)), inv_hs);
                if (dsum > 0.0f) {
                    const float nlen = len(nsum);
                    if (nlen > PXB_EPSILON) {
                        const f3 nrm = divs(nsum, nlen);
                        const float vn = dot(vv, nrm);
                        const f3 vt = sub(vv, smul(vn, nrm));
                        if (vn < 0.0f) vv = sub(vv, smul(vn, nrm));
                        const float budget = sP.friction * dsum * inv_hs;
                        const float vt_len = len(vt);
                        if (vt_len > PXB_EPSILON) vv = sub(vv, mul(vt, minr(1.0f, budget / vt_len)));
                    }
                }
                const float v2 = dot(vv, vv);
                if (v2 > sP.max_velocity2) vv = mul(vv, sP.max_velocity / sqrtf(v2));
                const float real = gvel[gl].w;
                gvel[gl] = make_float4(vv.x, vv.y, vv.z, real);
            }
        }
        grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
    }

    // epilogue: anchors prev <- world, bounds and max speed (order-preserving keys)
    if (blockIdx.x == 0)
        for (int a = tid; a < sC.n_anchors; a += kThreads) {
            PxbAnchorRec* rec = reinterpret_cast<PxbAnchorRec*>(sC.anchors) + a;
            rec->prev[0] = rec->world[0];
            rec->prev[1] = rec->world[1];
            rec->prev[2] = rec->world[2];
        }
    float r[7] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f,
                  -3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f, 0.0f};
    for (int gl = gt; gl < n; gl += GT) {
        const float4 vv = gvel[gl];
        if (vv.w == 0.0f) continue;
        const float4 p = pos[gl];
        r[0] = minr(r[0], p.x); r[1] = minr(r[1], p.y); r[2] = minr(r[2], p.z);
        r[3] = maxr(r[3], p.x); r[4] = maxr(r[4], p.y); r[5] = maxr(r[5], p.z);
        r[6] = maxr(r[6], dot(xyz(vv), xyz(vv)));
    }
    r[0] = warp_min(r[0]); r[1] = warp_min(r[1]); r[2] = warp_min(r[2]);
    r[3] = warp_max(r[3]); r[4] = warp_max(r[4]); r[5] = warp_max(r[5]); r[6] = warp_max(r[6]);
    if ((tid & 31) == 0)
        for (int k = 0; k < 7; ++k) s_red[tid >> 5][k] = r[k];
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
            for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], s_red[w][k]);
            for (int k = 3; k < 7; ++k) r[k] = fmaxf(r[k], s_red[w][k]);
        }
        for (int k = 0; k < 3; ++k) atomicMin(&gs->keys[k], fkey(r[k]));
        for (int k = 3; k < 7; ++k) atomicMax(&gs->keys[k], fkey(r[k]));
    }
    grid_sync(gs, epoch, err, sP.grid_wait_polls, sP.grid_extra_arrivals);
    if (blockIdx.x == 0 && tid == 0) {
        PxbFrameResult* out = &results[slot];
        for (int k = 0; k < 3; ++k) {
            out->bounds_min[k] = fdecode(gs->keys[k]);
            out->bounds_max[k] = fdecode(gs->keys[3 + k]);
        }
        out->max_speed = sqrtf(fdecode(gs->keys[6]));
        out->time = 0.0f;
    }
}

template <bool kExt>
static cudaError_t launch_grid_variant(const PxbClothDev* cloths, const PxbClothStep* steps,
                                       const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                                       const int32_t* order, PxbFrameResult* results, uint32_t* err,
                                       PxbGridSync* gs, int slot, int n_sms, cudaStream_t stream) {
    constexpr int kThreads = 1024;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cloth_grid_kernel<kThreads, kExt>, kThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    unsigned int blocks = static_cast<unsigned int>(n_sms);  // one CTA per SM: every one co-resident
    void* args[] = {(void*)&cloths, (void*)&steps, (void*)&colliders, (void*)&sources, (void*)&order,
                    (void*)&results, (void*)&err, (void*)&gs, (void*)&slot};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(cloth_grid_kernel<kThreads, kExt>), dim3(blocks),
                                       dim3(kThreads), args, 0, stream);
}

cudaError_t launch_cloth_grid(const PxbClothDev* cloths, const PxbClothStep* steps, const PxbDevCollider* colliders,
                              const pxb_gravity_source* sources, const int32_t* order, PxbFrameResult* results,
                              uint32_t* err, PxbGridSync* gs, int slot, int n_sms, cudaStream_t stream, bool geo) {
    return geo ? launch_grid_variant<true>(cloths, steps, colliders, sources, order, results, err, gs, slot, n_sms, stream)
               : launch_grid_variant<false>(cloths, steps, colliders, sources, order, results, err, gs, slot, n_sms, stream);
}

int cloth_variant_threads(int variant) {
    return variant == 0 ? 512 : (variant == 1 ? 768 : 1024);
}

cudaError_t launch_cloth_step(int variant, int cluster, const PxbClothDev* cloths,
                              const PxbClothStep* steps, const PxbDevCollider* colliders,
                              const pxb_gravity_source* sources, const int32_t* order,
                              PxbFrameResult* results, uint32_t* err, int n_cloths, int threads,
                              int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int ext, int* queue, int persistent_units) {
    if (n_cloths <= 0) return cudaSuccess;
    if (ext == 5 || ext == 6) return launch_cloth_soa(ext == 6, variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    if (ext == 3 || ext == 4) return launch_cloth_lean(ext == 4, variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    if (ext == 2) return launch_cloth_gmem(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    if (ext) return launch_cloth_geo(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    if (wsteps) return launch_cloth_warm(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    return launch_cloth_plain(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
}

cudaError_t launch_project_points(const PxbDevCollider* collider, float thickness, const float* pts,
                                  const float* starts, int n, float* out, float* normals, float* depths,
                                  int32_t* hits, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int tb = 256;
    project_points_kernel<<<(n + tb - 1) / tb, tb, 0, stream>>>(collider, thickness, pts, starts, n, out,
                                                                 normals, depths, hits);
    return cudaGetLastError();
}

}  // namespace pxb
