// strand_kernel.cu -- the XPBD hair-strand substep on sm_100a: one warp per strand, one lane
// per particle, the whole strand in registers.
//
// Replaces hair::solve_strands (physxcoopa/hair/strand_solver.h:121-327) for sets built by
// make_strands (strand_builder.h:58-127). Per warp and substep:
//   1+2 integrate with air drag and the speed clamp          (lane = particle)
//   3   root lerp                                             (lane 0)
//   4   stretch, even then odd constraints, `iterations` times: both lanes of a constraint fetch
//       the other endpoint with a shuffle and evaluate the same projection, each keeping its own
//       endpoint -- bit-identical on both sides, so nothing is written back
//   5   global shape toward the root-frame rest pose          (lane = particle)
//   6   local shape, the reference's serial chain k = 1..n-2: one thread walks each strand of
//       the block over positions gathered in shared memory
//   7   collider projection keeping the deepest contact       (lane = particle)
//   8   velocities + positional friction                      (lane = particle)
// Bounds and the largest speed of the whole set are reduced with warp shuffles and combined
// across warps with integer atomics on an order-preserving float encoding (exact, order-free).
//
// Arithmetic follows the reference's operation order in IEEE single precision without
// contraction. The transcendental calls (sin / acos / cos in the wind gust, slerp and the
// local-shape rotation) use CUDA's libm, which can differ from the host's by an ulp.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"
#include "pxb_kernels.h"
#include "pxb_device_math.cuh"

namespace pxb {
namespace {

constexpr int kWarpsPerBlock = 32;

struct q4 {
    float x, y, z, w;
};
__device__ __forceinline__ q4 mkq(float w, float x, float y, float z) { return q4{x, y, z, w}; }

// Unit-quaternion rotation v + 2*(w*(u x v) + u x (u x v)).
__device__ __forceinline__ f3 qrot(q4 q, f3 v) {
    const f3 u = mk(q.x, q.y, q.z);
    const f3 uv = cross(u, v);
    const f3 uuv = cross(u, uv);
    return add(v, mul(add(mul(uv, q.w), uuv), 2.0f));
}
__device__ __forceinline__ float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
__device__ __forceinline__ f3 mixv(f3 x, f3 y, float a) { return add(mul(x, 1.0f - a), mul(y, a)); }

// Shortest-arc slerp with the component-wise lerp when cos(theta) > 1 - FLT_EPSILON.
__device__ q4 slerp(q4 a, q4 b, float t) {
    float c = a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    if (c < 0.0f) {
        b = mkq(-b.w, -b.x, -b.y, -b.z);
        c = -c;
    }
    if (c > 1.0f - 1.19209290e-07f)
        return mkq(mixf(a.w, b.w, t), mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t));
    const float theta = acosf(c);
    const float sa = sinf((1.0f - t) * theta), sb = sinf(t * theta), sn = sinf(theta);
    return mkq((sa * a.w + sb * b.w) / sn, (sa * a.x + sb * b.x) / sn, (sa * a.y + sb * b.y) / sn,
               (sa * a.z + sb * b.z) / sn);
}
__device__ __forceinline__ q4 angle_axis(float angle, f3 axis) {
    const float s = sinf(angle * 0.5f);
    return mkq(cosf(angle * 0.5f), axis.x * s, axis.y * s, axis.z * s);
}
// hair::detail::rotation_between (strand_solver.h:91-105).
__device__ q4 rotation_between(f3 from, f3 to) {
    const float d = minr(maxr(dot(from, to), -1.0f), 1.0f);
    if (d > 0.999999f) return mkq(1.0f, 0.0f, 0.0f, 0.0f);
    if (d < -0.999999f) {
        f3 axis = cross(mk(0.0f, 0.0f, 1.0f), from);
        if (dot(axis, axis) < 1e-8f) axis = cross(mk(1.0f, 0.0f, 0.0f), from);
        return angle_axis(3.14159265358979323846f, mul(axis, 1.0f / sqrtf(dot(axis, axis))));
    }
    const f3 axis = cross(from, to);
    const float l = len(axis);
    if (l < 1e-8f) return mkq(1.0f, 0.0f, 0.0f, 0.0f);
    return angle_axis(acosf(d), divs(axis, l));
}

__device__ __forceinline__ f3 shfl3(f3 v, int src) {
    return mk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
              __shfl_sync(0xffffffffu, v.z, src));
}

// Order-preserving int encoding of a float for atomicMin / atomicMax.
__device__ __forceinline__ int fkey(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}

}  // namespace

template <bool kGeo>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
strand_step_kernel(PxbStrandDev D, PxbStrandStep P, const PxbDevCollider* __restrict__ colliders,
                   const pxb_gravity_source* __restrict__ sources) {
    // local-shape chains run one thread per strand over this block's strands (shared memory)
    __shared__ float4 s_chain[kWarpsPerBlock][32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int strand_raw = blockIdx.x * kWarpsPerBlock + warp;
    // warps past the last strand stay (with no particles) for the block-wide barriers
    const bool valid = strand_raw < D.n_strands;
    const int strand = valid ? strand_raw : 0;
    const int count = valid ? __ldg(&D.count[strand]) : 0;
    const int slot = strand * 32 + lane;
    const bool live = lane < count;

    // --- gravity: uniform, or the source field at the set's last bounds centre (world.h:1941) --
    f3 accel = mk(P.accel[0], P.accel[1], P.accel[2]);
    if (P.src_count > 0) {
        const float* b = D.bounds_prev;
        const f3 bmin = mk(b[0], b[1], b[2]), bmax = mk(b[3], b[4], b[5]);
        const f3 centre = smul(0.5f, add(bmin, bmax));
        float best = 0.0f;
        f3 pull = mk(P.gravity[0], P.gravity[1], P.gravity[2]);
        bool found = false;
        for (int k = 0; k < P.src_count; ++k) {
            const pxb_gravity_source* g = &sources[P.src_begin + k];
            const f3 d = sub(ld3(g->centre), centre);
            const float r = len(d);
            const float range = __ldg(&g->range), radius = __ldg(&g->radius), strength = __ldg(&g->strength);
            if (range > 0.0f && r > range) continue;
            if (r < 1e-6f) continue;
            const float a = r <= radius ? strength : strength * (radius / r) * (radius / r);
            if (!found || a > best) {
                best = a;
                pull = mul(divs(d, r), a);
                found = true;
            }
        }
        accel = add(mul(pull, P.gravity_scale), mk(P.external_acceleration[0], P.external_acceleration[1],
                                                   P.external_acceleration[2]));
    }

    float4 p4 = live ? D.pos[slot] : make_float4(0, 0, 0, 0);
    f3 p = xyz(p4);
    const float w = p4.w;
    f3 v = live ? xyz(D.vel[slot]) : mk(0, 0, 0);
    f3 prev = live ? xyz(D.prv[slot]) : mk(0, 0, 0);
    const f3 rest_local = live ? xyz(D.rest_local[slot]) : mk(0, 0, 0);
    const float rest_next = live ? __ldg(&D.rest[slot]) : 0.0f;   // constraint (lane, lane + 1)
    const float wshape = live ? __ldg(&D.wshape[slot]) : 0.0f;     // pow(1 - along, falloff)
    const float* rr = D.roots + 16 * static_cast<size_t>(strand);
    const f3 root_pos = mk(__ldg(rr + 0), __ldg(rr + 1), __ldg(rr + 2));
    const q4 root_q = q4{__ldg(rr + 3), __ldg(rr + 4), __ldg(rr + 5), __ldg(rr + 6)};
    const f3 prev_root_pos = mk(__ldg(rr + 8), __ldg(rr + 9), __ldg(rr + 10));
    const q4 prev_root_q = q4{__ldg(rr + 11), __ldg(rr + 12), __ldg(rr + 13), __ldg(rr + 14)};
    float lam = 0.0f;
    float time = P.time;
    const f3 wind0 = mk(P.wind[0], P.wind[1], P.wind[2]);

    for (int step = 0; step < P.steps; ++step) {
        const float t = static_cast<float>(step + 1) / static_cast<float>(P.steps);
        // --- 1 + 2: aerodynamics and integration (strand_solver.h:162-189) --------------
        if (live && w > 0.0f) {
            f3 a = accel;
            if (P.air_drag > 0.0f) {
                f3 wind = wind0;
                if (P.wind_turbulence > 0.0f) {
                    const float phase = time * 2.3f + p.x * 1.7f + p.y * 2.1f + p.z * 1.3f;
                    const f3 gust = mk(sinf(phase), sinf(phase * 1.37f + 2.1f), sinf(phase * 0.81f + 4.2f));
                    wind = add(wind, smul(P.turbulence_amp, gust));
                }
                a = add(a, mul(sub(wind, v), P.air_drag));
            }
            v = add(v, mul(a, P.hs));
            v = mul(v, P.damping_factor);
            const float v2 = dot(v, v);
            if (v2 > P.max_speed2) v = mul(v, P.max_velocity / sqrtf(v2));
            prev = p;
            p = add(p, mul(v, P.hs));
        }
        // --- 3: roots (strand_solver.h:194-201) ------------------------------------------
        if (lane == 0 && count > 0) {
            prev = p;
            p = mixv(prev_root_pos, root_pos, t);
            v = mk(0.0f, 0.0f, 0.0f);
        }
        // --- 4: stretch, even then odd batch (strand_solver.h:204-211) ---------------------
        lam = 0.0f;
        for (int it = 0; it < P.iters; ++it) {
            for (int parity = 0; parity < 2; ++parity) {
                // Lane k is endpoint `a` of constraint k (k -> k+1) when k has this parity, and
                // endpoint `b` of constraint k-1 when k-1 has it.
                const bool is_a = live && lane + 1 < count && (lane & 1) == parity;
                const bool is_b = live && lane >= 1 && ((lane - 1) & 1) == parity;
                const f3 up = shfl3(p, min(lane + 1, 31));
                const float w_up = __shfl_sync(0xffffffffu, w, min(lane + 1, 31));
                const f3 dn = shfl3(p, max(lane - 1, 0));
                const float w_dn = __shfl_sync(0xffffffffu, w, max(lane - 1, 0));
                const float rest_dn = __shfl_sync(0xffffffffu, rest_next, max(lane - 1, 0));
                const float lam_dn = __shfl_sync(0xffffffffu, lam, max(lane - 1, 0));
                float4 pa, pb;
                float rest, lam_c;
                if (is_a) {
                    pa = make_float4(p.x, p.y, p.z, w);
                    pb = make_float4(up.x, up.y, up.z, w_up);
                    rest = rest_next;
                    lam_c = lam;
                } else {
                    pa = make_float4(dn.x, dn.y, dn.z, w_dn);
                    pb = make_float4(p.x, p.y, p.z, w);
                    rest = rest_dn;
                    lam_c = lam_dn;
                }
                float dl = 0.0f;
                if ((is_a || is_b) && solve_pair(pa, pb, rest, lam_c, P.alpha, dl)) {
                    if (is_a) {
                        p = xyz(pa);
                        lam = lam_c + dl;
                    } else {
                        p = xyz(pb);
                    }
                }
            }
        }
        // --- 5: global shape (strand_solver.h:216-235) -----------------------------------
        if (P.global_shape_on && count >= 2) {
            const q4 orientation = slerp(prev_root_q, root_q, t);
            const f3 root = mixv(prev_root_pos, root_pos, t);
            if (live && lane >= 1 && w > 0.0f) {
                const float weight = P.global_per_substep * wshape;
                if (weight > 0.0f) {
                    const f3 target = add(root, qrot(orientation, rest_local));
                    p = mixv(p, target, minr(weight, 1.0f));
                }
            }
        }
        // --- 6: local shape, the serial chain (strand_solver.h:241-272) -------------------
        // Serial along a strand: one thread walks each strand of the block (instead of a whole
        // warp computing the same chain redundantly), on the block's positions in shared memory.
        if (P.local_shape_on) {
            s_chain[warp][lane] = make_float4(p.x, p.y, p.z, w);
            __syncthreads();
            if (threadIdx.x < kWarpsPerBlock) {
                const int ws_ = threadIdx.x;
                const int sg = blockIdx.x * kWarpsPerBlock + ws_;
                const int cnt = sg < D.n_strands ? __ldg(&D.count[sg]) : 0;
                float4* sp = s_chain[ws_];
                const float4* ro = D.rest_offset + static_cast<size_t>(sg) * 32;
                for (int k = 1; k + 1 < cnt; ++k) {
                    const float4 qp = sp[k - 1], qc = sp[k], qn = sp[k + 1];
                    const f3 pp = xyz(qp), pc = xyz(qc), pn = xyz(qn);
                    const f3 ro_c = xyz(__ldg(&ro[k])), ro_n = xyz(__ldg(&ro[k + 1]));
                    const float wc = qc.w, wn = qn.w;
                    const f3 live_prev = sub(pc, pp);
                    const float rest_len = len(ro_c);
                    const float live_len = len(live_prev);
                    if (rest_len <= 1e-8f || live_len <= 1e-8f) continue;
                    const q4 turn = rotation_between(divs(ro_c, rest_len), divs(live_prev, live_len));
                    const f3 target = add(pc, qrot(turn, ro_n));
                    const f3 delta = mul(sub(target, pn), P.local_per_substep);
                    const float wsum = wc + wn;
                    if (wsum <= 0.0f) continue;
                    const f3 nn = add(pn, mul(delta, wn / wsum));
                    const f3 nc = sub(pc, mul(delta, wc / wsum));
                    sp[k + 1] = make_float4(nn.x, nn.y, nn.z, wn);
                    sp[k] = make_float4(nc.x, nc.y, nc.z, wc);
                }
            }
            __syncthreads();
            p = xyz(s_chain[warp][lane]);
        }
        // --- 7: collisions, deepest contact kept (strand_solver.h:275-298) ---------------
        bool contacted = false;
        f3 cn = mk(0.0f, 0.0f, 0.0f);
        float cd = 0.0f;
        if (live && w > 0.0f) {
            for (int k = 0; k < P.col_count; ++k) {
                f3 n = mk(0.0f, 0.0f, 0.0f);
                float depth = 0.0f;
                // a mesh's swept test starts from the substep's start (strand_solver.h:283-284)
                const PxbDevCollider* c = &colliders[P.col_begin + k];
                const bool mesh = kGeo && __ldg(&c->type) == PXB_SHAPE_TRIANGLE_MESH;
                if (!project_particle<kGeo>(c, P.thickness, p, n, depth, prev, mesh)) continue;
                if (!contacted || depth > cd) {
                    cn = n;
                    cd = depth;
                }
                contacted = true;
            }
        }
        // --- 8: finalize + positional friction (strand_solver.h:301-321) ----------------
        if (live && w > 0.0f) {
            v = mul(sub(p, prev), P.inv_hs);
            if (contacted && P.friction > 0.0f) {
                const f3 motion = sub(p, prev);
                const f3 tangential = sub(motion, mul(cn, dot(motion, cn)));
                const float t_len = len(tangential);
                if (t_len > PXB_EPSILON) {
                    const float limit = P.friction * cd;
                    const float scale = maxr(0.0f, 1.0f - minr(limit, t_len) / t_len);
                    p = sub(p, mul(tangential, 1.0f - scale));
                    v = mul(sub(p, prev), P.inv_hs);
                }
            }
        }
        time = time + P.hs;
    }

    if (live) {
        D.pos[slot] = make_float4(p.x, p.y, p.z, w);
        D.vel[slot] = make_float4(v.x, v.y, v.z, 0.0f);
        D.prv[slot] = make_float4(prev.x, prev.y, prev.z, 0.0f);
        D.lam[slot] = lam;
    }
    // --- set bounds and largest speed (strand.h:195-211) ---------------------------------
    float r[7];
    r[0] = live ? p.x : 3.402823466e+38f;
    r[1] = live ? p.y : 3.402823466e+38f;
    r[2] = live ? p.z : 3.402823466e+38f;
    r[3] = live ? p.x : -3.402823466e+38f;
    r[4] = live ? p.y : -3.402823466e+38f;
    r[5] = live ? p.z : -3.402823466e+38f;
    r[6] = live ? dot(v, v) : 0.0f;
    for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], __shfl_xor_sync(0xffffffffu, r[k], o));
        for (int k = 3; k < 7; ++k) r[k] = fmaxf(r[k], __shfl_xor_sync(0xffffffffu, r[k], o));
    }
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) atomicMin(&D.bounds_next[k], fkey(r[k]));
        for (int k = 3; k < 7; ++k) atomicMax(&D.bounds_next[k], fkey(r[k]));
    }
}

// Strands of any length (a set with one longer than 32 particles): one warp per strand, lane j
// taking particles j, j + 32, ...; the strand's positions and lambdas in shared memory, its
// velocities and substep-start positions in the set's HBM arrays (only the particle's owner lane
// touches them). The same stages, in the same order and arithmetic, as strand_step_kernel; the
// stretch batches run constraint c = parity + 2m on lane m % 32 with a warp barrier between
// parities, and the local-shape chain is walked by lane 0. No block-wide barrier: each warp only
// waits for its own lanes, so a warp past the last strand simply leaves.
template <bool kGeo>
__global__ void __launch_bounds__(256)
strand_long_kernel(PxbStrandDev D, PxbStrandStep P, const PxbDevCollider* __restrict__ colliders,
                   const pxb_gravity_source* __restrict__ sources) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    const int pad = D.pad_count;
    float4* sp = reinterpret_cast<float4*>(smem) + static_cast<size_t>(warp) * pad;
    float* sl = reinterpret_cast<float*>(reinterpret_cast<float4*>(smem) + static_cast<size_t>(W) * pad) +
                static_cast<size_t>(warp) * pad;
    const int strand = blockIdx.x * W + warp;
    if (strand >= D.n_strands) return;
    const int count = __ldg(&D.count[strand]);
    const int base = __ldg(&D.base[strand]);
    if (count > pad) return;  // the host sizes pad_count for the longest strand

    // --- gravity: uniform, or the source field at the set's last bounds centre (world.h:1941) --
    f3 accel = mk(P.accel[0], P.accel[1], P.accel[2]);
    if (P.src_count > 0) {
        const float* b = D.bounds_prev;
        const f3 bmin = mk(b[0], b[1], b[2]), bmax = mk(b[3], b[4], b[5]);
        const f3 centre = smul(0.5f, add(bmin, bmax));
        float best = 0.0f;
        f3 pull = mk(P.gravity[0], P.gravity[1], P.gravity[2]);
        bool found = false;
        for (int k = 0; k < P.src_count; ++k) {
            const pxb_gravity_source* g = &sources[P.src_begin + k];
            const f3 d = sub(ld3(g->centre), centre);
            const float r = len(d);
            const float range = __ldg(&g->range), radius = __ldg(&g->radius), strength = __ldg(&g->strength);
            if (range > 0.0f && r > range) continue;
            if (r < 1e-6f) continue;
            const float a = r <= radius ? strength : strength * (radius / r) * (radius / r);
            if (!found || a > best) {
                best = a;
                pull = mul(divs(d, r), a);
                found = true;
            }
        }
        accel = add(mul(pull, P.gravity_scale), mk(P.external_acceleration[0], P.external_acceleration[1],
                                                   P.external_acceleration[2]));
    }
    for (int k = lane; k < count; k += 32) sp[k] = D.pos[base + k];
    const float* rr = D.roots + 16 * static_cast<size_t>(strand);
    const f3 root_pos = mk(__ldg(rr + 0), __ldg(rr + 1), __ldg(rr + 2));
    const q4 root_q = q4{__ldg(rr + 3), __ldg(rr + 4), __ldg(rr + 5), __ldg(rr + 6)};
    const f3 prev_root_pos = mk(__ldg(rr + 8), __ldg(rr + 9), __ldg(rr + 10));
    const q4 prev_root_q = q4{__ldg(rr + 11), __ldg(rr + 12), __ldg(rr + 13), __ldg(rr + 14)};
    float time = P.time;
    const f3 wind0 = mk(P.wind[0], P.wind[1], P.wind[2]);
    __syncwarp();

    for (int step = 0; step < P.steps; ++step) {
        const float t = static_cast<float>(step + 1) / static_cast<float>(P.steps);
        // --- 1 + 2: aerodynamics and integration (strand_solver.h:162-189) --------------
        for (int k = lane; k < count; k += 32) {
            const float4 p4 = sp[k];
            if (!(p4.w > 0.0f)) continue;
            f3 p = xyz(p4);
            f3 v = xyz(D.vel[base + k]);
            f3 a = accel;
            if (P.air_drag > 0.0f) {
                f3 wind = wind0;
                if (P.wind_turbulence > 0.0f) {
                    const float phase = time * 2.3f + p.x * 1.7f + p.y * 2.1f + p.z * 1.3f;
                    const f3 gust = mk(sinf(phase), sinf(phase * 1.37f + 2.1f), sinf(phase * 0.81f + 4.2f));
                    wind = add(wind, smul(P.turbulence_amp, gust));
                }
                a = add(a, mul(sub(wind, v), P.air_drag));
            }
            v = add(v, mul(a, P.hs));
            v = mul(v, P.damping_factor);
            const float v2 = dot(v, v);
            if (v2 > P.max_speed2) v = mul(v, P.max_velocity / sqrtf(v2));
            D.prv[base + k] = make_float4(p.x, p.y, p.z, 0.0f);
            p = add(p, mul(v, P.hs));
            D.vel[base + k] = make_float4(v.x, v.y, v.z, 0.0f);
            sp[k] = make_float4(p.x, p.y, p.z, p4.w);
        }
        // --- 3: roots (strand_solver.h:194-201) ------------------------------------------
        if (lane == 0 && count > 0) {
            const float4 p4 = sp[0];
            D.prv[base] = make_float4(p4.x, p4.y, p4.z, 0.0f);
            const f3 r = mixv(prev_root_pos, root_pos, t);
            sp[0] = make_float4(r.x, r.y, r.z, p4.w);
            D.vel[base] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        // --- 4: stretch, even then odd batch (strand_solver.h:204-211) ---------------------
        for (int c = lane; c + 1 < count; c += 32) sl[c] = 0.0f;
        __syncwarp();
        for (int it = 0; it < P.iters; ++it) {
            for (int parity = 0; parity < 2; ++parity) {
                for (int c = parity + 2 * lane; c + 1 < count; c += 64) {
                    float4 pa = sp[c], pb = sp[c + 1];
                    const float lam_c = sl[c];
                    float dl = 0.0f;
                    if (solve_pair(pa, pb, __ldg(&D.rest[base + c]), lam_c, P.alpha, dl)) {
                        sp[c] = pa;
                        sp[c + 1] = pb;
                        sl[c] = lam_c + dl;
                    }
                }
                __syncwarp();
            }
        }
        // --- 5: global shape (strand_solver.h:216-235) -----------------------------------
        if (P.global_shape_on && count >= 2) {
            const q4 orientation = slerp(prev_root_q, root_q, t);
            const f3 root = mixv(prev_root_pos, root_pos, t);
            for (int k = lane; k < count; k += 32) {
                const float4 p4 = sp[k];
                if (k < 1 || !(p4.w > 0.0f)) continue;
                const float weight = P.global_per_substep * __ldg(&D.wshape[base + k]);
                if (weight > 0.0f) {
                    const f3 target = add(root, qrot(orientation, xyz(D.rest_local[base + k])));
                    const f3 p = mixv(xyz(p4), target, minr(weight, 1.0f));
                    sp[k] = make_float4(p.x, p.y, p.z, p4.w);
                }
            }
            __syncwarp();
        }
        // --- 6: local shape, the serial chain (strand_solver.h:241-272), by lane 0 ----------
        if (P.local_shape_on) {
            if (lane == 0) {
                const float4* ro = D.rest_offset + base;
                for (int k = 1; k + 1 < count; ++k) {
                    const float4 qp = sp[k - 1], qc = sp[k], qn = sp[k + 1];
                    const f3 pp = xyz(qp), pc = xyz(qc), pn = xyz(qn);
                    const f3 ro_c = xyz(__ldg(&ro[k])), ro_n = xyz(__ldg(&ro[k + 1]));
                    const float wc = qc.w, wn = qn.w;
                    const f3 live_prev = sub(pc, pp);
                    const float rest_len = len(ro_c);
                    const float live_len = len(live_prev);
                    if (rest_len <= 1e-8f || live_len <= 1e-8f) continue;
                    const q4 turn = rotation_between(divs(ro_c, rest_len), divs(live_prev, live_len));
                    const f3 target = add(pc, qrot(turn, ro_n));
                    const f3 delta = mul(sub(target, pn), P.local_per_substep);
                    const float wsum = wc + wn;
                    if (wsum <= 0.0f) continue;
                    const f3 nn = add(pn, mul(delta, wn / wsum));
                    const f3 nc = sub(pc, mul(delta, wc / wsum));
                    sp[k + 1] = make_float4(nn.x, nn.y, nn.z, wn);
                    sp[k] = make_float4(nc.x, nc.y, nc.z, wc);
                }
            }
            __syncwarp();
        }
        // --- 7 + 8: collisions (deepest contact kept), velocities, positional friction -----
        for (int k = lane; k < count; k += 32) {
            const float4 p4 = sp[k];
            if (!(p4.w > 0.0f)) continue;
            f3 p = xyz(p4);
            const f3 prev = xyz(D.prv[base + k]);
            bool contacted = false;
            f3 cn = mk(0.0f, 0.0f, 0.0f);
            float cd = 0.0f;
            for (int q = 0; q < P.col_count; ++q) {
                f3 n = mk(0.0f, 0.0f, 0.0f);
                float depth = 0.0f;
                const PxbDevCollider* c = &colliders[P.col_begin + q];
                const bool mesh = kGeo && __ldg(&c->type) == PXB_SHAPE_TRIANGLE_MESH;
                if (!project_particle<kGeo>(c, P.thickness, p, n, depth, prev, mesh)) continue;
                if (!contacted || depth > cd) {
                    cn = n;
                    cd = depth;
                }
                contacted = true;
            }
            f3 v = mul(sub(p, prev), P.inv_hs);
            if (contacted && P.friction > 0.0f) {
                const f3 motion = sub(p, prev);
                const f3 tangential = sub(motion, mul(cn, dot(motion, cn)));
                const float t_len = len(tangential);
                if (t_len > PXB_EPSILON) {
                    const float limit = P.friction * cd;
                    const float scale = maxr(0.0f, 1.0f - minr(limit, t_len) / t_len);
                    p = sub(p, mul(tangential, 1.0f - scale));
                    v = mul(sub(p, prev), P.inv_hs);
                }
            }
            D.vel[base + k] = make_float4(v.x, v.y, v.z, 0.0f);
            sp[k] = make_float4(p.x, p.y, p.z, p4.w);
        }
        __syncwarp();
        time = time + P.hs;
    }

    float r[7] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f,
                  -3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f, 0.0f};
    for (int k = lane; k < count; k += 32) {
        const float4 p = sp[k];
        D.pos[base + k] = p;
        if (k + 1 < count) D.lam[base + k] = sl[k];
        const f3 v = xyz(D.vel[base + k]);
        r[0] = fminf(r[0], p.x); r[1] = fminf(r[1], p.y); r[2] = fminf(r[2], p.z);
        r[3] = fmaxf(r[3], p.x); r[4] = fmaxf(r[4], p.y); r[5] = fmaxf(r[5], p.z);
        r[6] = fmaxf(r[6], dot(v, v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], __shfl_xor_sync(0xffffffffu, r[k], o));
        for (int k = 3; k < 7; ++k) r[k] = fmaxf(r[k], __shfl_xor_sync(0xffffffffu, r[k], o));
    }
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) atomicMin(&D.bounds_next[k], fkey(r[k]));
        for (int k = 3; k < 7; ++k) atomicMax(&D.bounds_next[k], fkey(r[k]));
    }
}

// Sets the 7 reduction keys of a bounds buffer to their identities.
__global__ void strand_bounds_reset_kernel(int* keys) {
    const int k = threadIdx.x;
    if (k < 3) keys[k] = fkey(3.402823466e+38f);
    else if (k < 6) keys[k] = fkey(-3.402823466e+38f);
    else if (k == 6) keys[k] = fkey(0.0f);
}

// Decodes a bounds buffer's keys into floats (min xyz, max xyz, max speed^2).
__global__ void strand_bounds_decode_kernel(const int* keys, float* out) {
    const int k = threadIdx.x;
    if (k < 7) {
        const int i = keys[k];
        out[k] = __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
    }
}

cudaError_t launch_strand_step(const PxbStrandDev& d, const PxbStrandStep& p,
                               const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                               cudaStream_t stream, bool geo) {
    strand_bounds_reset_kernel<<<1, 32, 0, stream>>>(d.bounds_next);
    if (d.long_mode) {
        static uint64_t configured = 0;  // one bit per device the attribute has been set on
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 64 && !(configured >> dev & 1ull)) {
            for (cudaError_t a : {cudaFuncSetAttribute(strand_long_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448 - 1024),
                                  cudaFuncSetAttribute(strand_long_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448 - 1024)})
                if (a != cudaSuccess) return a;
            configured |= 1ull << dev;
        }
        const int W = d.warps;
        const int blocks = (d.n_strands + W - 1) / W;
        const size_t smem = static_cast<size_t>(W) * d.pad_count * 20;
        if (blocks > 0) {
            if (geo)
                strand_long_kernel<true><<<blocks, 32 * W, smem, stream>>>(d, p, colliders, sources);
            else
                strand_long_kernel<false><<<blocks, 32 * W, smem, stream>>>(d, p, colliders, sources);
        }
        strand_bounds_decode_kernel<<<1, 32, 0, stream>>>(d.bounds_next, d.bounds_out);
        return cudaGetLastError();
    }
    const int blocks = (d.n_strands + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > 0) {
        if (geo)
            strand_step_kernel<true><<<blocks, kWarpsPerBlock * 32, 0, stream>>>(d, p, colliders, sources);
        else
            strand_step_kernel<false><<<blocks, kWarpsPerBlock * 32, 0, stream>>>(d, p, colliders, sources);
    }
    strand_bounds_decode_kernel<<<1, 32, 0, stream>>>(d.bounds_next, d.bounds_out);
    return cudaGetLastError();
}

}  // namespace pxb
