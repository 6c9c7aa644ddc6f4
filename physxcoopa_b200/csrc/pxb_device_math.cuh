// pxb_device_math.cuh -- device helpers shared by the cloth and strand kernels: single-
// precision vector arithmetic in the reference's operation order, the particle-vs-collider
// projection (cloth::project_particle, physxcoopa/cloth/cloth_collision.h:109-420) over a host-
// precomputed collider snapshot, and one XPBD distance projection
// (cloth::detail::project_distance, physxcoopa/cloth/cloth_solver.h:119-138).
#ifndef PXB_DEVICE_MATH_CUH
#define PXB_DEVICE_MATH_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"

namespace pxb {
namespace {

// ------------------------------------------------------------------------------------------
// Vector helpers, single precision, reference operation order
// ------------------------------------------------------------------------------------------

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 mul(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 smul(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ f3 divs(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }
__device__ __forceinline__ f3 ld3(const float* p) { return mk(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }
__device__ __forceinline__ float minr(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float maxr(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float clamp01(float t) { return t < 0.0f ? 0.0f : (1.0f < t ? 1.0f : t); }

// ------------------------------------------------------------------------------------------
// Collision: cloth::project_particle (cloth_collision.h:386-420) over a precomputed snapshot
// ------------------------------------------------------------------------------------------

// geometry::closest_point_on_segment (capsule.h:39-49).
__device__ __forceinline__ f3 closest_on_segment(f3 point, f3 a, f3 b) {
    const f3 ab = sub(b, a);
    const float len2 = dot(ab, ab);
    if (len2 < PXB_EPSILON) return a;
    const float t = clamp01(dot(sub(point, a), ab) / len2);
    return add(a, mul(ab, t));
}

// cloth::detail::project_at_pose_ (cloth_collision.h:109-203) for one pose of the snapshot.
__device__ __noinline__ bool project_pose(const PxbDevCollider* __restrict__ c, int pose, bool allow_sweep,
                             float thickness, f3& p, f3& normal_out, float& depth_out) {
    const PxbPose* ps = &c->pose[pose];
    const int type = __ldg(&c->type);
    if (type == PXB_SHAPE_SPHERE) {
        const f3 center = ld3(ps->center);
        f3 on_axis = center;
        if (allow_sweep && __ldg(&c->swept_sphere)) on_axis = closest_on_segment(p, center, ld3(ps->cb));
        const f3 d = sub(p, on_axis);
        const float l = len(d);
        const float target = __ldg(&c->radius) + thickness;
        if (l >= target) return false;
        const f3 n = (l > PXB_EPSILON) ? divs(d, l) : mk(0.0f, 0.0f, 1.0f);
        depth_out = target - l;
        p = add(on_axis, mul(n, target));
        normal_out = n;
        return true;
    }
    if (type == PXB_SHAPE_CAPSULE) {
        const f3 on_axis = closest_on_segment(p, ld3(ps->ca), ld3(ps->cb));
        const f3 d = sub(p, on_axis);
        const float l = len(d);
        const float target = __ldg(&c->radius) + thickness;
        if (l >= target) return false;
        const f3 n = (l > PXB_EPSILON) ? divs(d, l) : ld3(ps->t1);
        depth_out = target - l;
        p = add(on_axis, mul(n, target));
        normal_out = n;
        return true;
    }
    // Box
    const f3 center = ld3(ps->center);
    const f3 ax = ld3(ps->ax), ay = ld3(ps->ay), az = ld3(ps->az);
    const f3 d = sub(p, center);
    const f3 local = mk(dot(d, ax), dot(d, ay), dot(d, az));
    const f3 he = ld3(c->he);
    const bool inside = fabsf(local.x) <= he.x && fabsf(local.y) <= he.y && fabsf(local.z) <= he.z;
    f3 lt, ln;
    if (inside) {
        const f3 slack = mk(he.x - fabsf(local.x), he.y - fabsf(local.y), he.z - fabsf(local.z));
        const int axis = (slack.x <= slack.y && slack.x <= slack.z) ? 0 : (slack.y <= slack.z ? 1 : 2);
        const float lc = axis == 0 ? local.x : (axis == 1 ? local.y : local.z);
        const float hc = axis == 0 ? he.x : (axis == 1 ? he.y : he.z);
        const float sc = axis == 0 ? slack.x : (axis == 1 ? slack.y : slack.z);
        const float sign = (lc >= 0.0f) ? 1.0f : -1.0f;
        lt = local;
        ln = mk(0.0f, 0.0f, 0.0f);
        const float tv = sign * (hc + thickness);
        if (axis == 0) { lt.x = tv; ln.x = sign; }
        else if (axis == 1) { lt.y = tv; ln.y = sign; }
        else { lt.z = tv; ln.z = sign; }
        depth_out = sc + thickness;
    } else {
        lt = mk(minr(maxr(local.x, -he.x), he.x), minr(maxr(local.y, -he.y), he.y),
                minr(maxr(local.z, -he.z), he.z));
        const f3 delta = sub(local, lt);
        const float l = len(delta);
        if (l >= thickness) return false;
        ln = (l > PXB_EPSILON) ? divs(delta, l) : mk(0.0f, 0.0f, 1.0f);
        depth_out = thickness - l;
        lt = add(lt, mul(ln, thickness));
    }
    p = add(add(add(center, mul(ax, lt.x)), mul(ay, lt.y)), mul(az, lt.z));
    const f3 nw = add(add(mul(ax, ln.x), mul(ay, ln.y)), mul(az, ln.z));
    normal_out = mul(nw, 1.0f / sqrtf(dot(nw, nw)));
    return true;
}

__device__ __forceinline__ bool project_particle(const PxbDevCollider* __restrict__ c,
                                                 float thickness, f3& p, f3& n, float& depth) {
    if (!__ldg(&c->enabled)) return false;
    if (!__ldg(&c->two_pose)) return project_pose(c, 0, true, thickness, p, n, depth);
    f3 p0 = p, n0 = mk(0, 0, 0), p1 = p, n1 = mk(0, 0, 0);
    float d0 = 0.0f, d1 = 0.0f;
    const bool h0 = project_pose(c, 0, false, thickness, p0, n0, d0);
    const bool h1 = project_pose(c, 1, false, thickness, p1, n1, d1);
    if (!h0 && !h1) return false;
    if (h1 && (!h0 || d1 > d0)) {
        p = p1; n = n1; depth = d1;
    } else {
        p = p0; n = n0; depth = d0;
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// One XPBD distance projection (cloth_solver.h:119-138)
// ------------------------------------------------------------------------------------------

// Computes the new endpoint positions of one constraint. Returns false when the reference
// returns early (both pinned, or coincident endpoints) -- nothing is written then.
__device__ __forceinline__ bool solve_pair(float4& pa, float4& pb, float rest, float lam,
                                           float alpha, float& dlambda) {
    const float w = pa.w + pb.w;
    if (w <= 0.0f) return false;
    const float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    const float l = sqrtf(dx * dx + dy * dy + dz * dz);
    if (l < PXB_EPSILON) return false;
    const float nx = dx / l, ny = dy / l, nz = dz / l;
    const float c = l - rest;
    dlambda = (-c - alpha * lam) / (w + alpha);
    const float cx = dlambda * nx, cy = dlambda * ny, cz = dlambda * nz;
    pa.x = pa.x + pa.w * cx;
    pa.y = pa.y + pa.w * cy;
    pa.z = pa.z + pa.w * cz;
    pb.x = pb.x - pb.w * cx;
    pb.y = pb.y - pb.w * cy;
    pb.z = pb.z - pb.w * cz;
    return true;
}

}  // namespace
}  // namespace pxb

#endif  // PXB_DEVICE_MATH_CUH
