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
#include "pxb_quotient.cuh"

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

// util::safe_normalize (math.h:46-50).
__device__ __forceinline__ f3 safe_normalize(f3 v) {
    const float l2 = dot(v, v);
    if (l2 < PXB_EPSILON * PXB_EPSILON) return mk(0.0f, 0.0f, 0.0f);
    return mul(v, 1.0f / sqrtf(l2));
}
__device__ __forceinline__ f3 neg(f3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ f3 ldx(const float4* p) {
    const float4 v = __ldg(p);
    return mk(v.x, v.y, v.z);
}
// Rotation of v by the unit quaternion q (x, y, z, w): v + 2*(w*(u x v) + u x (u x v)).
__device__ __forceinline__ f3 qrot4(const float* q, f3 v) {
    const f3 u = mk(__ldg(q), __ldg(q + 1), __ldg(q + 2));
    const float w = __ldg(q + 3);
    const f3 uv = cross(u, v);
    const f3 uuv = cross(u, uv);
    return add(v, mul(add(mul(uv, w), uuv), 2.0f));
}

// ConvexHull branch of project_at_pose_ (cloth_collision.h:342-354): collision::hull_vs_sphere
// (sat_hull.h:649-688) with the particle as a probe sphere of radius `thickness`, over the hull
// posed for this step on the host (PxbDevCollider::geo), then point + normal * thickness.
__device__ __noinline__ bool project_hull(const PxbDevCollider* __restrict__ c, float thickness, f3& p,
                                          f3& normal_out, float& depth_out) {
    const float4* __restrict__ g = c->geo;
    const int F = __ldg(&c->geo_count), V = __ldg(&c->geo_aux);
    int best_face = 0;
    float best_dist = -3.40282347e38f;  // -numeric_limits<float>::max()
    bool any_positive = false;
    for (int f = 0; f < F; ++f) {
        const float4 pl = __ldg(&g[f]);
        const float dist = dot(mk(pl.x, pl.y, pl.z), p) - pl.w;
        if (dist > 0.0f) any_positive = true;
        if (dist > best_dist) {
            best_dist = dist;
            best_face = f;
        }
    }
    const float4 npl = __ldg(&g[best_face]);
    const f3 n = mk(npl.x, npl.y, npl.z);
    const float4 span = __ldg(&g[F + best_face]);
    const int first = __float_as_int(span.x), count = __float_as_int(span.y);
    const float4* __restrict__ poly = g + 2 * F + first;
    const float4* __restrict__ edge_out = g + 2 * F + V + first;
    // closest_point_on_convex_polygon_ (sat_hull.h:601-627)
    const f3 p0 = ldx(&poly[0]);
    const float plane_d = dot(n, p0);
    const f3 proj = sub(p, mul(n, dot(n, p) - plane_d));
    bool inside = true;
    for (int i = 0; i < count && inside; ++i)
        if (dot(ldx(&edge_out[i]), sub(proj, ldx(&poly[i]))) > 1e-6f) inside = false;
    f3 point = proj;
    if (!inside) {
        point = p0;
        float best_d2 = 3.40282347e38f;
        f3 a = p0;
        for (int i = 0; i < count; ++i) {
            const f3 b = ldx(&poly[i + 1 == count ? 0 : i + 1]);
            const f3 ab = sub(b, a);
            const float len2 = dot(ab, ab);
            const float t = len2 > 1e-12f ? clamp01(dot(sub(proj, a), ab) / len2) : 0.0f;
            const f3 q = add(a, mul(ab, t));
            const f3 dq = sub(proj, q);
            const float d2 = dot(dq, dq);
            if (d2 < best_d2) {
                best_d2 = d2;
                point = q;
            }
            a = b;
        }
    }
    f3 nrm;
    float pen;
    if (!any_positive) {
        const f3 diff = sub(point, p);
        const float dist = len(diff);
        nrm = dist > PXB_EPSILON ? divs(diff, dist) : n;
        pen = thickness + (-best_dist);
    } else {
        const f3 diff = sub(p, point);
        const float dist = len(diff);
        if (dist > thickness) return false;
        nrm = dist > PXB_EPSILON ? divs(diff, dist) : n;
        pen = thickness - dist;
    }
    p = add(point, mul(nrm, thickness));
    normal_out = nrm;
    depth_out = pen;
    return true;
}

// collision::closest_point_on_triangle (mesh_contact.h:63-99), Ericson's region analysis.
__device__ __forceinline__ f3 closest_on_triangle(f3 p, f3 a, f3 b, f3 c) {
    const f3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    const f3 bp = sub(p, b);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return add(a, smul(d1 / (d1 - d3), ab));
    const f3 cp = sub(p, c);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return add(a, smul(d2 / (d2 - d6), ac));
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f)
        return add(b, smul((d4 - d3) / ((d4 - d3) + (d5 - d6)), sub(c, b)));
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    return add(add(a, mul(ab, v)), mul(ac, w));
}

// geometry::ray_vs_triangle (ray.h:205-228), Moller-Trumbore.
__device__ __forceinline__ bool ray_triangle(f3 o, f3 dir, float max_d, f3 a, f3 b, f3 c, float& t) {
    const f3 e1 = sub(b, a), e2 = sub(c, a);
    const f3 pvec = cross(dir, e2);
    const float det = dot(e1, pvec);
    if (det > -PXB_EPSILON && det < PXB_EPSILON) return false;
    const float inv_det = 1.0f / det;
    const f3 tvec = sub(o, a);
    const float u = dot(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    const f3 qvec = cross(tvec, e1);
    const float v = dot(dir, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float cand = dot(e2, qvec) * inv_det;
    if (cand < 0.0f || cand > max_d) return false;
    t = cand;
    return true;
}

// Ray::intersect (ray.h:47-60), the slab test MeshBVH::raycast prunes with; inv = 1 / (dir + 1e-9).
__device__ __forceinline__ bool ray_box(f3 o, f3 inv, float max_d, float4 na, float4 nb) {
    const float t0x = (na.x - o.x) * inv.x, t0y = (na.y - o.y) * inv.y, t0z = (na.z - o.z) * inv.z;
    const float t1x = (nb.x - o.x) * inv.x, t1y = (nb.y - o.y) * inv.y, t1z = (nb.z - o.z) * inv.z;
    // glm::min / glm::max, then std::max / std::min over {x, y, z, bound} (first extreme kept)
    float t_near = minr(t0x, t1x);
    float m = minr(t0y, t1y);
    if (t_near < m) t_near = m;
    m = minr(t0z, t1z);
    if (t_near < m) t_near = m;
    if (t_near < 0.0f) t_near = 0.0f;
    float t_far = maxr(t0x, t1x);
    m = maxr(t0y, t1y);
    if (m < t_far) t_far = m;
    m = maxr(t0z, t1z);
    if (m < t_far) t_far = m;
    if (max_d < t_far) t_far = max_d;
    return !(t_far < t_near);
}

// TriangleMesh branch of project_at_pose_ (cloth_collision.h:205-340), in the mesh's own frame:
// the swept crossing test (a MeshBVH::raycast from the substep's start, gated by the motion's
// length), then the proximity query (MeshBVH::query over the thickness box). Both walk the
// hierarchy depth first, left child before right, which is MeshBVH's recursion order, so every
// tie between equally near triangles resolves as in the reference.
// A stored mesh's triangles: the hierarchy in PxbMeshNode records, the triangles in its order
// with their normals (PxbMeshTri). Walks are depth-first, left before right (MeshBVH).
struct BvhTris {
    const float4* __restrict__ nodes;
    const float4* __restrict__ tris;
    __device__ __forceinline__ void tri(int j, f3& v0, f3& v1, f3& v2) const {
        v0 = ldx(&tris[4 * j]);
        v1 = ldx(&tris[4 * j + 1]);
        v2 = ldx(&tris[4 * j + 2]);
    }
    __device__ __forceinline__ f3 normal(int j) const { return ldx(&tris[4 * j + 3]); }
    // every triangle of every node whose box passes `box(mn, mx)` (float4: xyz used)
    template <class Box, class Fn>
    __device__ __forceinline__ void visit(Box box, Fn fn) const {
        int stack[PXB_MESH_MAX_DEPTH + 4];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int idx = stack[--sp];
            const float4 na = __ldg(&nodes[2 * idx]), nb = __ldg(&nodes[2 * idx + 1]);
            if (!box(na, nb)) continue;
            const int left = __float_as_int(na.w), right = __float_as_int(nb.w);
            if (left >= 0) {
                stack[sp++] = right;
                stack[sp++] = left;
                continue;
            }
            const int t0 = -1 - left;
            for (int j = t0; j < t0 + right; ++j) fn(j);
        }
    }
};

// A height grid's triangles (geometry::HeightGrid, height_grid.h), from the geometry record:
// float4 (nx, ny as int bits, cell x, y), float4 (8-cell block columns, rows, 64-cell block
// columns, rows as int bits), then nx * ny heights (row j at j * nx), the 8-cell blocks' and the
// 64-cell blocks' (lowest, highest) sample. Cell (i, j)'s triangles are (i,j)-(i+1,j)-(i+1,j+1)
// and (i,j)-(i+1,j+1)-(i,j+1), numbered (j (nx - 1) + i) * 2 + half.
struct GridTris {
    const float* __restrict__ h;
    const float* __restrict__ fine;
    const float* __restrict__ coarse;
    int nx, ny, fw, fh, cw, ch;
    float cx, cy;
    __device__ __forceinline__ explicit GridTris(const float4* g) {
        const float4 a = __ldg(&g[0]), b = __ldg(&g[1]);
        nx = __float_as_int(a.x);
        ny = __float_as_int(a.y);
        cx = a.z;
        cy = a.w;
        fw = __float_as_int(b.x);
        fh = __float_as_int(b.y);
        cw = __float_as_int(b.z);
        ch = __float_as_int(b.w);
        h = reinterpret_cast<const float*>(g + 2);
        fine = h + static_cast<size_t>(nx) * ny;
        coarse = fine + 2 * static_cast<size_t>(fw) * fh;
    }
    __device__ __forceinline__ float at(int i, int j) const { return __ldg(&h[static_cast<size_t>(j) * nx + i]); }
    __device__ __forceinline__ f3 vertex(int i, int j) const {
        return mk(static_cast<float>(i) * cx, static_cast<float>(j) * cy, at(i, j));
    }
    __device__ __forceinline__ void tri(int t, f3& v0, f3& v1, f3& v2) const {
        const int half = t & 1, cell = t >> 1;
        const int j = cell / (nx - 1), i = cell - j * (nx - 1);
        v0 = vertex(i, j);
        if (half == 0) {
            v1 = vertex(i + 1, j);
            v2 = vertex(i + 1, j + 1);
        } else {
            v1 = vertex(i + 1, j + 1);
            v2 = vertex(i, j + 1);
        }
    }
    // HeightGrid::triangle_normal: normalize(cross(v1 - v0, v2 - v0)), +z when degenerate
    __device__ __forceinline__ f3 normal(int t) const {
        f3 v0, v1, v2;
        tri(t, v0, v1, v2);
        const f3 n = cross(sub(v1, v0), sub(v2, v0));
        const float l = len(n);
        return l > 0.0f ? divs(n, l) : mk(0.0f, 0.0f, 1.0f);
    }
    // HeightGrid::visit_: 64-cell blocks, their 8-cell blocks, their cells, each row-major, a
    // block or cell skipped when its box fails `box`; a cell's two triangles in order
    template <class Box, class Fn>
    __device__ __forceinline__ void visit(Box box, Fn fn) const {
        const int cxn = nx - 1, cyn = ny - 1;
        for (int gj = 0; gj < ch; ++gj)
            for (int gi = 0; gi < cw; ++gi) {
                const int c0i = gi * 64, c0j = gj * 64;
                const int c1i = min(c0i + 64, cxn), c1j = min(c0j + 64, cyn);
                const float* r = coarse + 2 * (static_cast<size_t>(gj) * cw + gi);
                if (!box(make_float4(static_cast<float>(c0i) * cx, static_cast<float>(c0j) * cy, __ldg(&r[0]), 0.0f),
                         make_float4(static_cast<float>(c1i) * cx, static_cast<float>(c1j) * cy, __ldg(&r[1]), 0.0f)))
                    continue;
                for (int fj = c0j / 8; fj * 8 < c1j; ++fj)
                    for (int fi = c0i / 8; fi * 8 < c1i; ++fi) {
                        const int f0i = fi * 8, f0j = fj * 8;
                        const int f1i = min(f0i + 8, cxn), f1j = min(f0j + 8, cyn);
                        const float* q = fine + 2 * (static_cast<size_t>(fj) * fw + fi);
                        if (!box(make_float4(static_cast<float>(f0i) * cx, static_cast<float>(f0j) * cy, __ldg(&q[0]), 0.0f),
                                 make_float4(static_cast<float>(f1i) * cx, static_cast<float>(f1j) * cy, __ldg(&q[1]), 0.0f)))
                            continue;
                        for (int j = f0j; j < f1j; ++j)
                            for (int i = f0i; i < f1i; ++i) {
                                // std::min / std::max of the cell's four samples, as the reference writes them
                                const float a = at(i, j), b = at(i + 1, j), c = at(i, j + 1), d = at(i + 1, j + 1);
                                const float lo1 = b < a ? b : a, lo2 = d < c ? d : c;
                                const float hi1 = a < b ? b : a, hi2 = c < d ? d : c;
                                if (!box(make_float4(static_cast<float>(i) * cx, static_cast<float>(j) * cy,
                                                     lo2 < lo1 ? lo2 : lo1, 0.0f),
                                         make_float4(static_cast<float>(i + 1) * cx, static_cast<float>(j + 1) * cy,
                                                     hi1 < hi2 ? hi2 : hi1, 0.0f)))
                                    continue;
                                fn((j * cxn + i) * 2);
                                fn((j * cxn + i) * 2 + 1);
                            }
                    }
            }
    }
};

// project_at_pose_'s TriangleMesh branch (cloth_collision.h:205-340) over either source: the
// swept crossing raycast (first hit along the substep's motion), else the proximity query (the
// last of equally near triangles kept).
template <class Tris>
__device__ __forceinline__ bool project_tris(const PxbDevCollider* __restrict__ c, const Tris& T, float thickness,
                                             f3& p, f3& normal_out, float& depth_out, f3 start, bool has_start) {
    const f3 origin = ld3(c->origin);
    const float scale = __ldg(&c->scale);
    const f3 local_p = divs(qrot4(c->qi, sub(p, origin)), scale);
    const float lt = thickness / scale;

    if (has_start) {
        const f3 local_start = divs(qrot4(c->qi, sub(start, origin)), scale);
        const f3 seg = sub(local_p, local_start);
        const float seg_len = len(seg);
        if (seg_len > lt) {
            const f3 dir = divs(seg, seg_len);
            const f3 inv = mk(1.0f / (dir.x + 1e-9f), 1.0f / (dir.y + 1e-9f), 1.0f / (dir.z + 1e-9f));
            float best_t = seg_len;
            int crossed = -1;
            T.visit([&](float4 na, float4 nb) { return ray_box(local_start, inv, seg_len, na, nb); },
                    [&](int j) {
                        f3 v0, v1, v2;
                        T.tri(j, v0, v1, v2);
                        float t = 0.0f;
                        if ((ray_triangle(local_start, dir, seg_len, v0, v1, v2, t) ||
                             ray_triangle(local_start, dir, seg_len, v0, v2, v1, t)) && t < best_t) {
                            best_t = t;
                            crossed = j;
                        }
                    });
            if (crossed >= 0) {
                const f3 local_hit = add(local_start, mul(dir, best_t));
                f3 face = safe_normalize(T.normal(crossed));
                if (dot(sub(local_start, local_hit), face) < 0.0f) face = neg(face);
                const f3 local_fixed = add(local_hit, mul(face, lt));
                depth_out = len(sub(local_p, local_fixed)) * scale;
                p = add(origin, qrot4(c->q, mul(local_fixed, scale)));
                normal_out = qrot4(c->q, face);
                return true;
            }
        }
    }

    const f3 qmn = mk(local_p.x - lt, local_p.y - lt, local_p.z - lt);
    const f3 qmx = mk(local_p.x + lt, local_p.y + lt, local_p.z + lt);
    const float lt2 = lt * lt;
    float best_d2 = lt2;
    f3 best_point = mk(0.0f, 0.0f, 0.0f), best_delta = mk(0.0f, 0.0f, 0.0f);
    int best_tri = -1;
    bool any_front = false;
    // AABB::overlaps (aabb.h:35-39)
    T.visit([&](float4 na, float4 nb) {
                return na.x <= qmx.x && nb.x >= qmn.x && na.y <= qmx.y && nb.y >= qmn.y && na.z <= qmx.z &&
                       nb.z >= qmn.z;
            },
            [&](int j) {
                f3 v0, v1, v2;
                T.tri(j, v0, v1, v2);
                const f3 closest = closest_on_triangle(local_p, v0, v1, v2);
                const f3 delta = sub(local_p, closest);
                const float d2 = dot(delta, delta);
                if (d2 > lt2) return;
                if (dot(delta, T.normal(j)) >= 0.0f) any_front = true;
                if (d2 > best_d2) return;
                best_d2 = d2;
                best_point = closest;
                best_delta = delta;
                best_tri = j;
            });
    if (best_tri < 0) return false;
    f3 bn;
    if (!any_front) {
        bn = safe_normalize(T.normal(best_tri));
    } else if (best_d2 > PXB_EPSILON * PXB_EPSILON) {
        bn = divs(best_delta, sqrtf(best_d2));
    } else {
        const f3 face = safe_normalize(T.normal(best_tri));
        bn = dot(best_delta, face) < 0.0f ? neg(face) : face;
    }
    const f3 local_fixed = add(best_point, mul(bn, lt));
    depth_out = len(sub(local_p, local_fixed)) * scale;
    p = add(origin, qrot4(c->q, mul(local_fixed, scale)));
    normal_out = qrot4(c->q, bn);
    return true;
}

// The two walks are separate calls so that each is register-allocated on its own.
__device__ __noinline__ bool project_grid_mesh(const PxbDevCollider* __restrict__ c, float thickness, f3& p,
                                               f3& normal_out, float& depth_out, f3 start, bool has_start) {
    return project_tris(c, GridTris(c->geo), thickness, p, normal_out, depth_out, start, has_start);
}

__device__ __noinline__ bool project_bvh_mesh(const PxbDevCollider* __restrict__ c, float thickness, f3& p,
                                              f3& normal_out, float& depth_out, f3 start, bool has_start) {
    return project_tris(c, BvhTris{c->nodes, c->geo}, thickness, p, normal_out, depth_out, start, has_start);
}

// A mesh collider: a stored mesh (geo_count hierarchy nodes, 0 when empty) or a height grid
// (geo_aux -1, geo its record).
__device__ __forceinline__ bool project_mesh(const PxbDevCollider* __restrict__ c, float thickness, f3& p,
                                             f3& normal_out, float& depth_out, f3 start, bool has_start) {
    if (__ldg(&c->geo_aux) < 0) return project_grid_mesh(c, thickness, p, normal_out, depth_out, start, has_start);
    if (__ldg(&c->geo_count) == 0) return false;  // TriangleMesh::empty()
    return project_bvh_mesh(c, thickness, p, normal_out, depth_out, start, has_start);
}

// cloth::project_particle (cloth_collision.h:386-420). `start` is the particle's position at
// the start of the substep (the motion_start the solvers pass), read by the mesh branch only.
// kGeo compiles the mesh and hull branches in: kernels whose launches carry no such collider
// are instantiated without them, since a called function's registers count against its caller.
template <bool kGeo>
__device__ __forceinline__ bool project_particle(const PxbDevCollider* __restrict__ c,
                                                 float thickness, f3& p, f3& n, float& depth,
                                                 f3 start = f3{0.0f, 0.0f, 0.0f}, bool has_start = false) {
    if (!__ldg(&c->enabled)) return false;
    if constexpr (kGeo) {
        const int type = __ldg(&c->type);
        if (type == PXB_SHAPE_CONVEX_HULL) return project_hull(c, thickness, p, n, depth);
        if (type == PXB_SHAPE_TRIANGLE_MESH) return project_mesh(c, thickness, p, n, depth, start, has_start);
    }
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

// The new endpoint positions and dlambda of one constraint, computed unconditionally; returns
// false where the reference returns early (both endpoints pinned, or coincident endpoints), and
// the caller then writes nothing. Every operation is the reference's, in its order and with its
// rounding: the pairs (x, y) of d, of d*d and of the corrections go through the two-lane FP32
// instructions (each lane rounded as the scalar one), (dz, w) = (a.z - b.z, a.w + b.w) through
// one of them (b times (-1, 1) is exact, the sum rounded once). kLam false means the colour's
// compliance is exactly +0, so -c - alpha * lambda is -c. pxb_check_projections compares this
// form with the scalar one, every output bit.
template <bool kLam = true>
__device__ __forceinline__ bool distance_core(float4& pa, float4& pb, float rest, float lam, float alpha,
                                              float& dlambda) {
    const float2 dxy = fma2_rn(make_float2(pb.x, pb.y), make_float2(-1.0f, -1.0f), make_float2(pa.x, pa.y));
    const float2 dzw = fma2_rn(make_float2(pb.z, pb.w), make_float2(-1.0f, 1.0f), make_float2(pa.z, pa.w));
    const float dz = dzw.x, w = dzw.y;
    const float2 sq = mul2_rn(dxy, dxy);
    const float l = sqrtf((sq.x + sq.y) + dz * dz);
    const bool ok = !(w <= 0.0f) && !(l < PXB_EPSILON);
    float nx, ny, nz;
    unit3(dxy.x, dxy.y, dz, l, nx, ny, nz);
    const float c = l - rest;
    const float num = kLam ? -c - alpha * lam : -c;
    dlambda = num / (w + alpha);
    const float2 cxy = mul2_rn(make_float2(dlambda, dlambda), make_float2(nx, ny));
    const float cz = dlambda * nz;
    // The endpoint updates stay scalar: built from an endpoint's own inverse mass (one register
    // of a loaded pair repeated in both lanes), the packed form measured wrong in the y lane.
    pa.x = pa.x + pa.w * cxy.x;
    pa.y = pa.y + pa.w * cxy.y;
    pa.z = pa.z + pa.w * cz;
    pb.x = pb.x - pb.w * cxy.x;
    pb.y = pb.y - pb.w * cxy.y;
    pb.z = pb.z - pb.w * cz;
    return ok;
}

// One XPBD distance projection: returns false (and leaves pa, pb alone) where the reference
// returns early.
__device__ __forceinline__ bool solve_pair(float4& pa, float4& pb, float rest, float lam,
                                           float alpha, float& dlambda) {
    float4 a = pa, b = pb;
    if (!distance_core(a, b, rest, lam, alpha, dlambda)) return false;
    pa = a;
    pb = b;
    return true;
}

}  // namespace
}  // namespace pxb

#endif  // PXB_DEVICE_MATH_CUH
