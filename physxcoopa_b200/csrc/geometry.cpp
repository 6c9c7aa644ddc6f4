// geometry.cpp -- collider geometry for the device path: geometry::ConvexHull and
// geometry::TriangleMesh registered once per context (C-ABI pxb_geometry_*), and the per-step
// collider records that point the kernels at them.
//
// Hulls stay on the host and are posed once per step and pose: the world vertices, face planes
// and outward edge normals that collision::world_posed_hull / hull_vs_sphere derive on every call
// (sat_hull.h:49-73, 160-194, 601-627) are evaluated here, with the reference's formulas and
// operation order, and copied to the device with the step. Meshes are copied to the device once,
// with a bounding-volume hierarchy built by MeshBVH::build's rule (mesh_bvh.h): leaves of at most
// four triangles, interior nodes split at the median centroid (std::nth_element) on the axis of
// their bounds' largest extent, nodes numbered in creation order (root first). The device walks
// it in the recursion's order, so the triangles a query visits, and the order it visits them in,
// are the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "host_math.h"
#include "pxb_internal.h"
#include "runtime_internal.h"

namespace {

using namespace pxb::hm;

V3 vmin(V3 a, V3 b) { return V3{b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z}; }
V3 vmax(V3 a, V3 b) { return V3{a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z}; }
float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

struct Bvh {
    std::vector<PxbMeshNode> nodes;
    std::vector<uint32_t> order;
    int depth = 0;
};

struct BvhBuilder {
    const std::vector<V3>& tmin;
    const std::vector<V3>& tmax;
    const std::vector<V3>& centroid;
    Bvh& out;

    int build(size_t start, size_t end, int level) {
        out.depth = std::max(out.depth, level);
        V3 mn{std::numeric_limits<float>::max(), std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
        V3 mx{std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
              std::numeric_limits<float>::lowest()};
        for (size_t i = start; i < end; ++i) {  // AABB::merge, in range order
            mn = vmin(mn, tmin[out.order[i]]);
            mx = vmax(mx, tmax[out.order[i]]);
        }
        const size_t count = end - start;
        const int idx = static_cast<int>(out.nodes.size());
        out.nodes.push_back(PxbMeshNode{});
        PxbMeshNode& nd = out.nodes[idx];
        nd.mn[0] = mn.x; nd.mn[1] = mn.y; nd.mn[2] = mn.z;
        nd.mx[0] = mx.x; nd.mx[1] = mx.y; nd.mx[2] = mx.z;
        if (count <= 4) {
            nd.left = -1 - static_cast<int32_t>(start);
            nd.right = static_cast<int32_t>(count);
            return idx;
        }
        const V3 ext = sub(mx, mn);
        int axis = 0;
        if (ext.y > comp(ext, axis)) axis = 1;
        if (ext.z > comp(ext, axis)) axis = 2;
        const size_t mid = start + count / 2;
        std::nth_element(out.order.begin() + start, out.order.begin() + mid, out.order.begin() + end,
                         [&](uint32_t a, uint32_t b) { return comp(centroid[a], axis) < comp(centroid[b], axis); });
        const int left = build(start, mid, level + 1);
        const int right = build(mid, end, level + 1);
        out.nodes[idx].left = left;
        out.nodes[idx].right = right;
        return idx;
    }
};

// Everything of one record that the posed hull depends on.
struct HullKey {
    uint32_t geometry;
    float position[3], orientation[4], local_center[3], local_rotation[4], scale;
    bool operator<(const HullKey& o) const { return std::memcmp(this, &o, sizeof(HullKey)) < 0; }
};

HullKey hull_key(const pxb_collider& c) {
    HullKey k;
    std::memset(&k, 0, sizeof(k));
    k.geometry = c.geometry;
    std::memcpy(k.position, c.position, 12);
    std::memcpy(k.orientation, c.orientation, 16);
    std::memcpy(k.local_center, c.local_center, 12);
    std::memcpy(k.local_rotation, c.local_rotation, 16);
    k.scale = c.geometry_scale;
    return k;
}

size_t hull_float4s(const GeometryEntry& g) { return 2 * (g.planes.size() / 4) + 2 * g.face_vertices.size(); }

// collision::world_posed_hull (sat_hull.h:66-73) at the collider's pose, then every quantity
// hull_vs_sphere and closest_point_on_convex_polygon_ derive from the posed hull.
void pose_hull(const GeometryEntry& g, const pxb_collider& c, float4* out) {
    const Q4 pose_rot = ldq(c.orientation);
    const V3 position = add(ld(c.position), qrot(pose_rot, ld(c.local_center)));
    const Q4 rotation = qmul(pose_rot, ldq(c.local_rotation));
    const float scale = c.geometry_scale;
    const size_t F = g.planes.size() / 4, V = g.face_vertices.size();
    const size_t nv = g.vertices.size() / 3;
    std::vector<V3> wv(nv);
    for (size_t i = 0; i < nv; ++i)  // PosedHull::world_vertex
        wv[i] = add(position, qrot(rotation, mul(ld(&g.vertices[3 * i]), scale)));
    for (size_t f = 0; f < F; ++f) {
        const V3 n = qrot(rotation, ld(&g.planes[4 * f]));  // PosedHull::world_face_normal
        const uint32_t s = g.starts[f], e = g.starts[f + 1];
        const float d = dot(n, wv[g.face_vertices[s]]);
        out[f] = make_float4(n.x, n.y, n.z, d);
        float4 span = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const int32_t first = static_cast<int32_t>(s), count = static_cast<int32_t>(e - s);
        std::memcpy(&span.x, &first, 4);
        std::memcpy(&span.y, &count, 4);
        out[F + f] = span;
        for (uint32_t i = 0; i < e - s; ++i) {
            const V3 a = wv[g.face_vertices[s + i]];
            const V3 b = wv[g.face_vertices[s + (i + 1) % (e - s)]];
            out[2 * F + s + i] = make_float4(a.x, a.y, a.z, 0.0f);
            // outward_edge_normal_ (sat_hull.h:162-166)
            const V3 m = cross(sub(b, a), n);
            const float l = length(m);
            const V3 o = l > 1e-12f ? V3{m.x / l, m.y / l, m.z / l} : n;
            out[2 * F + V + s + i] = make_float4(o.x, o.y, o.z, 0.0f);
        }
    }
}

uint32_t add_geometry(pxb_context* ctx, GeometryEntry&& g) {
    for (size_t i = 0; i < ctx->geometries.size(); ++i)
        if (!ctx->geometries[i].alive) {
            ctx->geometries[i] = std::move(g);
            return static_cast<uint32_t>(i + 1);
        }
    ctx->geometries.push_back(std::move(g));
    return static_cast<uint32_t>(ctx->geometries.size());
}

}  // namespace

pxb_status ColliderStage::plan(pxb_context* ctx, const pxb_collider* c, uint32_t n) {
    hull_block.assign(n, SIZE_MAX);
    geo.assign(n, 0);
    block_start.clear();
    block_record.clear();
    n_float4 = 0;
    std::map<HullKey, size_t> seen;
    for (uint32_t k = 0; k < n; ++k) {
        if (c[k].type != PXB_SHAPE_TRIANGLE_MESH && c[k].type != PXB_SHAPE_CONVEX_HULL) continue;
        if (!c[k].enabled || c[k].geometry == 0) continue;  // never collides (Shape::mesh / hull null)
        const GeometryEntry* g = ctx->lookup_geometry(c[k].geometry);
        if (!g) return ctx->fail(PXB_ERR_INVALID_HANDLE, "collider %u names geometry %u, which is not live", k, c[k].geometry);
        if (g->type != c[k].type)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider %u: geometry %u is a %s", k, c[k].geometry,
                             g->type == PXB_SHAPE_CONVEX_HULL ? "convex hull" : "triangle mesh");
        geo[k] = 1;
        if (c[k].type != PXB_SHAPE_CONVEX_HULL) continue;
        const HullKey key = hull_key(c[k]);
        auto it = seen.find(key);
        if (it == seen.end()) {
            it = seen.emplace(key, block_start.size()).first;
            block_start.push_back(n_float4);
            block_record.push_back(k);
            n_float4 += hull_float4s(*g);
        }
        hull_block[k] = block_start[it->second];
    }
    return PXB_OK;
}

void ColliderStage::fill(const pxb_context* ctx, const pxb_collider* c, uint32_t n, PxbDevCollider* out,
                         float4* host_geo, const float4* dev_geo) const {
    for (size_t b = 0; b < block_start.size(); ++b) {
        const pxb_collider& r = c[block_record[b]];
        pose_hull(*ctx->lookup_geometry(r.geometry), r, host_geo + block_start[b]);
    }
    for (uint32_t k = 0; k < n; ++k) {
        pxb_make_dev_collider(c[k], out[k]);
        PxbDevCollider& o = out[k];
        if (c[k].type != PXB_SHAPE_TRIANGLE_MESH && c[k].type != PXB_SHAPE_CONVEX_HULL) continue;
        o.two_pose = 0;  // neither is ever probed at two poses (cloth_collision.h:391-393)
        o.swept_sphere = 0;
        const GeometryEntry* g = c[k].enabled && c[k].geometry ? ctx->lookup_geometry(c[k].geometry) : nullptr;
        if (!g) {
            o.enabled = 0;
            continue;
        }
        if (c[k].type == PXB_SHAPE_CONVEX_HULL) {
            o.geo_count = static_cast<int32_t>(g->planes.size() / 4);
            o.geo_aux = static_cast<int32_t>(g->face_vertices.size());
            o.geo = dev_geo + hull_block[k];
            continue;
        }
        // TriangleMesh: project_at_pose_'s frame (cloth_collision.h:209-213)
        const Q4 pose_rot = ldq(c[k].orientation);
        const Q4 rot = qmul(pose_rot, ldq(c[k].local_rotation));
        const float qq = rot.x * rot.x + rot.y * rot.y + rot.z * rot.z + rot.w * rot.w;  // dot(q, q)
        const Q4 inv{-rot.x / qq, -rot.y / qq, -rot.z / qq, rot.w / qq};                 // conjugate / dot
        const V3 origin = add(ld(c[k].position), qrot(pose_rot, ld(c[k].local_center)));
        o.q[0] = rot.x; o.q[1] = rot.y; o.q[2] = rot.z; o.q[3] = rot.w;
        o.qi[0] = inv.x; o.qi[1] = inv.y; o.qi[2] = inv.z; o.qi[3] = inv.w;
        st(o.origin, origin);
        o.scale = c[k].geometry_scale > 1e-6f ? c[k].geometry_scale : 1.0f;
        if (g->grid) {  // a height grid: its record, walked through its block pyramid
            o.geo_count = 1;
            o.geo_aux = -1;
            o.geo = g->d_tris;
            o.nodes = nullptr;
            continue;
        }
        o.geo_count = g->n_nodes;
        o.geo_aux = g->depth;
        o.geo = g->d_tris;
        o.nodes = g->d_nodes;
    }
}

extern "C" {

pxb_status pxb_geometry_create_hull(pxb_context* ctx, const pxb_hull_desc* d, uint32_t* id_out) {
    if (!ctx || !d || !id_out) return PXB_ERR_INVALID_ARGUMENT;
    if (d->n_faces == 0) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "a hull needs at least one face");
    if (!d->vertices || !d->face_planes || !d->face_starts || !d->face_vertices || d->n_vertices == 0)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null hull arrays");
    if (d->n_faces > PXB_HULL_MAX_FACES) return ctx->fail(PXB_ERR_TOO_LARGE, "hull has %u faces (at most %d)", d->n_faces, PXB_HULL_MAX_FACES);
    if (d->face_starts[0] != 0) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "face_starts[0] must be 0");
    for (uint32_t f = 0; f < d->n_faces; ++f) {
        const uint32_t s = d->face_starts[f], e = d->face_starts[f + 1];
        if (e <= s) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "hull face %u has no vertex", f);
        if (e - s > PXB_HULL_MAX_FACE_VERTICES)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "hull face %u has %u vertices (at most %d)", f, e - s, PXB_HULL_MAX_FACE_VERTICES);
    }
    const uint32_t nfv = d->face_starts[d->n_faces];
    if (nfv > PXB_HULL_MAX_ENTRIES) return ctx->fail(PXB_ERR_TOO_LARGE, "hull has %u face-vertex entries (at most %d)", nfv, PXB_HULL_MAX_ENTRIES);
    for (uint32_t i = 0; i < nfv; ++i)
        if (d->face_vertices[i] >= d->n_vertices)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "hull face vertex %u is out of range", i);
    GeometryEntry g;
    g.alive = true;
    g.type = PXB_SHAPE_CONVEX_HULL;
    g.vertices.assign(d->vertices, d->vertices + 3 * static_cast<size_t>(d->n_vertices));
    g.planes.assign(d->face_planes, d->face_planes + 4 * static_cast<size_t>(d->n_faces));
    g.starts.assign(d->face_starts, d->face_starts + d->n_faces + 1);
    g.face_vertices.assign(d->face_vertices, d->face_vertices + nfv);
    *id_out = add_geometry(ctx, std::move(g));
    return PXB_OK;
}

pxb_status pxb_geometry_create_mesh(pxb_context* ctx, const pxb_mesh_desc* d, uint32_t* id_out) {
    if (!ctx || !d || !id_out) return PXB_ERR_INVALID_ARGUMENT;
    const size_t T = d->n_indices / 3;  // TriangleMesh reads indices.size() / 3 triangles
    if (T > PXB_MESH_MAX_TRIANGLES) return ctx->fail(PXB_ERR_TOO_LARGE, "mesh has %zu triangles (at most %u)", T, PXB_MESH_MAX_TRIANGLES);
    if (T && (!d->vertices || !d->indices)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null mesh arrays");
    for (size_t i = 0; i < 3 * T; ++i)
        if (d->indices[i] >= d->n_vertices) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "mesh index %zu is out of range", i);
    GeometryEntry g;
    g.alive = true;
    g.type = PXB_SHAPE_TRIANGLE_MESH;
    if (T) {
        std::vector<V3> v0(T), v1(T), v2(T), nrm(T), tmin(T), tmax(T), cen(T);
        for (size_t t = 0; t < T; ++t) {
            v0[t] = ld(&d->vertices[3 * static_cast<size_t>(d->indices[3 * t])]);
            v1[t] = ld(&d->vertices[3 * static_cast<size_t>(d->indices[3 * t + 1])]);
            v2[t] = ld(&d->vertices[3 * static_cast<size_t>(d->indices[3 * t + 2])]);
            if (d->normals) {
                nrm[t] = ld(&d->normals[3 * t]);
            } else {  // TriangleMesh::from_triangles: normalize(cross(b - a, c - a))
                const V3 cr = cross(sub(v1[t], v0[t]), sub(v2[t], v0[t]));
                nrm[t] = mul(cr, 1.0f / std::sqrt(dot(cr, cr)));
            }
            tmin[t] = vmin(v0[t], vmin(v1[t], v2[t]));
            tmax[t] = vmax(v0[t], vmax(v1[t], v2[t]));
            cen[t] = mul(add(add(v0[t], v1[t]), v2[t]), 1.0f / 3.0f);
        }
        Bvh bvh;
        bvh.order.resize(T);
        for (size_t t = 0; t < T; ++t) bvh.order[t] = static_cast<uint32_t>(t);
        BvhBuilder{tmin, tmax, cen, bvh}.build(0, T, 0);
        if (bvh.depth > PXB_MESH_MAX_DEPTH)
            return ctx->fail(PXB_ERR_TOO_LARGE, "mesh hierarchy is %d levels deep (at most %d)", bvh.depth, PXB_MESH_MAX_DEPTH);
        std::vector<PxbMeshTri> tris(T);
        for (size_t j = 0; j < T; ++j) {
            const uint32_t t = bvh.order[j];
            PxbMeshTri& r = tris[j];
            std::memset(&r, 0, sizeof(r));
            const V3 vs[3] = {v0[t], v1[t], v2[t]};
            for (int k = 0; k < 3; ++k) st(r.v[k], vs[k]);
            st(r.n, nrm[t]);
        }
        const size_t b_nodes = sizeof(PxbMeshNode) * bvh.nodes.size(), b_tris = sizeof(PxbMeshTri) * T;
        void* mem = nullptr;
        if (pxb_status s = ctx->cuda(cudaMalloc(&mem, b_nodes + b_tris), "mesh geometry")) return s;
        pxb_status s = ctx->cuda(cudaMemcpy(mem, bvh.nodes.data(), b_nodes, cudaMemcpyHostToDevice), "upload mesh hierarchy");
        if (!s) s = ctx->cuda(cudaMemcpy(static_cast<char*>(mem) + b_nodes, tris.data(), b_tris, cudaMemcpyHostToDevice),
                              "upload mesh triangles");
        if (s) {
            cudaFree(mem);
            return s;
        }
        g.dmem = mem;
        g.d_nodes = static_cast<const float4*>(mem);
        g.d_tris = reinterpret_cast<const float4*>(static_cast<char*>(mem) + b_nodes);
        g.n_nodes = static_cast<int>(bvh.nodes.size());
        g.depth = bvh.depth;
    }
    *id_out = add_geometry(ctx, std::move(g));
    return PXB_OK;
}

pxb_status pxb_geometry_create_height_grid(pxb_context* ctx, const pxb_height_grid_desc* d, uint32_t* id_out) {
    if (!ctx || !d || !id_out) return PXB_ERR_INVALID_ARGUMENT;
    if (d->n_heights && !d->heights) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null heights");
    // HeightGrid's constructor (height_grid.h): at least 2 x 2 samples, heights padded with zeros
    const int nx = std::max<int>(2, static_cast<int>(std::min<uint32_t>(d->nx, 1u << 15)));
    const int ny = std::max<int>(2, static_cast<int>(std::min<uint32_t>(d->ny, 1u << 15)));
    if (d->nx > (1u << 15) || d->ny > (1u << 15) || static_cast<uint64_t>(nx) * ny > (1ull << 24))
        return ctx->fail(PXB_ERR_TOO_LARGE, "height grid of %u x %u samples (at most 2^24 samples, sides up to 32768)",
                         d->nx, d->ny);
    const size_t n = static_cast<size_t>(nx) * ny;
    std::vector<float> h(n, 0.0f);
    std::memcpy(h.data(), d->heights, sizeof(float) * std::min<size_t>(n, d->n_heights));
    // build_pyramid_: each 8- and 64-cell block's lowest and highest sample over its cells
    const int cx = nx - 1, cy = ny - 1;
    const int fw = (cx + 7) / 8, fh = (cy + 7) / 8, cw = (cx + 63) / 64, ch = (cy + 63) / 64;
    std::vector<float> fine(2 * static_cast<size_t>(fw) * fh), coarse(2 * static_cast<size_t>(cw) * ch);
    for (size_t k = 0; k < fine.size(); k += 2) { fine[k] = std::numeric_limits<float>::max(); fine[k + 1] = std::numeric_limits<float>::lowest(); }
    for (size_t k = 0; k < coarse.size(); k += 2) { coarse[k] = std::numeric_limits<float>::max(); coarse[k + 1] = std::numeric_limits<float>::lowest(); }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const float hv = h[static_cast<size_t>(j) * nx + i];
            for (int dj = -1; dj <= 0; ++dj)
                for (int di = -1; di <= 0; ++di) {
                    const int ci = i + di, cj = j + dj;
                    if (ci < 0 || cj < 0 || ci >= cx || cj >= cy) continue;
                    float* f = &fine[2 * (static_cast<size_t>(cj / 8) * fw + ci / 8)];
                    float* c = &coarse[2 * (static_cast<size_t>(cj / 64) * cw + ci / 64)];
                    f[0] = std::min(f[0], hv);
                    f[1] = std::max(f[1], hv);
                    c[0] = std::min(c[0], hv);
                    c[1] = std::max(c[1], hv);
                }
        }
    // the device record: two header float4s, heights, 8-cell ranges, 64-cell ranges
    std::vector<float> rec(8 + n + fine.size() + coarse.size());
    const int32_t head[8] = {nx, ny, 0, 0, fw, fh, cw, ch};
    std::memcpy(rec.data(), head, sizeof(head));
    std::memcpy(&rec[2], &d->cell_x, 4);
    std::memcpy(&rec[3], &d->cell_y, 4);
    std::memcpy(&rec[8], h.data(), 4 * n);
    std::memcpy(&rec[8 + n], fine.data(), 4 * fine.size());
    std::memcpy(&rec[8 + n + fine.size()], coarse.data(), 4 * coarse.size());
    void* mem = nullptr;
    if (pxb_status s = ctx->cuda(cudaMalloc(&mem, 4 * rec.size()), "height grid")) return s;
    if (pxb_status s = ctx->cuda(cudaMemcpy(mem, rec.data(), 4 * rec.size(), cudaMemcpyHostToDevice), "upload height grid")) {
        cudaFree(mem);
        return s;
    }
    GeometryEntry g;
    g.alive = true;
    g.type = PXB_SHAPE_TRIANGLE_MESH;
    g.grid = true;
    g.dmem = mem;
    g.d_tris = static_cast<const float4*>(mem);
    g.n_nodes = 1;
    g.depth = -1;
    *id_out = add_geometry(ctx, std::move(g));
    return PXB_OK;
}

pxb_status pxb_geometry_destroy(pxb_context* ctx, uint32_t id) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (!ctx->lookup_geometry(id)) return ctx->fail(PXB_ERR_INVALID_HANDLE, "geometry %u is not live", id);
    GeometryEntry& g = ctx->geometries[id - 1];
    if (g.dmem) {
        if (pxb_status s = ctx->cuda(cudaStreamSynchronize(ctx->stream), "wait before freeing geometry")) return s;
        cudaFree(g.dmem);
    }
    g = GeometryEntry{};
    ctx->drop_graph();  // a captured step may hold the freed pointers in its upload
    return PXB_OK;
}

}  // extern "C"
