/*
 * xpbd_oracle.c -- CPU restatement of physxcoopa's XPBD cloth substep (see xpbd_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU path, never part of the shipped library.
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off). All arithmetic is IEEE single precision
 * in the order the reference writes it; glm's vector helpers are spelled out with the GLSL
 * definitions (dot left to right, length = sqrt(dot), mix = x*(1-a) + y*a).
 */
#include "xpbd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* util::k_epsilon (physxcoopa/util/math.h:19). */
#define K_EPSILON 1e-6f
/* util::k_max_cloth_substeps (physxcoopa/util/math.h:37). */
#define K_MAX_CLOTH_SUBSTEPS 16u

typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } q4;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld(const float* p) { return mk(p[0], p[1], p[2]); }
static inline void st(float* p, v3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
static inline q4 ldq(const float* p) { q4 q = {p[0], p[1], p[2], p[3]}; return q; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 smul(float s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline v3 divs(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float len(v3 a) { return sqrtf(dot(a, a)); }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline float fminr(float a, float b) { return b < a ? b : a; } /* glm::min / std::min */
static inline float fmaxr(float a, float b) { return a < b ? b : a; } /* glm::max / std::max */
static inline v3 mixv(v3 x, v3 y, float a) { return add(mul(x, 1.0f - a), mul(y, a)); }
static inline float clampf(float x, float lo, float hi) { /* std::clamp */
    return x < lo ? lo : (hi < x ? hi : x);
}

/* Unit-quaternion rotation v + 2*(w*(u x v) + u x (u x v)), u = (x,y,z). */
static inline v3 qrot(q4 q, v3 v) {
    const v3 u = mk(q.x, q.y, q.z);
    const v3 uv = cross(u, v);
    const v3 uuv = cross(u, uv);
    return add(v, mul(add(mul(uv, q.w), uuv), 2.0f));
}
/* Hamilton product p*q. */
static inline q4 qmul(q4 p, q4 q) {
    q4 r;
    r.w = p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z;
    r.x = p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y;
    r.y = p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z;
    r.z = p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x;
    return r;
}
/* Columns of the rotation matrix of unit q (glm::mat3_cast), i.e. the rotated basis. */
static inline void qaxes(q4 q, v3* ax, v3* ay, v3* az) {
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xz = q.x * q.z, xy = q.x * q.y, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    *ax = mk(1.0f - 2.0f * (yy + zz), 2.0f * (xy + wz), 2.0f * (xz - wy));
    *ay = mk(2.0f * (xy - wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + wx));
    *az = mk(2.0f * (xz + wy), 2.0f * (yz - wx), 1.0f - 2.0f * (xx + yy));
}
static inline float comp(v3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
static inline void setcomp(v3* v, int i, float s) {
    if (i == 0) v->x = s; else if (i == 1) v->y = s; else v->z = s;
}

/* util::safe_normalize (math.h:46-50). */
static v3 safe_normalize(v3 v) {
    const float l2 = dot(v, v);
    if (l2 < K_EPSILON * K_EPSILON) return mk(0.0f, 0.0f, 0.0f);
    return mul(v, 1.0f / sqrtf(l2));
}
/* util::orthonormal_basis (math.h:62-68), first tangent only. */
static v3 orthonormal_t1(v3 n) {
    const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    return mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
}
/* geometry::closest_point_on_segment (capsule.h:39-49). */
static v3 closest_point_on_segment(v3 point, v3 a, v3 b) {
    const v3 ab = sub(b, a);
    const float len2 = dot(ab, ab);
    if (len2 < K_EPSILON) return a;
    float t = dot(sub(point, a), ab) / len2;
    t = clampf(t, 0.0f, 1.0f);
    return add(a, mul(ab, t));
}

/* ---- collider geometry, by pxb_collider::geometry id ---------------------------------- */

typedef struct {
    int type; /* 0: free slot */
    /* geometry::ConvexHull (convex_hull.h:41-57) */
    float* verts;
    uint32_t n_verts;
    float* planes;
    uint32_t n_faces;
    uint32_t* starts;
    uint32_t* fverts;
    /* geometry::TriangleMesh (triangle_mesh.h:70-96) and its MeshBVH */
    float* mverts;
    uint32_t* idx;
    float* normals;
    uint32_t n_tris;
    orc_bvh_node* nodes;
    uint32_t n_nodes;
    uint32_t* order;
    /* geometry::HeightGrid (height_grid.h) behind TriangleMesh::from_height_grid */
    int grid;
    int nx, ny;
    float cell_x, cell_y;
    float* h;                     /* nx * ny heights, row j at j * nx */
    float* fine;                  /* (lo, hi) per 8 x 8-cell block */
    float* coarse;                /* (lo, hi) per 64 x 64-cell block */
    int fine_w, fine_h, coarse_w, coarse_h;
} orc_geometry;

#define ORC_MAX_GEOMETRY 1024
static orc_geometry g_geo[ORC_MAX_GEOMETRY];

static void free_geometry(orc_geometry* g) {
    free(g->verts); free(g->planes); free(g->starts); free(g->fverts);
    free(g->mverts); free(g->idx); free(g->normals); free(g->nodes); free(g->order);
    free(g->h); free(g->fine); free(g->coarse);
    memset(g, 0, sizeof(*g));
}

void orc_geometry_clear(void) {
    for (int i = 0; i < ORC_MAX_GEOMETRY; ++i) free_geometry(&g_geo[i]);
}

static void* dup(const void* src, size_t bytes) {
    void* d = malloc(bytes ? bytes : 1);
    if (bytes) memcpy(d, src, bytes);
    return d;
}

int orc_geometry_set_hull(uint32_t id, const pxb_hull_desc* d) {
    if (id == 0 || id >= ORC_MAX_GEOMETRY || d->n_faces == 0) return -1;
    orc_geometry* g = &g_geo[id];
    free_geometry(g);
    const uint32_t nfv = d->face_starts[d->n_faces];
    g->type = PXB_SHAPE_CONVEX_HULL;
    g->n_verts = d->n_vertices;
    g->n_faces = d->n_faces;
    g->verts = (float*)dup(d->vertices, sizeof(float) * 3 * d->n_vertices);
    g->planes = (float*)dup(d->face_planes, sizeof(float) * 4 * d->n_faces);
    g->starts = (uint32_t*)dup(d->face_starts, sizeof(uint32_t) * (d->n_faces + 1));
    g->fverts = (uint32_t*)dup(d->face_vertices, sizeof(uint32_t) * nfv);
    return 0;
}

int orc_geometry_set_mesh(uint32_t id, const pxb_mesh_desc* d) {
    if (id == 0 || id >= ORC_MAX_GEOMETRY) return -1;
    orc_geometry* g = &g_geo[id];
    free_geometry(g);
    const uint32_t T = d->n_indices / 3;
    g->type = PXB_SHAPE_TRIANGLE_MESH;
    g->n_tris = T;
    g->mverts = (float*)dup(d->vertices, sizeof(float) * 3 * d->n_vertices);
    g->idx = (uint32_t*)dup(d->indices, sizeof(uint32_t) * 3 * T);
    g->normals = (float*)malloc(sizeof(float) * 3 * (T ? T : 1));
    for (uint32_t t = 0; t < T; ++t) {
        if (d->normals) {
            memcpy(&g->normals[3 * t], &d->normals[3 * t], 12);
        } else { /* TriangleMesh::from_triangles: normalize(cross(b - a, c - a)) */
            const v3 a = ld(&d->vertices[3 * g->idx[3 * t]]), b = ld(&d->vertices[3 * g->idx[3 * t + 1]]),
                     c = ld(&d->vertices[3 * g->idx[3 * t + 2]]);
            const v3 cr = cross(sub(b, a), sub(c, a));
            st(&g->normals[3 * t], mul(cr, 1.0f / sqrtf(dot(cr, cr))));
        }
    }
    g->nodes = (orc_bvh_node*)malloc(sizeof(orc_bvh_node) * (2 * T + 1));
    g->order = (uint32_t*)malloc(sizeof(uint32_t) * (T ? T : 1));
    g->n_nodes = T ? orc_bvh_build(g->mverts, g->idx, T, g->nodes, g->order) : 0;
    return 0;
}

/* HeightGrid's constructor and build_pyramid_ (height_grid.h): at least 2 x 2 samples, heights
 * padded with zeros; per 8- and 64-cell block the lowest and highest sample of its cells. */
int orc_geometry_set_height_grid(uint32_t id, int nx, int ny, float cell_x, float cell_y, const float* heights,
                                 uint32_t n_heights) {
    if (id == 0 || id >= ORC_MAX_GEOMETRY) return -1;
    orc_geometry* g = &g_geo[id];
    free_geometry(g);
    g->type = PXB_SHAPE_TRIANGLE_MESH;
    g->grid = 1;
    g->nx = nx < 2 ? 2 : nx;
    g->ny = ny < 2 ? 2 : ny;
    g->cell_x = cell_x;
    g->cell_y = cell_y;
    const size_t n = (size_t)g->nx * g->ny;
    g->h = (float*)calloc(n, sizeof(float));
    memcpy(g->h, heights, sizeof(float) * (n_heights < n ? n_heights : n));
    const int cx = g->nx - 1, cy = g->ny - 1;
    g->fine_w = (cx + 7) / 8;
    g->fine_h = (cy + 7) / 8;
    g->coarse_w = (cx + 63) / 64;
    g->coarse_h = (cy + 63) / 64;
    g->fine = (float*)malloc(sizeof(float) * 2 * g->fine_w * g->fine_h);
    g->coarse = (float*)malloc(sizeof(float) * 2 * g->coarse_w * g->coarse_h);
    for (int k = 0; k < g->fine_w * g->fine_h; ++k) { g->fine[2 * k] = FLT_MAX; g->fine[2 * k + 1] = -FLT_MAX; }
    for (int k = 0; k < g->coarse_w * g->coarse_h; ++k) { g->coarse[2 * k] = FLT_MAX; g->coarse[2 * k + 1] = -FLT_MAX; }
    for (int j = 0; j < g->ny; ++j)
        for (int i = 0; i < g->nx; ++i) {
            const float hv = g->h[(size_t)j * g->nx + i];
            for (int dj = -1; dj <= 0; ++dj)
                for (int di = -1; di <= 0; ++di) {
                    const int ci = i + di, cj = j + dj;
                    if (ci < 0 || cj < 0 || ci >= cx || cj >= cy) continue;
                    float* f = &g->fine[2 * ((cj / 8) * g->fine_w + ci / 8)];
                    float* c = &g->coarse[2 * ((cj / 64) * g->coarse_w + ci / 64)];
                    if (hv < f[0]) f[0] = hv; /* std::min(lo, h) */
                    if (f[1] < hv) f[1] = hv; /* std::max(hi, h) */
                    if (hv < c[0]) c[0] = hv;
                    if (c[1] < hv) c[1] = hv;
                }
        }
    return 0;
}

static const orc_geometry* geometry_of(const pxb_collider* s, int type) {
    if (s->geometry == 0 || s->geometry >= ORC_MAX_GEOMETRY) return NULL;
    const orc_geometry* g = &g_geo[s->geometry];
    return g->type == type ? g : NULL;
}

/* conjugate(q) / dot(q, q) (glm::inverse of a quaternion) */
static inline q4 qinverse(q4 q) {
    const float qq = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    q4 r = {-q.x / qq, -q.y / qq, -q.z / qq, q.w / qq};
    return r;
}

/* ---- ConvexHull: collision::hull_vs_sphere (sat_hull.h:649-688) ----------------------- */

typedef struct {
    const orc_geometry* g;
    v3 position;
    q4 rotation;
    float scale;
} posed_hull;

static v3 hull_world_vertex(const posed_hull* h, uint32_t i) { /* PosedHull::world_vertex */
    return add(h->position, qrot(h->rotation, mul(ld(&h->g->verts[3 * i]), h->scale)));
}
static v3 hull_world_normal(const posed_hull* h, uint32_t f) { /* PosedHull::world_face_normal */
    return qrot(h->rotation, ld(&h->g->planes[4 * f]));
}
/* outward_edge_normal_ (sat_hull.h:162-166) */
static v3 outward_edge_normal(v3 edge_dir, v3 face_normal) {
    const v3 n = cross(edge_dir, face_normal);
    const float l = len(n);
    return l > 1e-12f ? divs(n, l) : face_normal;
}
/* closest_point_on_convex_polygon_ (sat_hull.h:601-627) */
static v3 closest_on_convex_polygon(const v3* poly, int n, v3 normal, v3 point) {
    const float plane_d = dot(normal, poly[0]);
    const v3 proj = sub(point, mul(normal, dot(normal, point) - plane_d));
    int inside = 1;
    for (int i = 0; i < n && inside; ++i) {
        const v3 a = poly[i], b = poly[(i + 1) % n];
        const v3 outward = outward_edge_normal(sub(b, a), normal);
        if (dot(outward, sub(proj, a)) > 1e-6f) inside = 0;
    }
    if (inside) return proj;
    v3 best = poly[0];
    float best_dist2 = 3.402823466e+38f;
    for (int i = 0; i < n; ++i) {
        const v3 a = poly[i], b = poly[(i + 1) % n];
        const v3 ab = sub(b, a);
        const float len2 = dot(ab, ab);
        const float t = len2 > 1e-12f ? clampf(dot(sub(proj, a), ab) / len2, 0.0f, 1.0f) : 0.0f;
        const v3 q = add(a, mul(ab, t));
        const float d2 = dot(sub(proj, q), sub(proj, q));
        if (d2 < best_dist2) {
            best_dist2 = d2;
            best = q;
        }
    }
    return best;
}
static int hull_vs_sphere(const posed_hull* h, v3 center, float radius, v3* normal, float* pen, v3* point) {
    uint32_t best_face = 0;
    float best_dist = -3.402823466e+38f;
    int any_positive = 0;
    for (uint32_t f = 0; f < h->g->n_faces; ++f) {
        const v3 n = hull_world_normal(h, f);
        const float d = dot(n, hull_world_vertex(h, h->g->fverts[h->g->starts[f]]));
        const float dist = dot(n, center) - d;
        if (dist > 0.0f) any_positive = 1;
        if (dist > best_dist) {
            best_dist = dist;
            best_face = f;
        }
    }
    const v3 n = hull_world_normal(h, best_face);
    v3 poly[160]; /* k_hull_clip_cap (sat_hull.h:157) */
    const uint32_t s0 = h->g->starts[best_face], e0 = h->g->starts[best_face + 1];
    const int count = (int)(e0 - s0) < 160 ? (int)(e0 - s0) : 160;
    for (int i = 0; i < count; ++i) poly[i] = hull_world_vertex(h, h->g->fverts[s0 + i]);
    *point = closest_on_convex_polygon(poly, count, n, center);
    if (!any_positive) {
        const v3 diff = sub(*point, center);
        const float dist = len(diff);
        *normal = dist > K_EPSILON ? divs(diff, dist) : n;
        *pen = radius + (-best_dist);
        return 1;
    }
    const v3 diff = sub(center, *point);
    const float dist = len(diff);
    if (dist > radius) return 0;
    *normal = dist > K_EPSILON ? divs(diff, dist) : n;
    *pen = radius - dist;
    return 1;
}

/* ---- TriangleMesh: MeshBVH queries (mesh_bvh.h) and the mesh branch ------------------- */

/* collision::closest_point_on_triangle (mesh_contact.h:63-99) */
static v3 closest_on_triangle(v3 p, v3 a, v3 b, v3 c) {
    const v3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    const v3 bp = sub(p, b);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        return add(a, smul(v, ab));
    }
    const v3 cp = sub(p, c);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        return add(a, smul(w, ac));
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return add(b, smul(w, sub(c, b)));
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom;
    const float w = vc * denom;
    return add(add(a, mul(ab, v)), mul(ac, w));
}

typedef struct {
    v3 origin, direction;
    float max_distance;
} ray3;

/* Ray::intersect (ray.h:47-60) */
static int ray_box(const ray3* r, const float* mn, const float* mx) {
    const v3 inv = mk(1.0f / (r->direction.x + 1e-9f), 1.0f / (r->direction.y + 1e-9f),
                      1.0f / (r->direction.z + 1e-9f));
    const v3 t0 = mk((mn[0] - r->origin.x) * inv.x, (mn[1] - r->origin.y) * inv.y, (mn[2] - r->origin.z) * inv.z);
    const v3 t1 = mk((mx[0] - r->origin.x) * inv.x, (mx[1] - r->origin.y) * inv.y, (mx[2] - r->origin.z) * inv.z);
    const v3 tmin = mk(fminr(t0.x, t1.x), fminr(t0.y, t1.y), fminr(t0.z, t1.z));
    const v3 tmax = mk(fmaxr(t0.x, t1.x), fmaxr(t0.y, t1.y), fmaxr(t0.z, t1.z));
    /* std::max / std::min over an initializer list keep the first extreme */
    float t_near = tmin.x;
    if (t_near < tmin.y) t_near = tmin.y;
    if (t_near < tmin.z) t_near = tmin.z;
    if (t_near < 0.0f) t_near = 0.0f;
    float t_far = tmax.x;
    if (tmax.y < t_far) t_far = tmax.y;
    if (tmax.z < t_far) t_far = tmax.z;
    if (r->max_distance < t_far) t_far = r->max_distance;
    return !(t_far < t_near);
}

/* geometry::ray_vs_triangle (ray.h:205-228) */
static int ray_triangle(const ray3* r, v3 a, v3 b, v3 c, float* t) {
    const v3 edge1 = sub(b, a), edge2 = sub(c, a);
    const v3 pvec = cross(r->direction, edge2);
    const float det = dot(edge1, pvec);
    if (det > -K_EPSILON && det < K_EPSILON) return 0;
    const float inv_det = 1.0f / det;
    const v3 tvec = sub(r->origin, a);
    const float u = dot(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return 0;
    const v3 qvec = cross(tvec, edge1);
    const float v = dot(r->direction, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return 0;
    const float candidate = dot(edge2, qvec) * inv_det;
    if (candidate < 0.0f || candidate > r->max_distance) return 0;
    *t = candidate;
    return 1;
}

static void mesh_tri(const orc_geometry* g, uint32_t t, v3* v0, v3* v1, v3* v2) {
    *v0 = ld(&g->mverts[3 * g->idx[3 * t]]);
    *v1 = ld(&g->mverts[3 * g->idx[3 * t + 1]]);
    *v2 = ld(&g->mverts[3 * g->idx[3 * t + 2]]);
}

/* HeightGrid::vertex / triangle_vertices (height_grid.h): cell (i, j)'s triangles are
 * (i,j)-(i+1,j)-(i+1,j+1) and (i,j)-(i+1,j+1)-(i,j+1), numbered (j (nx - 1) + i) * 2 + half */
static v3 grid_vertex(const orc_geometry* g, int i, int j) {
    return mk((float)i * g->cell_x, (float)j * g->cell_y, g->h[(size_t)j * g->nx + i]);
}
static void grid_tri(const orc_geometry* g, uint32_t tri, v3* v0, v3* v1, v3* v2) {
    const int half = (int)(tri & 1u);
    const int cell = (int)(tri >> 1);
    const int i = cell % (g->nx - 1), j = cell / (g->nx - 1);
    *v0 = grid_vertex(g, i, j);
    if (half == 0) {
        *v1 = grid_vertex(g, i + 1, j);
        *v2 = grid_vertex(g, i + 1, j + 1);
    } else {
        *v1 = grid_vertex(g, i + 1, j + 1);
        *v2 = grid_vertex(g, i, j + 1);
    }
}

/* TriangleMesh::triangle_vertices / triangle_normal (triangle_mesh.h:224, 280-290); a grid's
 * normal is HeightGrid::triangle_normal, normalize(cross(v1 - v0, v2 - v0)), +z when degenerate */
static void tri_verts(const orc_geometry* g, uint32_t tri, v3* v0, v3* v1, v3* v2) {
    if (g->grid) grid_tri(g, tri, v0, v1, v2);
    else mesh_tri(g, tri, v0, v1, v2);
}
static v3 tri_normal(const orc_geometry* g, uint32_t tri) {
    if (!g->grid) return ld(&g->normals[3 * tri]);
    v3 v0, v1, v2;
    grid_tri(g, tri, &v0, &v1, &v2);
    const v3 n = cross(sub(v1, v0), sub(v2, v0));
    const float l = len(n);
    return l > 0.0f ? divs(n, l) : mk(0.0f, 0.0f, 1.0f);
}

typedef int (*box_pred)(const void* ctx, const float* mn, const float* mx);
typedef void (*tri_fn)(void* ctx, uint32_t tri);

/* HeightGrid::visit_ (height_grid.h): 64-cell blocks, their 8-cell blocks, their cells, each in
 * row-major order, a block or cell skipped when its box (cells x, y; lowest to highest sample)
 * fails the test; a cell's two triangles in order */
static void grid_visit(const orc_geometry* g, box_pred pred, const void* pctx, tri_fn fn, void* fctx) {
    const int cx = g->nx - 1, cy = g->ny - 1;
#define GH(i, j) g->h[(size_t)(j) * g->nx + (i)]
    for (int gj = 0; gj < g->coarse_h; ++gj)
        for (int gi = 0; gi < g->coarse_w; ++gi) {
            const int c0i = gi * 64, c0j = gj * 64;
            const int c1i = c0i + 64 < cx ? c0i + 64 : cx, c1j = c0j + 64 < cy ? c0j + 64 : cy;
            const float* cr = &g->coarse[2 * (gj * g->coarse_w + gi)];
            float mn[3] = {(float)c0i * g->cell_x, (float)c0j * g->cell_y, cr[0]};
            float mx[3] = {(float)c1i * g->cell_x, (float)c1j * g->cell_y, cr[1]};
            if (!pred(pctx, mn, mx)) continue;
            for (int fj = c0j / 8; fj * 8 < c1j; ++fj)
                for (int fi = c0i / 8; fi * 8 < c1i; ++fi) {
                    const int f0i = fi * 8, f0j = fj * 8;
                    const int f1i = f0i + 8 < cx ? f0i + 8 : cx, f1j = f0j + 8 < cy ? f0j + 8 : cy;
                    const float* fr = &g->fine[2 * (fj * g->fine_w + fi)];
                    float fmn[3] = {(float)f0i * g->cell_x, (float)f0j * g->cell_y, fr[0]};
                    float fmx[3] = {(float)f1i * g->cell_x, (float)f1j * g->cell_y, fr[1]};
                    if (!pred(pctx, fmn, fmx)) continue;
                    for (int j = f0j; j < f1j; ++j)
                        for (int i = f0i; i < f1i; ++i) {
                            /* std::min / std::max of the cell's four samples, as written */
                            const float a = GH(i, j), b = GH(i + 1, j), c = GH(i, j + 1), d = GH(i + 1, j + 1);
                            const float lo1 = b < a ? b : a, lo2 = d < c ? d : c;
                            const float hi1 = a < b ? b : a, hi2 = c < d ? d : c;
                            float cmn[3] = {(float)i * g->cell_x, (float)j * g->cell_y, lo2 < lo1 ? lo2 : lo1};
                            float cmx[3] = {(float)(i + 1) * g->cell_x, (float)(j + 1) * g->cell_y,
                                            hi1 < hi2 ? hi2 : hi1};
                            if (!pred(pctx, cmn, cmx)) continue;
                            fn(fctx, (uint32_t)((j * cx + i) * 2));
                            fn(fctx, (uint32_t)((j * cx + i) * 2 + 1));
                        }
                }
        }
#undef GH
}

typedef struct {
    const orc_geometry* g;
    ray3 ray;
    float best_t;
    uint32_t crossed_tri;
    int crossed;
} raycast_state;

/* the swept crossing callback (cloth_collision.h:243-257) on one triangle */
static void raycast_tri(void* ctx, uint32_t tri) {
    raycast_state* s = (raycast_state*)ctx;
    v3 v0, v1, v2;
    tri_verts(s->g, tri, &v0, &v1, &v2);
    float t = 0.0f;
    if ((ray_triangle(&s->ray, v0, v1, v2, &t) || ray_triangle(&s->ray, v0, v2, v1, &t)) && t < s->best_t) {
        s->best_t = t;
        s->crossed_tri = tri;
        s->crossed = 1;
    }
}

/* MeshBVH::raycast_recursive_ */
static void raycast_node(raycast_state* s, int32_t idx) {
    const orc_bvh_node* node = &s->g->nodes[idx];
    if (!ray_box(&s->ray, node->mn, node->mx)) return;
    if (node->left < 0) {
        for (uint32_t i = 0; i < node->tri_count; ++i) raycast_tri(s, s->g->order[node->tri_start + i]);
    } else {
        raycast_node(s, node->left);
        raycast_node(s, node->right);
    }
}

static int ray_pred(const void* ctx, const float* mn, const float* mx) {
    return ray_box(&((const raycast_state*)ctx)->ray, mn, mx);
}

typedef struct {
    const orc_geometry* g;
    v3 local_p, qmin, qmax;
    float lt2;
    float best_d2;
    v3 best_point, best_delta;
    uint32_t best_tri;
    int hit, any_front;
} query_state;

/* the proximity callback (cloth_collision.h:291-310) on one triangle */
static void query_tri(void* ctx, uint32_t tri) {
    query_state* s = (query_state*)ctx;
    v3 v0, v1, v2;
    tri_verts(s->g, tri, &v0, &v1, &v2);
    const v3 closest = closest_on_triangle(s->local_p, v0, v1, v2);
    const v3 delta = sub(s->local_p, closest);
    const float d2 = dot(delta, delta);
    if (d2 > s->lt2) return;
    if (dot(delta, tri_normal(s->g, tri)) >= 0.0f) s->any_front = 1;
    if (d2 > s->best_d2) return;
    s->best_d2 = d2;
    s->best_point = closest;
    s->best_delta = delta;
    s->best_tri = tri;
    s->hit = 1;
}

/* AABB::overlaps (aabb.h:35-39) of a box with the query box */
static int overlap_pred(const void* ctx, const float* mn, const float* mx) {
    const query_state* s = (const query_state*)ctx;
    return mn[0] <= s->qmax.x && mx[0] >= s->qmin.x && mn[1] <= s->qmax.y && mx[1] >= s->qmin.y &&
           mn[2] <= s->qmax.z && mx[2] >= s->qmin.z;
}

/* MeshBVH::query_recursive_ */
static void query_node(query_state* s, int32_t idx) {
    const orc_bvh_node* node = &s->g->nodes[idx];
    if (!overlap_pred(s, node->mn, node->mx)) return;
    if (node->left < 0) {
        for (uint32_t i = 0; i < node->tri_count; ++i) query_tri(s, s->g->order[node->tri_start + i]);
    } else {
        query_node(s, node->left);
        query_node(s, node->right);
    }
}

/* project_at_pose_'s TriangleMesh branch (cloth_collision.h:205-340) */
static int project_mesh(const pxb_collider* s, v3 pose_pos, q4 pose_rot, float thickness, v3* p,
                        v3* normal_out, float* depth_out, const v3* motion_start) {
    const orc_geometry* g = geometry_of(s, PXB_SHAPE_TRIANGLE_MESH);
    if (!g || (!g->grid && g->n_nodes == 0)) return 0; /* TriangleMesh::empty() */
    const q4 rot = qmul(pose_rot, ldq(s->local_rotation));
    const q4 inv_rot = qinverse(rot);
    const v3 mesh_origin = add(pose_pos, qrot(pose_rot, ld(s->local_center)));
    const float scale = (s->geometry_scale > K_EPSILON) ? s->geometry_scale : 1.0f;
    const v3 local_p = divs(qrot(inv_rot, sub(*p, mesh_origin)), scale);
    const float local_thickness = thickness / scale;

    if (motion_start) {
        const v3 local_start = divs(qrot(inv_rot, sub(*motion_start, mesh_origin)), scale);
        const v3 seg = sub(local_p, local_start);
        const float seg_len = len(seg);
        if (seg_len > local_thickness) {
            raycast_state rs;
            rs.g = g;
            rs.ray.origin = local_start;
            rs.ray.direction = divs(seg, seg_len);
            rs.ray.max_distance = seg_len;
            rs.best_t = seg_len;
            rs.crossed_tri = 0;
            rs.crossed = 0;
            if (g->grid) grid_visit(g, ray_pred, &rs, raycast_tri, &rs);
            else raycast_node(&rs, 0);
            if (rs.crossed) {
                const v3 local_hit = add(rs.ray.origin, mul(rs.ray.direction, rs.best_t));
                v3 face = safe_normalize(tri_normal(g, rs.crossed_tri));
                if (dot(sub(local_start, local_hit), face) < 0.0f) face = neg(face);
                const v3 local_fixed = add(local_hit, mul(face, local_thickness));
                *depth_out = len(sub(local_p, local_fixed)) * scale;
                *p = add(mesh_origin, qrot(rot, mul(local_fixed, scale)));
                *normal_out = qrot(rot, face);
                return 1;
            }
        }
    }

    query_state qs;
    memset(&qs, 0, sizeof(qs));
    qs.g = g;
    qs.local_p = local_p;
    qs.qmin = sub(local_p, mk(local_thickness, local_thickness, local_thickness));
    qs.qmax = add(local_p, mk(local_thickness, local_thickness, local_thickness));
    qs.lt2 = local_thickness * local_thickness;
    qs.best_d2 = local_thickness * local_thickness;
    if (g->grid) grid_visit(g, overlap_pred, &qs, query_tri, &qs);
    else query_node(&qs, 0);
    if (!qs.hit) return 0;
    v3 best_normal;
    if (!qs.any_front) {
        best_normal = safe_normalize(tri_normal(g, qs.best_tri));
    } else if (qs.best_d2 > K_EPSILON * K_EPSILON) {
        best_normal = divs(qs.best_delta, sqrtf(qs.best_d2));
    } else {
        const v3 face = safe_normalize(tri_normal(g, qs.best_tri));
        best_normal = (dot(qs.best_delta, face) < 0.0f) ? neg(face) : face;
    }
    const v3 local_fixed = add(qs.best_point, mul(best_normal, local_thickness));
    *depth_out = len(sub(local_p, local_fixed)) * scale;
    *p = add(mesh_origin, qrot(rot, mul(local_fixed, scale)));
    *normal_out = qrot(rot, best_normal);
    return 1;
}

/* cloth::detail::project_at_pose_ (cloth_collision.h:109-356). */
static int project_at_pose(const pxb_collider* s, v3 pose_pos, q4 pose_rot, v3 sweep,
                           float thickness, v3* p, v3* normal_out, float* depth_out,
                           const v3* motion_start) {
    const int swept = dot(sweep, sweep) > K_EPSILON * K_EPSILON;
    const v3 local_center = ld(s->local_center);
    switch (s->type) {
        case PXB_SHAPE_SPHERE: {
            /* collision::world_sphere (shape.h:160-165) */
            const v3 center = add(pose_pos, qrot(pose_rot, local_center));
            const v3 axis_a = center;
            const v3 axis_b = add(center, sweep);
            const v3 on_axis = swept ? closest_point_on_segment(*p, axis_a, axis_b) : axis_a;
            const v3 d = sub(*p, on_axis);
            const float l = len(d);
            const float target = s->radius + thickness;
            if (l >= target) return 0;
            const v3 n = (l > K_EPSILON) ? divs(d, l) : mk(0.0f, 0.0f, 1.0f);
            *depth_out = target - l;
            *p = add(on_axis, mul(n, target));
            *normal_out = n;
            return 1;
        }
        case PXB_SHAPE_CAPSULE: {
            /* collision::world_capsule (shape.h:177-188) */
            v3 axis_local = mk(0.0f, 0.0f, 0.0f);
            setcomp(&axis_local, s->capsule_axis, 1.0f);
            const v3 axis_world = qrot(qmul(pose_rot, ldq(s->local_rotation)), axis_local);
            const v3 center = add(pose_pos, qrot(pose_rot, local_center));
            const v3 ca = sub(center, mul(axis_world, s->capsule_half_height));
            const v3 cb = add(center, mul(axis_world, s->capsule_half_height));
            const v3 on_axis = closest_point_on_segment(*p, ca, cb);
            const v3 d = sub(*p, on_axis);
            const float l = len(d);
            const float target = s->capsule_radius + thickness;
            if (l >= target) return 0;
            v3 n = d;
            if (l > K_EPSILON) {
                n = divs(d, l);
            } else {
                const v3 axis = safe_normalize(sub(cb, ca));
                n = orthonormal_t1(axis);
            }
            *depth_out = target - l;
            *p = add(on_axis, mul(n, target));
            *normal_out = n;
            return 1;
        }
        case PXB_SHAPE_BOX: {
            /* collision::world_obb (shape.h:168-174), OBB::axes (obb.h:31-36) */
            const v3 center = add(pose_pos, qrot(pose_rot, local_center));
            const q4 orient = qmul(pose_rot, ldq(s->local_rotation));
            v3 ax, ay, az;
            qaxes(orient, &ax, &ay, &az);
            const v3 d = sub(*p, center);
            const v3 local = mk(dot(d, ax), dot(d, ay), dot(d, az));
            const v3 he = ld(s->half_extents);
            const int inside = fabsf(local.x) <= he.x && fabsf(local.y) <= he.y &&
                               fabsf(local.z) <= he.z;
            v3 local_target, local_normal;
            if (inside) {
                const v3 slack = mk(he.x - fabsf(local.x), he.y - fabsf(local.y),
                                    he.z - fabsf(local.z));
                const int axis = (slack.x <= slack.y && slack.x <= slack.z)
                                     ? 0 : (slack.y <= slack.z ? 1 : 2);
                const float sign = (comp(local, axis) >= 0.0f) ? 1.0f : -1.0f;
                local_target = local;
                setcomp(&local_target, axis, sign * (comp(he, axis) + thickness));
                local_normal = mk(0.0f, 0.0f, 0.0f);
                setcomp(&local_normal, axis, sign);
                *depth_out = comp(slack, axis) + thickness;
            } else {
                /* glm::clamp(local, -he, he) = min(max(local, -he), he) */
                local_target = mk(fminr(fmaxr(local.x, -he.x), he.x),
                                  fminr(fmaxr(local.y, -he.y), he.y),
                                  fminr(fmaxr(local.z, -he.z), he.z));
                const v3 delta = sub(local, local_target);
                const float l = len(delta);
                if (l >= thickness) return 0;
                local_normal = (l > K_EPSILON) ? divs(delta, l) : mk(0.0f, 0.0f, 1.0f);
                *depth_out = thickness - l;
                local_target = add(local_target, mul(local_normal, thickness));
            }
            *p = add(add(add(center, mul(ax, local_target.x)), mul(ay, local_target.y)),
                     mul(az, local_target.z));
            {
                const v3 nw = add(add(mul(ax, local_normal.x), mul(ay, local_normal.y)),
                                  mul(az, local_normal.z));
                *normal_out = mul(nw, 1.0f / sqrtf(dot(nw, nw))); /* glm::normalize */
            }
            return 1;
        }
        case PXB_SHAPE_TRIANGLE_MESH:
            return project_mesh(s, pose_pos, pose_rot, thickness, p, normal_out, depth_out, motion_start);
        case PXB_SHAPE_CONVEX_HULL: {
            /* collision::world_posed_hull (sat_hull.h:66-73), probe sphere of radius thickness */
            posed_hull h;
            h.g = geometry_of(s, PXB_SHAPE_CONVEX_HULL);
            if (!h.g) return 0;
            h.position = add(pose_pos, qrot(pose_rot, local_center));
            h.rotation = qmul(pose_rot, ldq(s->local_rotation));
            h.scale = s->geometry_scale;
            v3 point, normal;
            float pen = 0.0f;
            if (!hull_vs_sphere(&h, *p, thickness, &normal, &pen, &point)) return 0;
            *normal_out = normal;
            *p = add(point, mul(normal, thickness));
            *depth_out = pen;
            return 1;
        }
        default:
            return -1;
    }
}

/* cloth::project_particle (cloth_collision.h:386-420). */
static int project_particle(const pxb_collider* col, float thickness, v3* p, v3* normal_out,
                            float* depth_out, const v3* motion_start) {
    if (!col->enabled) return 0;
    if (col->type < PXB_SHAPE_SPHERE || col->type > PXB_SHAPE_CONVEX_HULL) return -1;
    const v3 sweep = ld(col->sweep);
    const int is_swept = dot(sweep, sweep) > K_EPSILON * K_EPSILON;
    const int two_pose = is_swept && (col->type == PXB_SHAPE_BOX || col->type == PXB_SHAPE_CAPSULE);
    const v3 pos = ld(col->position);
    const q4 rot = ldq(col->orientation);
    if (!two_pose) {
        return project_at_pose(col, pos, rot, sweep, thickness, p, normal_out, depth_out, motion_start);
    }
    v3 p_start = *p, n_start = mk(0, 0, 0);
    float d_start = 0.0f;
    const v3 zero = mk(0.0f, 0.0f, 0.0f);
    const int hit_start = project_at_pose(col, pos, rot, zero, thickness, &p_start, &n_start,
                                          &d_start, motion_start);
    v3 p_end = *p, n_end = mk(0, 0, 0);
    float d_end = 0.0f;
    const int hit_end = project_at_pose(col, add(pos, sweep), ldq(col->end_orientation), zero,
                                        thickness, &p_end, &n_end, &d_end, motion_start);
    if (!hit_start && !hit_end) return 0;
    if (hit_end && (!hit_start || d_end > d_start)) {
        *p = p_end; *normal_out = n_end; *depth_out = d_end;
    } else {
        *p = p_start; *normal_out = n_start; *depth_out = d_start;
    }
    return 1;
}

int orc_project_particle(const pxb_collider* collider, float thickness, float p[3],
                         float normal_out[3], float* depth_out, const float* motion_start) {
    v3 pp = ld(p), n = mk(0, 0, 0);
    float d = 0.0f;
    v3 start = mk(0, 0, 0);
    if (motion_start) start = ld(motion_start);
    const int r = project_particle(collider, thickness, &pp, &n, &d, motion_start ? &start : NULL);
    if (r == 1) {
        st(p, pp);
        st(normal_out, n);
        *depth_out = d;
    }
    return r;
}

/* cloth::detail::project_distance (cloth_solver.h:119-138). */
static inline void project_distance(pxb_particle* particles, pxb_constraint* k, float alpha) {
    pxb_particle* pa = &particles[k->a];
    pxb_particle* pb = &particles[k->b];
    const float w = pa->inv_mass + pb->inv_mass;
    if (w <= 0.0f) return;
    const v3 d = sub(ld(pa->position), ld(pb->position));
    const float l = len(d);
    if (l < K_EPSILON) return;
    const v3 n = divs(d, l);
    const float c = l - k->rest_length;
    const float dlambda = (-c - alpha * k->lambda) / (w + alpha);
    k->lambda += dlambda;
    const v3 correction = smul(dlambda, n);
    st(pa->position, add(ld(pa->position), smul(pa->inv_mass, correction)));
    st(pb->position, sub(ld(pb->position), smul(pb->inv_mass, correction)));
}

/* cloth::detail::hash_cell / hash_bucket_count (cloth_solver.h:101-115). */
static inline uint32_t hash_cell(int32_t x, int32_t y, int32_t z, uint32_t buckets) {
    const uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^
                       ((uint32_t)z * 83492791u);
    return h & (buckets - 1u);
}
static uint32_t hash_bucket_count(size_t n) {
    uint32_t b = 16;
    while (b < n * 2u && b < (1u << 22)) b <<= 1;
    return b;
}

/* Stage 6, self-collision (cloth_solver.h:295-366). */
static void self_collide(orc_cloth* c, uint32_t buckets, uint32_t* cell_of, uint32_t* counts,
                         uint32_t* sorted) {
    const uint32_t n = c->n_particles;
    const float d_min = c->params.self_distance;
    const float inv_cell = 1.0f / d_min;
    memset(counts, 0, sizeof(uint32_t) * (buckets + 1));
    for (uint32_t i = 0; i < n; ++i) {
        const v3 p = ld(c->particles[i].position);
        const uint32_t cell = hash_cell((int32_t)floorf(p.x * inv_cell),
                                        (int32_t)floorf(p.y * inv_cell),
                                        (int32_t)floorf(p.z * inv_cell), buckets);
        cell_of[i] = cell;
        ++counts[cell];
    }
    uint32_t running = 0;
    for (uint32_t b = 0; b < buckets; ++b) {
        const uint32_t cnt = counts[b];
        counts[b] = running;
        running += cnt;
    }
    counts[buckets] = running;
    for (uint32_t i = 0; i < n; ++i) sorted[counts[cell_of[i]]++] = i;

    for (uint32_t i = 0; i < n; ++i) {
        pxb_particle* pi = &c->particles[i];
        if (pi->inv_mass == 0.0f) continue;
        const v3 base = mul(ld(pi->position), inv_cell);
        const int32_t cx = (int32_t)floorf(base.x);
        const int32_t cy = (int32_t)floorf(base.y);
        const int32_t cz = (int32_t)floorf(base.z);
        for (int32_t dz = -1; dz <= 1; ++dz)
        for (int32_t dy = -1; dy <= 1; ++dy)
        for (int32_t dx = -1; dx <= 1; ++dx) {
            const uint32_t b = hash_cell(cx + dx, cy + dy, cz + dz, buckets);
            const uint32_t first = (b == 0) ? 0u : counts[b - 1];
            const uint32_t last = counts[b];
            for (uint32_t s = first; s < last; ++s) {
                const uint32_t j = sorted[s];
                if (j <= i) continue;
                if (c->columns > 0) {
                    const int32_t xi = (int32_t)(i % c->columns), yi = (int32_t)(i / c->columns);
                    const int32_t xj = (int32_t)(j % c->columns), yj = (int32_t)(j / c->columns);
                    if (abs(xi - xj) <= 1 && abs(yi - yj) <= 1) continue;
                }
                pxb_particle* pj = &c->particles[j];
                const float w = pi->inv_mass + pj->inv_mass;
                if (w <= 0.0f) continue;
                const v3 d = sub(ld(pi->position), ld(pj->position));
                const float len2 = dot(d, d);
                if (len2 >= d_min * d_min || len2 < K_EPSILON) continue;
                const float l = sqrtf(len2);
                const v3 push = mul(divs(d, l), (d_min - l) / w);
                st(pi->position, add(ld(pi->position), mul(push, pi->inv_mass)));
                st(pj->position, sub(ld(pj->position), mul(push, pj->inv_mass)));
            }
        }
    }
}

/* geometry::AABB over the particles, cloth::compute_bounds (cloth.h:319-326). */
static void compute_bounds(const pxb_particle* particles, uint32_t n, float mn[3], float mx[3]) {
    v3 lo = mk(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f);
    v3 hi = mk(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f);
    for (uint32_t i = 0; i < n; ++i) {
        const v3 p = ld(particles[i].position);
        lo = mk(fminr(lo.x, p.x), fminr(lo.y, p.y), fminr(lo.z, p.z));
        hi = mk(fmaxr(hi.x, p.x), fmaxr(hi.y, p.y), fmaxr(hi.z, p.z));
    }
    st(mn, lo);
    st(mx, hi);
}

int orc_solve_cloth(orc_cloth* c, const pxb_collider* colliders, uint32_t n_colliders,
                    const float gravity_in[3], uint32_t substeps, uint32_t iterations, float h) {
    /* cloth_solver.h:162-194: prologue */
    const uint32_t n = c->n_particles;
    if (n == 0 || h <= 0.0f) return 0;
    for (uint32_t k = 0; k < n_colliders; ++k)
        if (colliders[k].enabled && (colliders[k].type < PXB_SHAPE_SPHERE || colliders[k].type > PXB_SHAPE_CONVEX_HULL))
            return -1;
    const pxb_cloth_params* P = &c->params;
    uint32_t steps = P->substeps ? P->substeps : substeps;
    if (steps < 1) steps = 1;
    uint32_t iters = P->iterations ? P->iterations : iterations;
    if (iters < 1) iters = 1;
    const float hs = h / (float)steps;
    const float inv_hs = 1.0f / hs;

    const int self_collision = P->self_collision && P->self_distance > K_EPSILON;
    const uint32_t buckets = self_collision ? hash_bucket_count(n) : 16u;

    v3* accel = (v3*)calloc(n, sizeof(v3));
    v3* contact_normal = (v3*)calloc(n, sizeof(v3));
    float* contact_depth = (float*)calloc(n, sizeof(float));
    uint32_t* cell_of = self_collision ? (uint32_t*)calloc(n, sizeof(uint32_t)) : NULL;
    uint32_t* counts = self_collision ? (uint32_t*)calloc(buckets + 1, sizeof(uint32_t)) : NULL;
    uint32_t* sorted = self_collision ? (uint32_t*)calloc(n, sizeof(uint32_t)) : NULL;

    const float stretch_alpha = P->stretch_compliance / (hs * hs);
    const float bend_alpha = P->bend_compliance / (hs * hs);

    v3 wind = ld(P->wind);
    if (P->wind_turbulence > 0.0f) {
        const float t = c->time;
        const v3 gust = mk(sinf(t * 1.7f) * cosf(t * 0.9f), sinf(t * 1.1f + 1.3f) * cosf(t * 1.9f),
                           sinf(t * 0.7f + 2.7f) * cosf(t * 1.3f));
        wind = add(wind, smul(P->wind_turbulence, gust));
    }
    const v3 gravity = ld(gravity_in);
    const v3 base_accel = add(mul(gravity, P->gravity_scale), ld(P->external_acceleration));
    const int aero = (P->air_drag > 0.0f || P->air_lift > 0.0f) && c->n_triangle_indices > 0;
    const float max_velocity2 = P->max_velocity * P->max_velocity;

    for (uint32_t step = 0; step < steps; ++step) {
        /* 1. aerodynamics (cloth_solver.h:202-227) */
        memset(accel, 0, sizeof(v3) * n);
        if (aero) {
            for (uint32_t t = 0; t + 2 < c->n_triangle_indices; t += 3) {
                const uint32_t i0 = c->triangles[t], i1 = c->triangles[t + 1],
                               i2 = c->triangles[t + 2];
                const v3 p0 = ld(c->particles[i0].position);
                const v3 e1 = sub(ld(c->particles[i1].position), p0);
                const v3 e2 = sub(ld(c->particles[i2].position), p0);
                const v3 cr = cross(e1, e2);
                const float twice_area = len(cr);
                if (twice_area < K_EPSILON) continue;
                const v3 face_n = divs(cr, twice_area);
                const v3 vsum = add(add(ld(c->particles[i0].velocity), ld(c->particles[i1].velocity)),
                                    ld(c->particles[i2].velocity));
                const v3 v = sub(mul(vsum, 1.0f / 3.0f), wind);
                const float vn = dot(v, face_n);
                const v3 vt = sub(v, smul(vn, face_n));
                const float scale = -0.5f * twice_area * fabsf(vn);
                const v3 inner = add(smul(P->air_drag * vn, face_n), smul(P->air_lift, vt));
                const v3 force = smul(scale, inner);
                const v3 share = mul(force, 1.0f / 3.0f);
                accel[i0] = add(accel[i0], share);
                accel[i1] = add(accel[i1], share);
                accel[i2] = add(accel[i2], share);
            }
        }

        /* 2. integrate (cloth_solver.h:230-240) */
        const float damping_factor = 1.0f / (1.0f + P->damping * hs);
        for (uint32_t i = 0; i < n; ++i) {
            pxb_particle* p = &c->particles[i];
            memcpy(p->prev_position, p->position, sizeof(float) * 3);
            if (p->inv_mass == 0.0f) continue;
            v3 v = ld(p->velocity);
            v = add(v, mul(add(base_accel, mul(accel[i], p->inv_mass)), hs));
            v = mul(v, damping_factor);
            st(p->velocity, v);
            st(p->position, add(ld(p->position), mul(v, hs)));
        }

        /* 3. anchors (cloth_solver.h:245-250) */
        const float alpha_t = (float)(step + 1) / (float)steps;
        for (uint32_t a = 0; a < c->n_anchors; ++a) {
            const pxb_anchor* an = &c->anchors[a];
            if (an->particle >= n) continue;
            st(c->particles[an->particle].position,
               mixv(ld(an->prev_world_position), ld(an->world_position), alpha_t));
        }

        /* 4. constraints (cloth_solver.h:253-271) */
        for (uint32_t k = 0; k < c->n_stretch; ++k) c->stretch[k].lambda = 0.0f;
        for (uint32_t k = 0; k < c->n_bend; ++k) c->bend[k].lambda = 0.0f;
        for (uint32_t it = 0; it < iters; ++it) {
            for (uint32_t b = 0; b < c->n_stretch_batches; ++b) {
                const pxb_batch bt = c->stretch_batches[b];
                const float alpha = c->stretch_batch_compliance
                                        ? c->stretch_batch_compliance[b] / (hs * hs)
                                        : stretch_alpha;
                for (uint32_t i = bt.begin; i < bt.end; ++i)
                    project_distance(c->particles, &c->stretch[i], alpha);
            }
            for (uint32_t b = 0; b < c->n_bend_batches; ++b) {
                const pxb_batch bt = c->bend_batches[b];
                const float alpha = c->bend_batch_compliance
                                        ? c->bend_batch_compliance[b] / (hs * hs)
                                        : bend_alpha;
                for (uint32_t i = bt.begin; i < bt.end; ++i)
                    project_distance(c->particles, &c->bend[i], alpha);
            }
        }

        /* 5. tethers (cloth_solver.h:276-289) */
        for (uint32_t k = 0; k < c->n_tethers; ++k) {
            const pxb_tether* t = &c->tethers[k];
            pxb_particle* p = &c->particles[t->particle];
            if (p->inv_mass == 0.0f) continue;
            const v3 anchor = ld(c->particles[t->anchor].position);
            const v3 d = sub(ld(p->position), anchor);
            const float l = len(d);
            if (l <= t->max_length || l < K_EPSILON) continue;
            st(p->position, add(anchor, mul(d, t->max_length / l)));
        }

        /* 6. self-collision (cloth_solver.h:295-366) */
        if (self_collision) self_collide(c, buckets, cell_of, counts, sorted);

        /* 7. collisions (cloth_solver.h:376-411) */
        memset(contact_normal, 0, sizeof(v3) * n);
        memset(contact_depth, 0, sizeof(float) * n);
        if (n_colliders > 0) {
            const float m = P->thickness;
            for (uint32_t i = 0; i < n; ++i) {
                pxb_particle* p = &c->particles[i];
                if (p->inv_mass == 0.0f) continue;
                for (uint32_t k = 0; k < n_colliders; ++k) {
                    const pxb_collider* col = &colliders[k];
                    const float* lo = col->bounds_min;
                    const float* hi = col->bounds_max;
                    const float* x = p->position;
                    if (x[0] < lo[0] - m || x[0] > hi[0] + m || x[1] < lo[1] - m ||
                        x[1] > hi[1] + m || x[2] < lo[2] - m || x[2] > hi[2] + m) {
                        continue;
                    }
                    v3 pp = ld(p->position), normal = mk(0, 0, 0);
                    float depth = 0.0f;
                    /* prev_position is this substep's start (cloth_solver.h:398-403) */
                    const v3 start = ld(p->prev_position);
                    if (project_particle(col, P->thickness, &pp, &normal, &depth, &start) != 1) continue;
                    st(p->position, pp);
                    contact_normal[i] = add(contact_normal[i], normal);
                    contact_depth[i] += depth;
                }
            }
        }

        /* 8. finalize velocities + friction (cloth_solver.h:414-451) */
        for (uint32_t i = 0; i < n; ++i) {
            pxb_particle* p = &c->particles[i];
            v3 v = mul(sub(ld(p->position), ld(p->prev_position)), inv_hs);
            const float depth = contact_depth[i];
            if (depth > 0.0f) {
                const v3 nsum = contact_normal[i];
                const float nlen = len(nsum);
                if (nlen > K_EPSILON) {
                    const v3 nrm = divs(nsum, nlen);
                    const float vn = dot(v, nrm);
                    const v3 vt = sub(v, smul(vn, nrm));
                    if (vn < 0.0f) v = sub(v, smul(vn, nrm));
                    const float budget = P->friction * depth * inv_hs;
                    const float vt_len = len(vt);
                    if (vt_len > K_EPSILON) v = sub(v, mul(vt, fminr(1.0f, budget / vt_len)));
                }
            }
            const float v2 = dot(v, v);
            if (v2 > max_velocity2) v = mul(v, P->max_velocity / sqrtf(v2));
            st(p->velocity, v);
        }

        c->time += hs;
    }

    /* epilogue (cloth_solver.h:457-459) */
    for (uint32_t a = 0; a < c->n_anchors; ++a)
        memcpy(c->anchors[a].prev_world_position, c->anchors[a].world_position, sizeof(float) * 3);
    compute_bounds(c->particles, n, c->bounds_min, c->bounds_max);

    free(accel);
    free(contact_normal);
    free(contact_depth);
    free(cell_of);
    free(counts);
    free(sorted);
    return 0;
}

void orc_gravity_at(const float gravity[3], const pxb_gravity_source* sources,
                    uint32_t n_sources, const float p_in[3], float out[3]) {
    /* world.h:1186-1190 -> field_at_ world.h:2048-2068 */
    if (n_sources == 0) {
        memcpy(out, gravity, sizeof(float) * 3);
        return;
    }
    const v3 p = ld(p_in);
    float best = 0.0f;
    v3 pull = ld(gravity);
    int found = 0;
    for (uint32_t k = 0; k < n_sources; ++k) {
        const pxb_gravity_source* g = &sources[k];
        const v3 d = sub(ld(g->centre), p);
        const float r = len(d);
        if (g->range > 0.0f && r > g->range) continue;
        if (r < 1e-6f) continue;
        const float a = r <= g->radius ? g->strength
                                       : g->strength * (g->radius / r) * (g->radius / r);
        if (!found || a > best) {
            best = a;
            pull = mul(divs(d, r), a);
            found = 1;
        }
    }
    st(out, found ? pull : ld(gravity));
}

void orc_cloth_centre(const pxb_particle* particles, uint32_t n, float out[3]) {
    v3 sum = mk(0.0f, 0.0f, 0.0f);
    for (uint32_t i = 0; i < n; ++i) sum = add(sum, ld(particles[i].position));
    st(out, n == 0 ? sum : divs(sum, (float)n));
}

int orc_step_cloth(orc_cloth* c, const pxb_collider* colliders, uint32_t n_colliders,
                   const float gravity[3], const pxb_gravity_source* sources,
                   uint32_t n_sources, uint32_t substeps, uint32_t iterations, float h) {
    float g[3];
    if (n_sources == 0) {
        memcpy(g, gravity, sizeof(g));
    } else {
        float centre[3];
        orc_cloth_centre(c->particles, c->n_particles, centre);
        orc_gravity_at(gravity, sources, n_sources, centre, g);
    }
    return orc_solve_cloth(c, colliders, n_colliders, g, substeps, iterations, h);
}

float orc_max_particle_speed(const pxb_particle* particles, uint32_t n) {
    float max2 = 0.0f;
    for (uint32_t i = 0; i < n; ++i) max2 = fmaxr(max2, dot(ld(particles[i].velocity), ld(particles[i].velocity)));
    return sqrtf(max2);
}

uint32_t orc_frame_substeps(float dt, float fixed_dt, uint32_t cloth_substeps) {
    /* world.h:1753-1757 */
    float internal_h = fixed_dt / (float)(cloth_substeps > 1u ? cloth_substeps : 1u);
    if (internal_h < K_EPSILON) internal_h = K_EPSILON;
    long r = lroundf(dt / internal_h);
    uint32_t s = (uint32_t)r;
    if (s < 1u) s = 1u;
    if (s > K_MAX_CLOTH_SUBSTEPS) s = K_MAX_CLOTH_SUBSTEPS;
    return s;
}

/* ---------------------------------------------------------------------------------------- */
/* Hair                                                                                      */
/* ---------------------------------------------------------------------------------------- */

/* hair::k_reference_step (strand_solver.h:63). */
#define K_REFERENCE_STEP (1.0f / 60.0f)

static inline q4 mkq(float w, float x, float y, float z) { q4 q = {x, y, z, w}; return q; }
static inline q4 qscale(q4 q, float s) { return mkq(q.w * s, q.x * s, q.y * s, q.z * s); }
static inline q4 qadd(q4 a, q4 b) { return mkq(a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float qdot(q4 a, q4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }

/* Quaternion for a rotation of `angle` about unit `axis` (glm::angleAxis). */
static q4 angle_axis(float angle, v3 axis) {
    const float s = sinf(angle * 0.5f);
    return mkq(cosf(angle * 0.5f), axis.x * s, axis.y * s, axis.z * s);
}
/* Shortest-arc spherical interpolation with a component-wise lerp when the two rotations are
 * within FLT_EPSILON (glm::slerp, used at strand_solver.h:219-220). */
static q4 slerp(q4 a, q4 b, float t) {
    float cos_theta = qdot(a, b);
    if (cos_theta < 0.0f) {
        b = mkq(-b.w, -b.x, -b.y, -b.z);
        cos_theta = -cos_theta;
    }
    if (cos_theta > 1.0f - 1.19209290e-07f) {
        return mkq(mixf(a.w, b.w, t), mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t));
    }
    const float theta = acosf(cos_theta);
    const q4 r = qadd(qscale(a, sinf((1.0f - t) * theta)), qscale(b, sinf(t * theta)));
    const float sn = sinf(theta);
    return mkq(r.w / sn, r.x / sn, r.y / sn, r.z / sn);
}

/* hair::detail::rotation_between (strand_solver.h:91-105). */
static q4 rotation_between(v3 from, v3 to) {
    const float d = fminr(fmaxr(dot(from, to), -1.0f), 1.0f);
    if (d > 0.999999f) return mkq(1.0f, 0.0f, 0.0f, 0.0f);
    if (d < -0.999999f) {
        v3 axis = cross(mk(0.0f, 0.0f, 1.0f), from);
        if (dot(axis, axis) < 1e-8f) axis = cross(mk(1.0f, 0.0f, 0.0f), from);
        const v3 nrm = mul(axis, 1.0f / sqrtf(dot(axis, axis)));
        return angle_axis(3.14159265358979323846f, nrm);
    }
    const v3 axis = cross(from, to);
    const float l = len(axis);
    if (l < 1e-8f) return mkq(1.0f, 0.0f, 0.0f, 0.0f);
    return angle_axis(acosf(d), divs(axis, l));
}

int orc_solve_strands(orc_strand_set* s, const pxb_collider* colliders, uint32_t n_colliders,
                      const float gravity_in[3], uint32_t substeps, uint32_t iterations, float h) {
    /* strand_solver.h:124-155: prologue */
    const uint32_t n = s->n_particles;
    if (n == 0 || s->n_strands == 0 || h <= 0.0f) return 0;
    for (uint32_t k = 0; k < n_colliders; ++k)
        if (colliders[k].enabled && (colliders[k].type < PXB_SHAPE_SPHERE || colliders[k].type > PXB_SHAPE_CONVEX_HULL))
            return -1;
    const pxb_strand_params* P = &s->params;
    uint32_t steps = P->substeps ? P->substeps : substeps;
    if (steps < 1) steps = 1;
    uint32_t iters = P->iterations ? P->iterations : iterations;
    if (iters < 1) iters = 1;
    const float hs = h / (float)steps;
    const float inv_hs = 1.0f / hs;

    v3* contact_normal = (v3*)calloc(n, sizeof(v3));
    float* contact_depth = (float*)calloc(n, sizeof(float));
    uint8_t* contacted = (uint8_t*)calloc(n, 1);

    const float alpha = P->stretch_compliance * inv_hs * inv_hs;
    const v3 accel = add(mul(ld(gravity_in), P->gravity_scale), ld(P->external_acceleration));
    const float max_speed2 = P->max_velocity * P->max_velocity;
    const float substep_fraction = hs / K_REFERENCE_STEP;
    const float global_per_substep =
        1.0f - powf(1.0f - clampf(P->global_shape, 0.0f, 1.0f) , substep_fraction);
    const float local_per_substep =
        1.0f - powf(1.0f - clampf(P->local_shape, 0.0f, 1.0f), substep_fraction);

    for (uint32_t sub_i = 0; sub_i < steps; ++sub_i) {
        const float t = (float)(sub_i + 1) / (float)steps;

        /* 1 + 2: aerodynamics and integration (strand_solver.h:162-189) */
        for (uint32_t i = 0; i < n; ++i) {
            pxb_particle* p = &s->particles[i];
            if (p->inv_mass <= 0.0f) continue;
            v3 a = accel;
            v3 vel = ld(p->velocity);
            if (P->air_drag > 0.0f) {
                v3 wind = ld(P->wind);
                if (P->wind_turbulence > 0.0f) {
                    const float phase = s->time * 2.3f + p->position[0] * 1.7f +
                                        p->position[1] * 2.1f + p->position[2] * 1.3f;
                    const float amp = P->wind_turbulence * len(ld(P->wind));
                    wind = add(wind, smul(amp, mk(sinf(phase), sinf(phase * 1.37f + 2.1f),
                                                  sinf(phase * 0.81f + 4.2f))));
                }
                a = add(a, mul(sub(wind, vel), P->air_drag));
            }
            vel = add(vel, mul(a, hs));
            vel = mul(vel, 1.0f / (1.0f + P->damping * hs));
            const float v2 = dot(vel, vel);
            if (v2 > max_speed2) vel = mul(vel, P->max_velocity / sqrtf(v2));
            st(p->velocity, vel);
            memcpy(p->prev_position, p->position, sizeof(float) * 3);
            st(p->position, add(ld(p->position), mul(vel, hs)));
        }

        /* 3: roots (strand_solver.h:194-201) */
        for (uint32_t k = 0; k < s->n_strands; ++k) {
            const pxb_strand* sd = &s->strands[k];
            if (sd->count == 0) continue;
            const v3 root = mixv(ld(sd->prev_root_position), ld(sd->root_position), t);
            pxb_particle* p = &s->particles[sd->first];
            memcpy(p->prev_position, p->position, sizeof(float) * 3);
            st(p->position, root);
            st(p->velocity, mk(0.0f, 0.0f, 0.0f));
        }

        /* 4: stretch (strand_solver.h:204-211) */
        for (uint32_t k = 0; k < s->n_stretch; ++k) s->stretch[k].lambda = 0.0f;
        for (uint32_t it = 0; it < iters; ++it) {
            for (uint32_t b = 0; b < s->n_stretch_batches; ++b) {
                const pxb_batch bt = s->stretch_batches[b];
                for (uint32_t ci = bt.begin; ci < bt.end; ++ci)
                    project_distance(s->particles, &s->stretch[ci], alpha);
            }
        }

        /* 5: global shape (strand_solver.h:216-235) */
        if (P->global_shape > 0.0f) {
            for (uint32_t k = 0; k < s->n_strands; ++k) {
                const pxb_strand* sd = &s->strands[k];
                if (sd->count < 2) continue;
                const q4 orientation = slerp(ldq(sd->prev_root_orientation),
                                             ldq(sd->root_orientation), t);
                const v3 root = mixv(ld(sd->prev_root_position), ld(sd->root_position), t);
                const float inv_last = 1.0f / (float)(sd->count - 1);
                for (uint32_t j = 1; j < sd->count; ++j) {
                    const uint32_t i = sd->first + j;
                    pxb_particle* p = &s->particles[i];
                    if (p->inv_mass <= 0.0f) continue;
                    const float along = (float)j * inv_last;
                    const float weight = global_per_substep *
                                         powf(1.0f - along, P->global_shape_falloff);
                    if (weight <= 0.0f) continue;
                    const v3 target = add(root, qrot(orientation, ld(&s->rest_local[3 * i])));
                    st(p->position, mixv(ld(p->position), target, fminr(weight, 1.0f)));
                }
            }
        }

        /* 6: local shape (strand_solver.h:241-272) */
        if (P->local_shape > 0.0f) {
            const float k_local = local_per_substep;
            for (uint32_t k = 0; k < s->n_strands; ++k) {
                const pxb_strand* sd = &s->strands[k];
                if (sd->count < 3) continue;
                for (uint32_t j = 1; j + 1 < sd->count; ++j) {
                    const uint32_t prv = sd->first + j - 1;
                    const uint32_t cur = sd->first + j;
                    const uint32_t nxt = sd->first + j + 1;
                    const v3 rest_prev = ld(&s->rest_offset[3 * cur]);
                    const v3 live_prev = sub(ld(s->particles[cur].position),
                                             ld(s->particles[prv].position));
                    const float rest_len = len(rest_prev);
                    const float live_len = len(live_prev);
                    if (rest_len <= 1e-8f || live_len <= 1e-8f) continue;
                    const q4 turn = rotation_between(divs(rest_prev, rest_len),
                                                     divs(live_prev, live_len));
                    const v3 target = add(ld(s->particles[cur].position),
                                          qrot(turn, ld(&s->rest_offset[3 * nxt])));
                    const v3 delta = mul(sub(target, ld(s->particles[nxt].position)), k_local);
                    pxb_particle* pa = &s->particles[cur];
                    pxb_particle* pb = &s->particles[nxt];
                    const float w = pa->inv_mass + pb->inv_mass;
                    if (w <= 0.0f) continue;
                    st(pb->position, add(ld(pb->position), mul(delta, pb->inv_mass / w)));
                    st(pa->position, sub(ld(pa->position), mul(delta, pa->inv_mass / w)));
                }
            }
        }

        /* 7: collisions, deepest contact kept (strand_solver.h:275-298) */
        memset(contacted, 0, n);
        if (n_colliders > 0) {
            for (uint32_t i = 0; i < n; ++i) {
                pxb_particle* p = &s->particles[i];
                if (p->inv_mass <= 0.0f) continue;
                for (uint32_t k = 0; k < n_colliders; ++k) {
                    v3 pp = ld(p->position), normal = mk(0, 0, 0);
                    float depth = 0.0f;
                    const v3 start = ld(p->prev_position); /* strand_solver.h:283-284 */
                    if (project_particle(&colliders[k], P->thickness, &pp, &normal, &depth, &start) != 1)
                        continue;
                    st(p->position, pp);
                    if (contacted[i] == 0 || depth > contact_depth[i]) {
                        contact_normal[i] = normal;
                        contact_depth[i] = depth;
                    }
                    contacted[i] = 1;
                }
            }
        }

        /* 8: finalize + positional friction (strand_solver.h:301-321) */
        for (uint32_t i = 0; i < n; ++i) {
            pxb_particle* p = &s->particles[i];
            if (p->inv_mass <= 0.0f) continue;
            const v3 prev = ld(p->prev_position);
            st(p->velocity, mul(sub(ld(p->position), prev), inv_hs));
            if (contacted[i] != 0 && P->friction > 0.0f) {
                const v3 normal = contact_normal[i];
                const v3 motion = sub(ld(p->position), prev);
                const v3 tangential = sub(motion, mul(normal, dot(motion, normal)));
                const float t_len = len(tangential);
                if (t_len > K_EPSILON) {
                    const float limit = P->friction * contact_depth[i];
                    const float scale = fmaxr(0.0f, 1.0f - fminr(limit, t_len) / t_len);
                    st(p->position, sub(ld(p->position), mul(tangential, 1.0f - scale)));
                    st(p->velocity, mul(sub(ld(p->position), prev), inv_hs));
                }
            }
        }

        s->time += hs;
    }

    compute_bounds(s->particles, n, s->bounds_min, s->bounds_max);
    free(contact_normal);
    free(contact_depth);
    free(contacted);
    return 0;
}

int orc_step_strands(orc_strand_set* s, const pxb_collider* colliders, uint32_t n_colliders,
                     const float gravity[3], const pxb_gravity_source* sources,
                     uint32_t n_sources, uint32_t substeps, uint32_t iterations, float h) {
    float g[3];
    if (n_sources == 0) {
        memcpy(g, gravity, sizeof(g));
    } else {
        /* world.h:1941: centre = 0.5 * (bounds.min + bounds.max) */
        const v3 centre = smul(0.5f, add(ld(s->bounds_min), ld(s->bounds_max)));
        float c[3];
        st(c, centre);
        orc_gravity_at(gravity, sources, n_sources, c, g);
    }
    return orc_solve_strands(s, colliders, n_colliders, g, substeps, iterations, h);
}

void orc_set_strand_roots(orc_strand_set* s, const float* positions, uint32_t n_positions,
                          const float* orientations, uint32_t n_orientations) {
    const uint32_t n = s->n_strands < n_positions ? s->n_strands : n_positions;
    for (uint32_t i = 0; i < n; ++i) {
        pxb_strand* sd = &s->strands[i];
        memcpy(sd->prev_root_position, sd->root_position, sizeof(float) * 3);
        memcpy(sd->prev_root_orientation, sd->root_orientation, sizeof(float) * 4);
        memcpy(sd->root_position, &positions[3 * i], sizeof(float) * 3);
        if (i < n_orientations) memcpy(sd->root_orientation, &orientations[4 * i], sizeof(float) * 4);
    }
}

int orc_world_step_cloth(orc_cloth* c, const pxb_body_pose* bodies, uint32_t n_bodies, int collider_moving,
                         const pxb_collider* colliders, uint32_t n_colliders, const float gravity[3],
                         const pxb_gravity_source* sources, uint32_t n_sources, float fixed_dt,
                         uint32_t cloth_substeps, uint32_t cloth_iterations, float dt, int* awake,
                         float* sleep_timer) {
    const uint32_t frame_substeps = orc_frame_substeps(dt, fixed_dt, cloth_substeps);
    /* world.h:1765-1772: each anchor's target from its body's live pose */
    int anchor_moved = 0;
    for (uint32_t a = 0; a < c->n_anchors; ++a) {
        pxb_anchor* an = &c->anchors[a];
        const pxb_body_pose* b = NULL;
        if (bodies && an->body_index < n_bodies && bodies[an->body_index].alive &&
            bodies[an->body_index].generation == an->body_generation)
            b = &bodies[an->body_index];
        const v3 world = ld(an->world_position);
        const v3 target = b ? add(ld(b->position), qrot(ldq(b->orientation), ld(an->local_position))) : world;
        const v3 delta = sub(target, world);
        if (dot(delta, delta) > K_EPSILON) anchor_moved = 1;
        st(an->world_position, target);
    }
    /* world.h:1815-1825: the sleep gate */
    if (anchor_moved || collider_moving) {
        *awake = 1;
        *sleep_timer = 0.0f;
    }
    if (!*awake) {
        for (uint32_t a = 0; a < c->n_anchors; ++a)
            memcpy(c->anchors[a].prev_world_position, c->anchors[a].world_position, sizeof(float) * 3);
        return 0;
    }
    const int r = orc_step_cloth(c, colliders, n_colliders, gravity, sources, n_sources, frame_substeps,
                                 cloth_iterations, dt);
    if (r != 0) return r;
    /* world.h:1831-1845: sleep bookkeeping */
    if (orc_max_particle_speed(c->particles, c->n_particles) < c->params.sleep_threshold) {
        *sleep_timer += dt;
        if (*sleep_timer >= c->params.sleep_time) {
            *awake = 0;
            for (uint32_t i = 0; i < c->n_particles; ++i)
                c->particles[i].velocity[0] = c->particles[i].velocity[1] = c->particles[i].velocity[2] = 0.0f;
        }
    } else {
        *sleep_timer = 0.0f;
    }
    return 1;
}

int orc_world_step_strands(orc_strand_set* s, int collider_moving, const pxb_collider* colliders,
                           uint32_t n_colliders, const float gravity[3], const pxb_gravity_source* sources,
                           uint32_t n_sources, float fixed_dt, uint32_t cloth_substeps,
                           uint32_t cloth_iterations, float dt, int* awake, float* sleep_timer) {
    const uint32_t frame_substeps = orc_frame_substeps(dt, fixed_dt, cloth_substeps);
    /* world.h:1872-1878: a root that moved is motion the groom has to answer */
    int root_moved = 0;
    for (uint32_t i = 0; i < s->n_strands && !root_moved; ++i) {
        const v3 delta = sub(ld(s->strands[i].root_position), ld(s->strands[i].prev_root_position));
        if (dot(delta, delta) > K_EPSILON) root_moved = 1;
    }
    /* world.h:1926-1937: the sleep gate */
    if (root_moved || collider_moving) {
        *awake = 1;
        *sleep_timer = 0.0f;
    }
    if (!*awake) {
        for (uint32_t i = 0; i < s->n_strands; ++i) {
            memcpy(s->strands[i].prev_root_position, s->strands[i].root_position, sizeof(float) * 3);
            memcpy(s->strands[i].prev_root_orientation, s->strands[i].root_orientation, sizeof(float) * 4);
        }
        return 0;
    }
    /* world.h:1941-1945 */
    const int r = orc_step_strands(s, colliders, n_colliders, gravity, sources, n_sources, frame_substeps,
                                   cloth_iterations, dt);
    if (r != 0) return r;
    /* world.h:1947-1955: sleep bookkeeping */
    if (orc_max_particle_speed(s->particles, s->n_particles) < s->params.sleep_threshold) {
        *sleep_timer += dt;
        if (*sleep_timer >= s->params.sleep_time) {
            *awake = 0;
            for (uint32_t i = 0; i < s->n_particles; ++i)
                s->particles[i].velocity[0] = s->particles[i].velocity[1] = s->particles[i].velocity[2] = 0.0f;
        }
    } else {
        *sleep_timer = 0.0f;
    }
    return 1;
}
