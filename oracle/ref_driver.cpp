// ref_driver.cpp -- drives the REFERENCE's own cloth / hair code, compiled unmodified.
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile from the reference tree's headers
// (physxcoopa/cloth/*.h, physxcoopa/hair/*.h and their include closure) against the glm-subset
// shim in oracle/glm_shim, into oracle/_ref/libpxbref.so. The tests use it to pin the C
// restatement (xpbd_oracle.c) and the library's host builders to the reference itself, and
// bench.py times it as the reference CPU baseline. It is never linked into the shipped library.
//
// Every function below is a thin adapter: it moves data between the plain reference-layout
// structs of include/physxcoopa_b200.h and the reference's C++ types, then calls the reference.
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include <physxcoopa/cloth/cloth_builder.h>
#include <physxcoopa/cloth/cloth_collision.h>
#include <physxcoopa/cloth/cloth_solver.h>
#include <physxcoopa/hair/strand_builder.h>
#include <physxcoopa/hair/strand_solver.h>

#include "../include/physxcoopa_b200.h"

namespace px = coopa::physx;

static_assert(sizeof(px::cloth::ClothParticle) == sizeof(pxb_particle), "particle layout");
static_assert(sizeof(px::cloth::ClothConstraint) == sizeof(pxb_constraint), "constraint layout");
static_assert(sizeof(px::cloth::ConstraintBatch) == sizeof(pxb_batch), "batch layout");
static_assert(sizeof(px::cloth::ClothTether) == sizeof(pxb_tether), "tether layout");
static_assert(sizeof(px::cloth::ClothAnchor) == sizeof(pxb_anchor), "anchor layout");
static_assert(sizeof(px::hair::Strand) == sizeof(pxb_strand), "strand layout");

namespace {

glm::vec3 v3(const float* p) { return glm::vec3(p[0], p[1], p[2]); }
glm::quat q4(const float* p) { return glm::quat(p[3], p[0], p[1], p[2]); }  // stored x,y,z,w
void put(float* o, const glm::vec3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

px::cloth::ClothParams to_params(const pxb_cloth_params& p) {
    px::cloth::ClothParams r;
    r.stretch_compliance = p.stretch_compliance;
    r.bend_compliance = p.bend_compliance;
    r.damping = p.damping;
    r.thickness = p.thickness;
    r.friction = p.friction;
    r.gravity_scale = p.gravity_scale;
    r.max_velocity = p.max_velocity;
    r.external_acceleration = v3(p.external_acceleration);
    r.wind = v3(p.wind);
    r.wind_turbulence = p.wind_turbulence;
    r.air_drag = p.air_drag;
    r.air_lift = p.air_lift;
    r.self_collision = p.self_collision != 0;
    r.self_distance = p.self_distance;
    r.tether_scale = p.tether_scale;
    r.substeps = p.substeps;
    r.iterations = p.iterations;
    r.sleep_threshold = p.sleep_threshold;
    r.sleep_time = p.sleep_time;
    r.layer = p.layer;
    return r;
}

void from_params(const px::cloth::ClothParams& r, pxb_cloth_params& p) {
    std::memset(&p, 0, sizeof(p));
    p.stretch_compliance = r.stretch_compliance;
    p.bend_compliance = r.bend_compliance;
    p.damping = r.damping;
    p.thickness = r.thickness;
    p.friction = r.friction;
    p.gravity_scale = r.gravity_scale;
    p.max_velocity = r.max_velocity;
    put(p.external_acceleration, r.external_acceleration);
    put(p.wind, r.wind);
    p.wind_turbulence = r.wind_turbulence;
    p.air_drag = r.air_drag;
    p.air_lift = r.air_lift;
    p.self_collision = r.self_collision ? 1 : 0;
    p.self_distance = r.self_distance;
    p.tether_scale = r.tether_scale;
    p.substeps = r.substeps;
    p.iterations = r.iterations;
    p.sleep_threshold = r.sleep_threshold;
    p.sleep_time = r.sleep_time;
    p.layer = r.layer;
}

px::hair::StrandParams to_params(const pxb_strand_params& p) {
    px::hair::StrandParams r;
    r.stretch_compliance = p.stretch_compliance;
    r.global_shape = p.global_shape;
    r.global_shape_falloff = p.global_shape_falloff;
    r.local_shape = p.local_shape;
    r.damping = p.damping;
    r.thickness = p.thickness;
    r.friction = p.friction;
    r.gravity_scale = p.gravity_scale;
    r.max_velocity = p.max_velocity;
    r.external_acceleration = v3(p.external_acceleration);
    r.wind = v3(p.wind);
    r.wind_turbulence = p.wind_turbulence;
    r.air_drag = p.air_drag;
    r.substeps = p.substeps;
    r.iterations = p.iterations;
    r.sleep_threshold = p.sleep_threshold;
    r.sleep_time = p.sleep_time;
    r.layer = p.layer;
    return r;
}

// Collider geometry by pxb_collider::geometry id: the reference's own ConvexHull and
// TriangleMesh objects (the mesh's constructor builds its MeshBVH).
std::map<uint32_t, std::unique_ptr<px::geometry::ConvexHull>> g_hulls;
std::map<uint32_t, std::unique_ptr<px::geometry::TriangleMesh>> g_meshes;

template <class M>
auto* find_geometry(M& m, uint32_t id) {
    auto it = m.find(id);
    return it == m.end() ? nullptr : it->second.get();
}

// A collider snapshot owns the collision::Shape its ClothCollider points at.
struct RefColliders {
    std::vector<px::collision::Shape> shapes;
    std::vector<px::cloth::ClothCollider> colliders;
    explicit RefColliders(const pxb_collider* c, uint32_t n) {
        shapes.resize(n);
        colliders.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            px::collision::Shape& s = shapes[i];
            s.enabled = c[i].enabled != 0;
            s.type = static_cast<px::collision::ShapeType>(c[i].type);
            s.local_center = v3(c[i].local_center);
            s.local_rotation = q4(c[i].local_rotation);
            s.radius = c[i].radius;
            s.half_extents = v3(c[i].half_extents);
            s.capsule_radius = c[i].capsule_radius;
            s.capsule_half_height = c[i].capsule_half_height;
            s.capsule_axis = c[i].capsule_axis;
            if (c[i].type == PXB_SHAPE_CONVEX_HULL) {
                s.hull = find_geometry(g_hulls, c[i].geometry);
                s.hull_scale = c[i].geometry_scale;
            } else if (c[i].type == PXB_SHAPE_TRIANGLE_MESH) {
                s.mesh = find_geometry(g_meshes, c[i].geometry);
                s.mesh_scale = c[i].geometry_scale;
            }
            px::cloth::ClothCollider& k = colliders[i];
            k.shape = &shapes[i];
            k.position = v3(c[i].position);
            k.orientation = q4(c[i].orientation);
            k.sweep = v3(c[i].sweep);
            k.end_orientation = q4(c[i].end_orientation);
            k.bounds.min = v3(c[i].bounds_min);
            k.bounds.max = v3(c[i].bounds_max);
        }
    }
};

// splitmix64 -> uniform float in [-amp, amp]; the same stream the library's builder uses.
struct Jitter {
    uint64_t state;
    float next(float amp) {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const float u = static_cast<float>(z >> 40) * (1.0f / 16777216.0f);
        return (u * 2.0f - 1.0f) * amp;
    }
};

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------------------------
// Cloth
// ---------------------------------------------------------------------------------------------

// make_grid_cloth (cloth_builder.h:81-219), then the optional seeded jitter with rest lengths
// re-captured by the builder's own formula (cloth_builder.h:119) and bounds recomputed.
void* pxbref_cloth_make_grid(const pxb_grid_cloth_desc* d) {
    px::cloth::GridClothDesc g;
    g.columns = d->columns;
    g.rows = d->rows;
    g.width = d->width;
    g.height = d->height;
    g.center = v3(d->center);
    g.orientation = q4(d->orientation);
    g.total_mass = d->total_mass;
    g.shear = d->shear != 0;
    g.params = to_params(d->params);
    auto* c = new px::cloth::Cloth(px::cloth::make_grid_cloth(g));
    if (d->jitter > 0.0f) {
        Jitter j{d->jitter_seed};
        for (auto& p : c->particles) {
            p.position.x += j.next(d->jitter);
            p.position.y += j.next(d->jitter);
            p.position.z += j.next(d->jitter);
            p.prev_position = p.position;
        }
        for (auto& k : c->stretch)
            k.rest_length = glm::length(c->particles[k.a].position - c->particles[k.b].position);
        for (auto& k : c->bend)
            k.rest_length = glm::length(c->particles[k.a].position - c->particles[k.b].position);
        c->bounds = px::cloth::compute_bounds(*c);
    }
    return c;
}

// A reference Cloth holding a copy of the given arrays.
void* pxbref_cloth_from_desc(const pxb_cloth_desc* d) {
    auto* c = new px::cloth::Cloth();
    auto copy = [](auto& dst, const auto* src, uint32_t n) {
        dst.resize(n);
        if (n) std::memcpy(dst.data(), src, sizeof(dst[0]) * n);
    };
    copy(c->particles, d->particles, d->n_particles);
    copy(c->stretch, d->stretch, d->n_stretch);
    copy(c->stretch_batches, d->stretch_batches, d->n_stretch_batches);
    copy(c->bend, d->bend, d->n_bend);
    copy(c->bend_batches, d->bend_batches, d->n_bend_batches);
    copy(c->tethers, d->tethers, d->n_tethers);
    copy(c->anchors, d->anchors, d->n_anchors);
    copy(c->triangles, d->triangles, d->n_triangle_indices);
    c->columns = d->columns;
    c->rows = d->rows;
    c->params = to_params(d->params);
    c->time = d->time;
    c->valid = true;
    c->bounds = px::cloth::compute_bounds(*c);
    return c;
}

void pxbref_cloth_free(void* h) { delete static_cast<px::cloth::Cloth*>(h); }

uint32_t pxbref_cloth_pin_static(void* h, const float* point, float radius) {
    return px::cloth::pin_static(*static_cast<px::cloth::Cloth*>(h), v3(point), radius);
}

// cloth::pin_to_body (cloth_builder.h:235-258) against a body at the given pose.
uint32_t pxbref_cloth_pin_to_body(void* h, uint32_t body_index, uint32_t body_generation, const float* body_position,
                                  const float* body_orientation, const float* point, float radius) {
    px::dynamics::BodyId id;
    id.index = body_index;
    id.generation = body_generation;
    px::dynamics::Body body;
    body.position = v3(body_position);
    body.orientation = q4(body_orientation);
    return px::cloth::pin_to_body(*static_cast<px::cloth::Cloth*>(h), id, body, v3(point), radius);
}

void pxbref_cloth_build_tethers(void* h) {
    px::cloth::build_tethers(*static_cast<px::cloth::Cloth*>(h));
}

// Pointers into the reference Cloth's own vectors (layouts are byte-identical).
void pxbref_cloth_view(void* h, pxb_cloth_desc* out) {
    auto* c = static_cast<px::cloth::Cloth*>(h);
    std::memset(out, 0, sizeof(*out));
    out->particles = reinterpret_cast<const pxb_particle*>(c->particles.data());
    out->n_particles = static_cast<uint32_t>(c->particles.size());
    out->stretch = reinterpret_cast<const pxb_constraint*>(c->stretch.data());
    out->n_stretch = static_cast<uint32_t>(c->stretch.size());
    out->stretch_batches = reinterpret_cast<const pxb_batch*>(c->stretch_batches.data());
    out->n_stretch_batches = static_cast<uint32_t>(c->stretch_batches.size());
    out->bend = reinterpret_cast<const pxb_constraint*>(c->bend.data());
    out->n_bend = static_cast<uint32_t>(c->bend.size());
    out->bend_batches = reinterpret_cast<const pxb_batch*>(c->bend_batches.data());
    out->n_bend_batches = static_cast<uint32_t>(c->bend_batches.size());
    out->tethers = reinterpret_cast<const pxb_tether*>(c->tethers.data());
    out->n_tethers = static_cast<uint32_t>(c->tethers.size());
    out->anchors = reinterpret_cast<const pxb_anchor*>(c->anchors.data());
    out->n_anchors = static_cast<uint32_t>(c->anchors.size());
    out->triangles = c->triangles.data();
    out->n_triangle_indices = static_cast<uint32_t>(c->triangles.size());
    out->columns = c->columns;
    out->rows = c->rows;
    from_params(c->params, out->params);
    out->time = c->time;
}

void pxbref_cloth_bounds(void* h, float* out6) {
    auto* c = static_cast<px::cloth::Cloth*>(h);
    put(out6, c->bounds.min);
    put(out6 + 3, c->bounds.max);
}

// cloth::solve_cloth, serial overload (cloth_solver.h:463-467).
void pxbref_solve_cloth(void* h, const pxb_collider* colliders, uint32_t n_colliders,
                        const float* gravity, uint32_t substeps, uint32_t iterations, float dt) {
    auto* c = static_cast<px::cloth::Cloth*>(h);
    RefColliders rc(colliders, n_colliders);
    px::cloth::ClothSolverScratch scratch;
    px::cloth::solve_cloth(*c, rc.colliders, v3(gravity), substeps, iterations, dt, scratch);
}

// Registers the reference's ConvexHull (its fields as given) under `id`.
int pxbref_geometry_set_hull(uint32_t id, const pxb_hull_desc* d) {
    auto h = std::make_unique<px::geometry::ConvexHull>();
    for (uint32_t i = 0; i < d->n_vertices; ++i) h->vertices.push_back(v3(&d->vertices[3 * i]));
    for (uint32_t f = 0; f < d->n_faces; ++f) {
        const float* q = &d->face_planes[4 * f];
        h->face_planes.push_back(glm::vec4(q[0], q[1], q[2], q[3]));
    }
    h->face_starts.assign(d->face_starts, d->face_starts + d->n_faces + 1);
    h->face_vertices.assign(d->face_vertices, d->face_vertices + d->face_starts[d->n_faces]);
    g_hulls[id] = std::move(h);
    return 0;
}

// Registers a TriangleMesh made by its four-argument constructor (normals NULL: from_triangles).
int pxbref_geometry_set_mesh(uint32_t id, const pxb_mesh_desc* d) {
    std::vector<glm::vec3> verts;
    for (uint32_t i = 0; i < d->n_vertices; ++i) verts.push_back(v3(&d->vertices[3 * i]));
    std::vector<uint32_t> idx(d->indices, d->indices + d->n_indices);
    if (!d->normals) {
        g_meshes[id] = std::make_unique<px::geometry::TriangleMesh>(
            px::geometry::TriangleMesh::from_triangles(verts, idx));
        return 0;
    }
    const uint32_t T = d->n_indices / 3;
    std::vector<glm::vec3> normals;
    for (uint32_t t = 0; t < T; ++t) normals.push_back(v3(&d->normals[3 * t]));
    std::vector<px::geometry::TriangleAdjacency> adjacency(T);
    g_meshes[id] = std::make_unique<px::geometry::TriangleMesh>(std::move(verts), std::move(idx), std::move(normals),
                                                                std::move(adjacency));
    return 0;
}

// Registers TriangleMesh::from_height_grid over the reference's own HeightGrid (height_grid.h).
int pxbref_geometry_set_height_grid(uint32_t id, int nx, int ny, float cell_x, float cell_y, const float* heights,
                                    uint32_t n_heights) {
    auto grid = std::make_shared<const px::geometry::HeightGrid>(
        nx, ny, glm::vec2(cell_x, cell_y), std::vector<float>(heights, heights + n_heights));
    g_meshes[id] = std::make_unique<px::geometry::TriangleMesh>(px::geometry::TriangleMesh::from_height_grid(grid));
    return 0;
}

void pxbref_geometry_clear() {
    g_hulls.clear();
    g_meshes.clear();
}

// geometry::build_convex_hull (convex_hull.h:211) over `count` points: the reference's own hull
// builder, so tests can use hulls exactly as the reference makes them. Writes up to the given
// capacities and returns the face count (0 for a degenerate cloud, -1 when a capacity is short).
int pxbref_build_convex_hull(const float* points, uint32_t count, float* vertices, uint32_t cap_vertices,
                             uint32_t* n_vertices, float* planes, uint32_t cap_faces, uint32_t* starts,
                             uint32_t* face_vertices, uint32_t cap_face_vertices) {
    std::vector<glm::vec3> pts;
    for (uint32_t i = 0; i < count; ++i) pts.push_back(v3(&points[3 * i]));
    px::geometry::ConvexHull h;
    if (!px::geometry::build_convex_hull(pts.data(), pts.size(), h)) return 0;
    if (h.vertices.size() > cap_vertices || h.face_planes.size() > cap_faces ||
        h.face_vertices.size() > cap_face_vertices)
        return -1;
    for (size_t i = 0; i < h.vertices.size(); ++i) put(&vertices[3 * i], h.vertices[i]);
    for (size_t f = 0; f < h.face_planes.size(); ++f) {
        planes[4 * f] = h.face_planes[f].x;
        planes[4 * f + 1] = h.face_planes[f].y;
        planes[4 * f + 2] = h.face_planes[f].z;
        planes[4 * f + 3] = h.face_planes[f].w;
    }
    for (size_t f = 0; f < h.face_starts.size(); ++f) starts[f] = h.face_starts[f];
    for (size_t i = 0; i < h.face_vertices.size(); ++i) face_vertices[i] = h.face_vertices[i];
    *n_vertices = static_cast<uint32_t>(h.vertices.size());
    return static_cast<int>(h.face_planes.size());
}

// cloth::project_particle (cloth_collision.h:386-420) on one point.
int pxbref_project_particle(const pxb_collider* collider, float thickness, float* p,
                            float* normal_out, float* depth_out, const float* motion_start) {
    RefColliders rc(collider, 1);
    glm::vec3 pp = v3(p), n(0.0f);
    float depth = 0.0f;
    glm::vec3 ms = motion_start ? v3(motion_start) : glm::vec3(0.0f);
    const bool hit = px::cloth::project_particle(rc.colliders[0], thickness, pp, n, depth,
                                                 motion_start ? &ms : nullptr);
    if (hit) {
        put(p, pp);
        put(normal_out, n);
        *depth_out = depth;
    }
    return hit ? 1 : 0;
}

// CPU baseline: advances every listed cloth by `steps` calls of solve_cloth on `threads` host
// threads, whole cloths handed out from a shared counter and each solved serially -- the
// reference's own SerialDispatch per cloth. Returns wall seconds.
// PhysicsWorld::cloth_centre_ and field_at_ (world.h:2048-2076) are private members of the world;
// the timing driver restates them over the same sources so each cloth is stepped with the
// gravity step_cloths_ would give it (world.h:1833).
static glm::vec3 bench_gravity(const px::cloth::Cloth& c, const glm::vec3& uniform,
                               const pxb_gravity_source* src, uint32_t n_src) {
    if (n_src == 0) return uniform;
    glm::vec3 sum(0.0f);
    for (const px::cloth::ClothParticle& p : c.particles) sum += p.position;
    const glm::vec3 centre = c.particles.empty() ? sum : sum / static_cast<float>(c.particles.size());
    float best = 0.0f;
    glm::vec3 pull = uniform;
    bool found = false;
    for (uint32_t k = 0; k < n_src; ++k) {
        const glm::vec3 d = v3(src[k].centre) - centre;
        const float r = glm::length(d);
        if (src[k].range > 0.0f && r > src[k].range) continue;
        if (r < 1e-6f) continue;
        const float a = r <= src[k].radius ? src[k].strength
                                           : src[k].strength * (src[k].radius / r) * (src[k].radius / r);
        if (!found || a > best) {
            best = a;
            pull = d / r * a;
            found = true;
        }
    }
    return found ? pull : uniform;
}

// Steps n reference cloths `steps` times over `threads` host threads (an atomic work counter,
// one solve_cloth per cloth per step, as PhysicsWorld::step_cloths_ with a thread-pool
// dispatcher). Sources (optional, per-cloth offsets) select each cloth's gravity. Returns the
// wall-clock seconds.
double pxbref_bench_cloths(void** handles, uint32_t n, const pxb_collider* colliders,
                           const uint32_t* collider_offsets, const pxb_gravity_source* sources,
                           const uint32_t* source_offsets, const float* gravity, uint32_t substeps,
                           uint32_t iterations, float dt, uint32_t steps, uint32_t threads) {
    if (threads < 1) threads = 1;
    std::vector<RefColliders> cols;
    cols.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t b = collider_offsets ? collider_offsets[i] : 0;
        const uint32_t e = collider_offsets ? collider_offsets[i + 1] : 0;
        cols.emplace_back(colliders + b, e - b);
    }
    const glm::vec3 g0 = v3(gravity);
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t s = 0; s < steps; ++s) {
        std::atomic<uint32_t> next{0};
        auto worker = [&]() {
            px::cloth::ClothSolverScratch scratch;
            for (;;) {
                const uint32_t i = next.fetch_add(1);
                if (i >= n) break;
                px::cloth::Cloth& c = *static_cast<px::cloth::Cloth*>(handles[i]);
                const uint32_t sb = source_offsets ? source_offsets[i] : 0;
                const uint32_t se = source_offsets ? source_offsets[i + 1] : 0;
                const glm::vec3 g = bench_gravity(c, g0, sources ? sources + sb : nullptr, se - sb);
                px::cloth::solve_cloth(c, cols[i].colliders, g, substeps, iterations, dt, scratch);
            }
        };
        if (threads == 1) {
            worker();
        } else {
            std::vector<std::thread> pool;
            for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(worker);
            for (auto& t : pool) t.join();
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// ---------------------------------------------------------------------------------------------
// Hair
// ---------------------------------------------------------------------------------------------

// make_strands (strand_builder.h:58-127) from n_strands polylines: counts[i] points each, packed
// in `points` (3 floats per point), one root orientation (x,y,z,w) and particle mass per strand.
void* pxbref_strands_make(uint32_t n_strands, const uint32_t* counts, const float* points,
                          const float* root_orientations, const float* particle_masses,
                          const pxb_strand_params* params) {
    std::vector<px::hair::StrandDesc> descs(n_strands);
    size_t off = 0;
    for (uint32_t i = 0; i < n_strands; ++i) {
        for (uint32_t k = 0; k < counts[i]; ++k, ++off) descs[i].points.push_back(v3(points + 3 * off));
        if (root_orientations) descs[i].root_orientation = q4(root_orientations + 4 * i);
        if (particle_masses) descs[i].particle_mass = particle_masses[i];
    }
    return new px::hair::StrandSet(px::hair::make_strands(descs, to_params(*params)));
}

void pxbref_strands_free(void* h) { delete static_cast<px::hair::StrandSet*>(h); }

void pxbref_strands_view(void* h, pxb_strand_set_desc* out) {
    auto* s = static_cast<px::hair::StrandSet*>(h);
    std::memset(out, 0, sizeof(*out));
    out->particles = reinterpret_cast<const pxb_particle*>(s->particles.data());
    out->n_particles = static_cast<uint32_t>(s->particles.size());
    out->stretch = reinterpret_cast<const pxb_constraint*>(s->stretch.data());
    out->n_stretch = static_cast<uint32_t>(s->stretch.size());
    out->stretch_batches = reinterpret_cast<const pxb_batch*>(s->stretch_batches.data());
    out->n_stretch_batches = static_cast<uint32_t>(s->stretch_batches.size());
    out->rest_local = reinterpret_cast<const float*>(s->rest_local.data());
    out->rest_offset = reinterpret_cast<const float*>(s->rest_offset.data());
    out->strands = reinterpret_cast<const pxb_strand*>(s->strands.data());
    out->n_strands = static_cast<uint32_t>(s->strands.size());
    out->time = s->time;
}

void pxbref_strands_bounds(void* h, float* out6) {
    auto* s = static_cast<px::hair::StrandSet*>(h);
    put(out6, s->bounds.min);
    put(out6 + 3, s->bounds.max);
}

void pxbref_strands_set_roots(void* h, const float* positions, uint32_t n_positions,
                              const float* orientations, uint32_t n_orientations) {
    std::vector<glm::vec3> pos(n_positions);
    for (uint32_t i = 0; i < n_positions; ++i) pos[i] = v3(positions + 3 * i);
    std::vector<glm::quat> rot(n_orientations);
    for (uint32_t i = 0; i < n_orientations; ++i) rot[i] = q4(orientations + 4 * i);
    px::hair::set_strand_roots(*static_cast<px::hair::StrandSet*>(h), pos, rot);
}

void pxbref_solve_strands(void* h, const pxb_collider* colliders, uint32_t n_colliders,
                          const float* gravity, uint32_t substeps, uint32_t iterations, float dt) {
    RefColliders rc(colliders, n_colliders);
    px::hair::StrandSolverScratch scratch;
    px::hair::solve_strands(*static_cast<px::hair::StrandSet*>(h), rc.colliders, v3(gravity),
                            substeps, iterations, dt, scratch);
}

}  // extern "C"
