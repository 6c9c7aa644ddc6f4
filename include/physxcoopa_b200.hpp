// physxcoopa_b200.hpp -- C++ drop-in facade over the C-ABI for physxcoopa code.
//
// Include this AFTER the physxcoopa headers (it uses cloth::Cloth, cloth::ClothCollider,
// hair::StrandSet, collision::Shape). It offers the reference's own solve signatures
//
//   cloth::solve_cloth(Cloth&, colliders, gravity, substeps, iterations, h, scratch[, dispatch])
//        (physxcoopa/cloth/cloth_solver.h:158-161, 463-467)
//   hair::solve_strands(StrandSet&, colliders, gravity, substeps, iterations, h, scratch)
//        (physxcoopa/hair/strand_solver.h:121-123)
//
// in namespace pxb::b200, backed by the device solver: a call site changes only its namespace
// (px::cloth::solve_cloth(c, cols, g, 4, 10, h, scratch) becomes pxb::b200::solve_cloth(c, cols,
// g, 4, 10, h, scratch)). Those overloads run on the calling thread's own context
// (thread_device(): CUDA device 0 unless set_thread_device chose another); the overloads that
// take a Device& first use the caller's. The Cloth / StrandSet is advanced in
// place exactly as the reference advances it; the scratch and dispatcher arguments are accepted
// for signature compatibility and not used (the device needs neither). Vectors are handed to
// the library as they are: pxb_particle, pxb_constraint, pxb_anchor... are the reference's own
// byte layouts (static_asserts below). Errors throw std::runtime_error with the library's
// message -- the reference throws nothing, so a caller that cannot accept an exception should
// call the C-ABI directly and read pxb_status.
#ifndef PHYSXCOOPA_B200_HPP
#define PHYSXCOOPA_B200_HPP

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "physxcoopa_b200.h"

namespace pxb {
namespace b200 {

static_assert(sizeof(coopa::physx::cloth::ClothParticle) == sizeof(pxb_particle), "particle layout");
static_assert(sizeof(coopa::physx::cloth::ClothConstraint) == sizeof(pxb_constraint), "constraint layout");
static_assert(sizeof(coopa::physx::cloth::ConstraintBatch) == sizeof(pxb_batch), "batch layout");
static_assert(sizeof(coopa::physx::cloth::ClothTether) == sizeof(pxb_tether), "tether layout");
static_assert(sizeof(coopa::physx::cloth::ClothAnchor) == sizeof(pxb_anchor), "anchor layout");
static_assert(sizeof(coopa::physx::hair::Strand) == sizeof(pxb_strand), "strand layout");

// One context per thread that steps cloths (the C-ABI is single-threaded per context).
class Device {
public:
    explicit Device(int device = 0) : index_(device) {
        if (pxb_context_create(device, &ctx_) != PXB_OK) throw std::runtime_error("pxb_context_create failed");
    }
    int index() const { return index_; }
    ~Device() { pxb_context_destroy(ctx_); }
    Device(const Device&) = delete;
    Device& operator=(const Device&) = delete;
    pxb_context* get() const { return ctx_; }
    void check(pxb_status s, const char* what) const {
        if (s != PXB_OK) throw std::runtime_error(std::string(what) + ": " + pxb_last_error(ctx_));
    }

    // The device copy of a Shape's hull (Shape::hull, shape.h:97), registered the first time a
    // collider names it. Like the reference's non-owning pointer, the object is assumed not to
    // change afterwards: after editing or freeing one, call forget_geometry.
    uint32_t geometry_id(const coopa::physx::geometry::ConvexHull* h) {
        if (!h) return 0;
        auto it = geometry_.find(h);
        if (it != geometry_.end()) return it->second;
        pxb_hull_desc d;
        std::memset(&d, 0, sizeof(d));
        d.vertices = reinterpret_cast<const float*>(h->vertices.data());
        d.n_vertices = static_cast<uint32_t>(h->vertices.size());
        d.face_planes = reinterpret_cast<const float*>(h->face_planes.data());
        d.n_faces = static_cast<uint32_t>(h->face_planes.size());
        d.face_starts = h->face_starts.data();
        d.face_vertices = h->face_vertices.data();
        uint32_t id = 0;
        check(pxb_geometry_create_hull(ctx_, &d, &id), "register convex hull");
        geometry_[h] = id;
        return id;
    }
    // The device copy of a Shape's triangle mesh (Shape::mesh, shape.h:85). A height-grid mesh
    // (TriangleMesh::from_height_grid, triangle_mesh.h:210) registers its grid's samples.
    uint32_t geometry_id(const coopa::physx::geometry::TriangleMesh* m) {
        if (!m) return 0;
        auto it = geometry_.find(m);
        if (it != geometry_.end()) return it->second;
        if (const coopa::physx::geometry::HeightGrid* g = m->height_grid()) {
            pxb_height_grid_desc hd;
            std::memset(&hd, 0, sizeof(hd));
            hd.nx = static_cast<uint32_t>(g->nx());
            hd.ny = static_cast<uint32_t>(g->ny());
            hd.cell_x = g->cell().x;
            hd.cell_y = g->cell().y;
            hd.heights = g->heights().data();
            hd.n_heights = static_cast<uint32_t>(g->heights().size());
            uint32_t id = 0;
            check(pxb_geometry_create_height_grid(ctx_, &hd, &id), "register height grid");
            geometry_[m] = id;
            return id;
        }
        pxb_mesh_desc d;
        std::memset(&d, 0, sizeof(d));
        d.vertices = reinterpret_cast<const float*>(m->vertices().data());
        d.n_vertices = static_cast<uint32_t>(m->vertices().size());
        d.indices = m->indices().data();
        d.n_indices = static_cast<uint32_t>(m->indices().size());
        d.normals = reinterpret_cast<const float*>(m->normals().data());
        uint32_t id = 0;
        check(pxb_geometry_create_mesh(ctx_, &d, &id), "register triangle mesh");
        geometry_[m] = id;
        return id;
    }
    void forget_geometry(const void* object) {
        auto it = geometry_.find(object);
        if (it == geometry_.end()) return;
        check(pxb_geometry_destroy(ctx_, it->second), "forget geometry");
        geometry_.erase(it);
    }

private:
    int index_ = 0;
    pxb_context* ctx_ = nullptr;
    std::unordered_map<const void*, uint32_t> geometry_;
};

inline void put3(float* o, const glm::vec3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }
inline void put4(float* o, const glm::quat& q) { o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w; }

// cloth::ClothCollider + the collision::Shape it points at -> the C-ABI snapshot (a mesh or
// hull names the device copy of its geometry).
inline pxb_collider to_collider(Device& dev, const coopa::physx::cloth::ClothCollider& c) {
    pxb_collider o;
    std::memset(&o, 0, sizeof(o));
    const coopa::physx::collision::Shape* s = c.shape;
    o.enabled = (s && s->enabled) ? 1 : 0;
    if (s) {
        o.type = static_cast<int32_t>(s->type);
        put3(o.local_center, s->local_center);
        put4(o.local_rotation, s->local_rotation);
        o.radius = s->radius;
        put3(o.half_extents, s->half_extents);
        o.capsule_radius = s->capsule_radius;
        o.capsule_half_height = s->capsule_half_height;
        o.capsule_axis = s->capsule_axis;
        if (s->type == coopa::physx::collision::ShapeType::ConvexHull) {
            o.geometry = dev.geometry_id(s->hull);
            o.geometry_scale = s->hull_scale;
        } else if (s->type == coopa::physx::collision::ShapeType::TriangleMesh) {
            o.geometry = dev.geometry_id(s->mesh);
            o.geometry_scale = s->mesh_scale;
        }
    }
    put3(o.position, c.position);
    put4(o.orientation, c.orientation);
    put3(o.sweep, c.sweep);
    put4(o.end_orientation, c.end_orientation);
    put3(o.bounds_min, c.bounds.min);
    put3(o.bounds_max, c.bounds.max);
    return o;
}

inline pxb_cloth_params to_params(const coopa::physx::cloth::ClothParams& p) {
    pxb_cloth_params o;
    pxb_cloth_params_default(&o);
    o.stretch_compliance = p.stretch_compliance;
    o.bend_compliance = p.bend_compliance;
    o.damping = p.damping;
    o.thickness = p.thickness;
    o.friction = p.friction;
    o.gravity_scale = p.gravity_scale;
    o.max_velocity = p.max_velocity;
    put3(o.external_acceleration, p.external_acceleration);
    put3(o.wind, p.wind);
    o.wind_turbulence = p.wind_turbulence;
    o.air_drag = p.air_drag;
    o.air_lift = p.air_lift;
    o.self_collision = p.self_collision ? 1 : 0;
    o.self_distance = p.self_distance;
    o.tether_scale = p.tether_scale;
    o.substeps = p.substeps;
    o.iterations = p.iterations;
    o.sleep_threshold = p.sleep_threshold;
    o.sleep_time = p.sleep_time;
    o.layer = p.layer;
    return o;
}

inline pxb_strand_params to_params(const coopa::physx::hair::StrandParams& p) {
    pxb_strand_params o;
    pxb_strand_params_default(&o);
    o.stretch_compliance = p.stretch_compliance;
    o.global_shape = p.global_shape;
    o.global_shape_falloff = p.global_shape_falloff;
    o.local_shape = p.local_shape;
    o.damping = p.damping;
    o.thickness = p.thickness;
    o.friction = p.friction;
    o.gravity_scale = p.gravity_scale;
    o.max_velocity = p.max_velocity;
    put3(o.external_acceleration, p.external_acceleration);
    put3(o.wind, p.wind);
    o.wind_turbulence = p.wind_turbulence;
    o.air_drag = p.air_drag;
    o.substeps = p.substeps;
    o.iterations = p.iterations;
    o.sleep_threshold = p.sleep_threshold;
    o.sleep_time = p.sleep_time;
    o.layer = p.layer;
    return o;
}

// cloth::solve_cloth on the device (cloth_solver.h:158-467 contract).
template <typename Scratch, typename Dispatch = int>
void solve_cloth(Device& dev, coopa::physx::cloth::Cloth& c,
                 const std::vector<coopa::physx::cloth::ClothCollider>& colliders,
                 const glm::vec3& gravity, uint32_t substeps, uint32_t iterations, float h,
                 Scratch& /*scratch*/, Dispatch&& /*dispatch*/ = Dispatch{}) {
    pxb_cloth_desc d;
    std::memset(&d, 0, sizeof(d));
    d.particles = reinterpret_cast<const pxb_particle*>(c.particles.data());
    d.n_particles = static_cast<uint32_t>(c.particles.size());
    d.stretch = reinterpret_cast<const pxb_constraint*>(c.stretch.data());
    d.n_stretch = static_cast<uint32_t>(c.stretch.size());
    d.stretch_batches = reinterpret_cast<const pxb_batch*>(c.stretch_batches.data());
    d.n_stretch_batches = static_cast<uint32_t>(c.stretch_batches.size());
    d.bend = reinterpret_cast<const pxb_constraint*>(c.bend.data());
    d.n_bend = static_cast<uint32_t>(c.bend.size());
    d.bend_batches = reinterpret_cast<const pxb_batch*>(c.bend_batches.data());
    d.n_bend_batches = static_cast<uint32_t>(c.bend_batches.size());
    d.tethers = reinterpret_cast<const pxb_tether*>(c.tethers.data());
    d.n_tethers = static_cast<uint32_t>(c.tethers.size());
    d.anchors = reinterpret_cast<const pxb_anchor*>(c.anchors.data());
    d.n_anchors = static_cast<uint32_t>(c.anchors.size());
    d.triangles = c.triangles.data();
    d.n_triangle_indices = static_cast<uint32_t>(c.triangles.size());
    d.columns = c.columns;
    d.rows = c.rows;
    d.params = to_params(c.params);
    d.time = c.time;
    std::vector<pxb_collider> cols;
    cols.reserve(colliders.size());
    for (const auto& k : colliders) cols.push_back(to_collider(dev, k));
    const float g[3] = {gravity.x, gravity.y, gravity.z};
    float bounds[6];
    dev.check(pxb_solve_cloth_host(dev.get(), &d, reinterpret_cast<pxb_particle*>(c.particles.data()),
                                   reinterpret_cast<pxb_constraint*>(c.stretch.data()),
                                   reinterpret_cast<pxb_constraint*>(c.bend.data()),
                                   reinterpret_cast<pxb_anchor*>(c.anchors.data()),
                                   cols.data(), static_cast<uint32_t>(cols.size()), g, substeps,
                                   iterations, h, &c.time, bounds),
              "solve_cloth");
    c.bounds.min = glm::vec3(bounds[0], bounds[1], bounds[2]);
    c.bounds.max = glm::vec3(bounds[3], bounds[4], bounds[5]);
}

// hair::solve_strands on the device (strand_solver.h:121-327 contract).
template <typename Scratch>
void solve_strands(Device& dev, coopa::physx::hair::StrandSet& set,
                   const std::vector<coopa::physx::cloth::ClothCollider>& colliders,
                   const glm::vec3& gravity, uint32_t substeps, uint32_t iterations, float h,
                   Scratch& /*scratch*/) {
    pxb_strand_set_desc d;
    std::memset(&d, 0, sizeof(d));
    d.particles = reinterpret_cast<const pxb_particle*>(set.particles.data());
    d.n_particles = static_cast<uint32_t>(set.particles.size());
    d.stretch = reinterpret_cast<const pxb_constraint*>(set.stretch.data());
    d.n_stretch = static_cast<uint32_t>(set.stretch.size());
    d.stretch_batches = reinterpret_cast<const pxb_batch*>(set.stretch_batches.data());
    d.n_stretch_batches = static_cast<uint32_t>(set.stretch_batches.size());
    d.rest_local = reinterpret_cast<const float*>(set.rest_local.data());
    d.rest_offset = reinterpret_cast<const float*>(set.rest_offset.data());
    d.strands = reinterpret_cast<const pxb_strand*>(set.strands.data());
    d.n_strands = static_cast<uint32_t>(set.strands.size());
    d.params = to_params(set.params);
    d.time = set.time;
    std::vector<pxb_collider> cols;
    for (const auto& k : colliders) cols.push_back(to_collider(dev, k));
    const float g[3] = {gravity.x, gravity.y, gravity.z};
    float bounds[6];
    dev.check(pxb_solve_strands_host(dev.get(), &d, reinterpret_cast<pxb_particle*>(set.particles.data()),
                                     reinterpret_cast<pxb_constraint*>(set.stretch.data()), cols.data(),
                                     static_cast<uint32_t>(cols.size()), g, substeps, iterations, h,
                                     &set.time, bounds),
              "solve_strands");
    set.bounds.min = glm::vec3(bounds[0], bounds[1], bounds[2]);
    set.bounds.max = glm::vec3(bounds[3], bounds[4], bounds[5]);
}

// ------------------------------------------------------------------------------------------
// The reference's exact signatures, on the calling thread's context
// ------------------------------------------------------------------------------------------

namespace detail {
inline int& thread_device_index() {
    thread_local int device = 0;
    return device;
}
inline std::unique_ptr<Device>& thread_device_slot() {
    thread_local std::unique_ptr<Device> dev;
    return dev;
}
}  // namespace detail

// The CUDA device the calling thread's reference-signature calls run on (default 0). Takes
// effect at the thread's next call; the thread's previous context (and the cloths it held) is
// released then.
inline void set_thread_device(int device) { detail::thread_device_index() = device; }

// The calling thread's context, created on its first use (one per host thread, as the C-ABI
// requires).
inline Device& thread_device() {
    auto& slot = detail::thread_device_slot();
    const int want = detail::thread_device_index();
    if (!slot || slot->index() != want) slot.reset(new Device(want));
    return *slot;
}

// cloth::solve_cloth(Cloth&, colliders, gravity, substeps, iterations, h, scratch, dispatch)
// (cloth_solver.h:158-161): the dispatcher is accepted and unused.
template <typename Dispatch>
void solve_cloth(coopa::physx::cloth::Cloth& c, const std::vector<coopa::physx::cloth::ClothCollider>& colliders,
                 const glm::vec3& gravity, uint32_t substeps, uint32_t iterations, float h,
                 coopa::physx::cloth::ClothSolverScratch& scratch, Dispatch&& dispatch) {
    solve_cloth(thread_device(), c, colliders, gravity, substeps, iterations, h, scratch,
                std::forward<Dispatch>(dispatch));
}

// The serial overload (cloth_solver.h:463-467).
inline void solve_cloth(coopa::physx::cloth::Cloth& c, const std::vector<coopa::physx::cloth::ClothCollider>& colliders,
                        const glm::vec3& gravity, uint32_t substeps, uint32_t iterations, float h,
                        coopa::physx::cloth::ClothSolverScratch& scratch) {
    solve_cloth(thread_device(), c, colliders, gravity, substeps, iterations, h, scratch);
}

// hair::solve_strands(StrandSet&, colliders, gravity, substeps, iterations, h, scratch)
// (strand_solver.h:121-123).
inline void solve_strands(coopa::physx::hair::StrandSet& set,
                          const std::vector<coopa::physx::cloth::ClothCollider>& colliders,
                          const glm::vec3& gravity, uint32_t substeps, uint32_t iterations, float h,
                          coopa::physx::hair::StrandSolverScratch& scratch) {
    solve_strands(thread_device(), set, colliders, gravity, substeps, iterations, h, scratch);
}

}  // namespace b200
}  // namespace pxb

#endif  // PHYSXCOOPA_B200_HPP
