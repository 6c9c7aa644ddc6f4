/*
 * physxcoopa_b200.h -- C-ABI of the B200 (sm_100a) XPBD cloth and hair-strand solver.
 *
 * This library replaces the CPU soft-body substep of physxcoopa (a header-only C++20 physics
 * library) behind its own boundary: `cloth::solve_cloth` (physxcoopa/cloth/cloth_solver.h:158-467)
 * and `hair::solve_strands` (physxcoopa/hair/strand_solver.h:121-327), batched at the granularity
 * of their per-frame callers `PhysicsWorld::step_cloths_` / `step_strands_`
 * (physxcoopa/world.h:1749-1847, 1861-1957).
 *
 * Conventions
 *  - Every entry point returns a pxb_status and never throws or aborts. On failure the context
 *    keeps a message retrievable with pxb_last_error().
 *  - One host thread per context. A context owns one CUDA stream on one device; all device work
 *    is ordered on it.
 *  - No CPU fallback: an input the device path does not implement (self-collision on a cloth
 *    larger than one CTA holds, cloths not built by make_grid_cloth) is refused with
 *    PXB_ERR_UNSUPPORTED instead of being solved on the host.
 *  - The plain-old-data structs below reproduce the reference's in-memory layouts byte for byte
 *    (glm::vec3 = 3 floats, glm::quat = x,y,z,w floats, no SIMD alignment), so a C++ caller can
 *    hand `std::vector<ClothParticle>::data()` and friends straight to this API.
 */
#ifndef PHYSXCOOPA_B200_H
#define PHYSXCOOPA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status                                                                                      */
/* ------------------------------------------------------------------------------------------ */

typedef enum pxb_status {
    PXB_OK = 0,
    PXB_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad index, inconsistent sizes */
    PXB_ERR_UNSUPPORTED = 2,      /* valid reference input the device path does not implement */
    PXB_ERR_CUDA = 3,             /* a CUDA runtime call failed (message has the CUDA error) */
    PXB_ERR_OUT_OF_MEMORY = 4,
    PXB_ERR_INVALID_HANDLE = 5,   /* stale or unknown cloth / strand-set id */
    PXB_ERR_DEVICE_STATUS = 6,    /* a kernel reported an error word (bounded wait expired, bad index) */
    PXB_ERR_TOO_LARGE = 7         /* input exceeds a documented capacity limit */
} pxb_status;

/* ------------------------------------------------------------------------------------------ */
/* Reference-layout data types                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* cloth::ClothParticle (physxcoopa/cloth/cloth.h:83-88). 40 bytes. inv_mass == 0 means pinned. */
typedef struct pxb_particle {
    float position[3];
    float prev_position[3];
    float velocity[3];
    float inv_mass;
} pxb_particle;

/* cloth::ClothConstraint (physxcoopa/cloth/cloth.h:103-108). 16 bytes. */
typedef struct pxb_constraint {
    uint32_t a;
    uint32_t b;
    float rest_length;
    float lambda;
} pxb_constraint;

/* cloth::ConstraintBatch (physxcoopa/cloth/cloth.h:270-273): particle-disjoint [begin, end). */
typedef struct pxb_batch {
    uint32_t begin;
    uint32_t end;
} pxb_batch;

/* cloth::ClothTether (physxcoopa/cloth/cloth.h:122-126). 12 bytes. */
typedef struct pxb_tether {
    uint32_t particle;
    uint32_t anchor;
    float max_length;
} pxb_tether;

/* cloth::ClothAnchor (physxcoopa/cloth/cloth.h:140-160), BodyId flattened. 48 bytes.
 * world_position is this frame's target (resolved by the caller from the body pose, as
 * PhysicsWorld::step_cloths_ does at world.h:1766-1773); prev_world_position is last frame's. */
typedef struct pxb_anchor {
    uint32_t particle;
    uint32_t body_index;
    uint32_t body_generation;
    float local_position[3];
    float world_position[3];
    float prev_world_position[3];
} pxb_anchor;

/* cloth::ClothParams (physxcoopa/cloth/cloth.h:167-256), field for field, plus one extension:
 * `has_shear_compliance` / `shear_compliance` are NOT in the reference; the reference solves
 * structural and shear edges with one `stretch_compliance`. Leave has_shear_compliance = 0 for
 * reference behaviour. pxb_cloth_params_default() returns the reference defaults. */
typedef struct pxb_cloth_params {
    float stretch_compliance;
    float bend_compliance;
    float damping;
    float thickness;
    float friction;
    float gravity_scale;
    float max_velocity;
    float external_acceleration[3];
    float wind[3];
    float wind_turbulence;
    float air_drag;
    float air_lift;
    int32_t self_collision;
    float self_distance;
    float tether_scale;
    uint32_t substeps;
    uint32_t iterations;
    float sleep_threshold;
    float sleep_time;
    uint32_t layer;
    int32_t has_shear_compliance;
    float shear_compliance;
} pxb_cloth_params;

/* collision::ShapeType (physxcoopa/collision/shape.h:33-39). */
typedef enum pxb_shape_type {
    PXB_SHAPE_SPHERE = 0,
    PXB_SHAPE_BOX = 1,
    PXB_SHAPE_CAPSULE = 2,
    PXB_SHAPE_TRIANGLE_MESH = 3, /* geometry from pxb_geometry_create_mesh */
    PXB_SHAPE_CONVEX_HULL = 4    /* geometry from pxb_geometry_create_hull */
} pxb_shape_type;

/* cloth::ClothCollider (physxcoopa/cloth/cloth_collision.h:53-78) with the fields of the
 * collision::Shape it points at (physxcoopa/collision/shape.h:54-102) copied in: the snapshot a
 * collider is for one step. Quaternions are (x, y, z, w). 152 bytes.
 * A TriangleMesh or ConvexHull collider names its geometry by the id pxb_geometry_create_mesh /
 * pxb_geometry_create_hull returned (Shape::mesh / Shape::hull, shape.h:85-98; 0 = none, which
 * like a null pointer there never collides) and carries Shape::mesh_scale / Shape::hull_scale in
 * geometry_scale. */
typedef struct pxb_collider {
    int32_t type;               /* pxb_shape_type */
    int32_t enabled;            /* Shape::enabled; a disabled shape never collides */
    float position[3];          /* owning body's world position */
    float orientation[4];       /* owning body's world orientation */
    float local_center[3];      /* Shape::local_center */
    float local_rotation[4];    /* Shape::local_rotation */
    float radius;               /* Sphere */
    float half_extents[3];      /* Box */
    float capsule_radius;       /* Capsule */
    float capsule_half_height;  /* Capsule, cylindrical half-length */
    int32_t capsule_axis;       /* Capsule long axis: 0=X, 1=Y, 2=Z */
    float sweep[3];             /* ClothCollider::sweep (PhysicsWorld leaves it zero) */
    float end_orientation[4];   /* ClothCollider::end_orientation */
    float bounds_min[3];        /* ClothCollider::bounds (world AABB over both poses) */
    float bounds_max[3];
    uint32_t geometry;          /* TriangleMesh / ConvexHull: registered geometry id, 0 = none */
    float geometry_scale;       /* Shape::mesh_scale or Shape::hull_scale */
} pxb_collider;

/* PhysicsWorld::GravitySource (physxcoopa/world.h:1154-1159). */
typedef struct pxb_gravity_source {
    float centre[3];
    float strength;
    float radius;
    float range; /* 0 = unlimited */
} pxb_gravity_source;

/* A cloth as the reference stores it (physxcoopa/cloth/cloth.h:284-315): plain pointers into
 * caller memory, reference layouts. The optional per-batch compliance arrays (NULL = every batch
 * uses params.stretch_compliance / params.bend_compliance, the reference behaviour) let a caller
 * give shear edges their own compliance; make_grid_cloth fills them when has_shear_compliance. */
typedef struct pxb_cloth_desc {
    const pxb_particle* particles;
    uint32_t n_particles;
    const pxb_constraint* stretch;
    uint32_t n_stretch;
    const pxb_batch* stretch_batches;
    uint32_t n_stretch_batches;
    const pxb_constraint* bend;
    uint32_t n_bend;
    const pxb_batch* bend_batches;
    uint32_t n_bend_batches;
    const pxb_tether* tethers;
    uint32_t n_tethers;
    const pxb_anchor* anchors;
    uint32_t n_anchors;
    const uint32_t* triangles; /* 3 indices per triangle */
    uint32_t n_triangle_indices;
    uint32_t columns; /* grid dimensions when built by make_grid_cloth, else 0 */
    uint32_t rows;
    pxb_cloth_params params;
    float time;       /* Cloth::time, drives the deterministic wind gust */
    const float* stretch_batch_compliance; /* optional, n_stretch_batches entries */
    const float* bend_batch_compliance;    /* optional, n_bend_batches entries */
} pxb_cloth_desc;


/* hair::Strand (physxcoopa/hair/strand.h:79-87). 64 bytes. `first` is the root particle. */
typedef struct pxb_strand {
    uint32_t first;
    uint32_t count;
    float root_position[3];
    float root_orientation[4];      /* (x, y, z, w) */
    float prev_root_position[3];
    float prev_root_orientation[4]; /* (x, y, z, w) */
} pxb_strand;

/* hair::StrandParams (physxcoopa/hair/strand.h:93-148), field for field. */
typedef struct pxb_strand_params {
    float stretch_compliance;
    float global_shape;
    float global_shape_falloff;
    float local_shape;
    float damping;
    float thickness;
    float friction;
    float gravity_scale;
    float max_velocity;
    float external_acceleration[3];
    float wind[3];
    float wind_turbulence;
    float air_drag;
    uint32_t substeps;
    uint32_t iterations;
    float sleep_threshold;
    float sleep_time;
    uint32_t layer;
} pxb_strand_params;

/* hair::StrandSet (physxcoopa/hair/strand.h:157-191) as plain pointers, reference layouts.
 * rest_local / rest_offset are 3 floats per particle, parallel to `particles`. */
typedef struct pxb_strand_set_desc {
    const pxb_particle* particles;
    uint32_t n_particles;
    const pxb_constraint* stretch;
    uint32_t n_stretch;
    const pxb_batch* stretch_batches;
    uint32_t n_stretch_batches;
    const float* rest_local;
    const float* rest_offset;
    const pxb_strand* strands;
    uint32_t n_strands;
    pxb_strand_params params;
    float time;
} pxb_strand_set_desc;

/* ------------------------------------------------------------------------------------------ */
/* Context                                                                                      */
/* ------------------------------------------------------------------------------------------ */

typedef struct pxb_context pxb_context;

/* Creates a context on CUDA device `device` with its own non-blocking stream. */
pxb_status pxb_context_create(int device, pxb_context** out);
pxb_status pxb_context_destroy(pxb_context* ctx);
/* Message of the last failure on this context ("" if none). Valid until the next call. */
const char* pxb_last_error(const pxb_context* ctx);
/* The context's cudaStream_t, for callers that want to time or order work around it. */
pxb_status pxb_context_stream(pxb_context* ctx, void** stream_out);
pxb_status pxb_context_synchronize(pxb_context* ctx);
/* Number of solver kernel launches issued on this context so far. */
uint64_t pxb_context_launch_count(const pxb_context* ctx);

/* Fills `out` with the reference's ClothParams defaults (physxcoopa/cloth/cloth.h:167-256). */
void pxb_cloth_params_default(pxb_cloth_params* out);

/* ------------------------------------------------------------------------------------------ */
/* Cloth registry: mirrors PhysicsWorld::add_cloth / remove_cloth / get_cloth                   */
/* (physxcoopa/world.h:552-596).                                                                */
/* ------------------------------------------------------------------------------------------ */

/* Uploads a cloth. Refuses an empty cloth (n_particles == 0) like add_cloth does, and a cloth
 * the device path does not implement (self_collision on) with PXB_ERR_UNSUPPORTED. A cloth of
 * general topology (constraint lists not make_grid_cloth's) may have up to 2^24 layout slots
 * (4 * ceil(n_particles / 4)); beyond, PXB_ERR_TOO_LARGE. The returned id is generational: it
 * goes stale after pxb_cloth_remove. */
pxb_status pxb_cloth_add(pxb_context* ctx, const pxb_cloth_desc* desc, uint64_t* id_out);
pxb_status pxb_cloth_remove(pxb_context* ctx, uint64_t id);

/* How pxb_cloth_add would lay a cloth out on the device. A cloth whose state does not fit one
 * CTA's shared memory is split by rows over a thread-block cluster of n_ranks CTAs (1, 2, 4 or
 * 8); beyond that (e.g. 512 x 512) every SM works on it with its state in global memory
 * (n_ranks 0). No counterpart in the reference, which has no device layout. */
typedef struct pxb_cloth_plan {
    int32_t n_ranks;          /* CTAs holding the cloth (a cluster when > 1; 0: the whole GPU) */
    int32_t rows_per_rank;    /* grid rows per CTA (the last CTA may hold fewer) */
    int32_t threads;          /* threads per CTA the cloth asks for */
    int32_t smem_bytes;       /* largest per-CTA dynamic shared memory */
    int32_t n_colours;        /* independent constraint sets solved one after another */
    int32_t n_segments;       /* affine segments over all CTAs and colours */
    int32_t layout_slots;     /* rows * 4 * ceil(columns / 4) particle slots */
    int32_t constraint_slots; /* rest-length slots over all CTAs, row padding included */
    int32_t self_collision;   /* 1: self-collision (ClothParams::self_collision) can run on this
                                 layout (one CTA, hash tables in shared memory); 0: a step with
                                 it enabled is refused with PXB_ERR_UNSUPPORTED */
    int32_t self_smem_bytes;  /* dynamic shared memory per CTA with self-collision on */
    int32_t topology;         /* 0: make_grid_cloth's lists, solved as colour segments; 1: any
                                 other lists (an imported mesh), one CTA, solved as runs of
                                 particle-disjoint items in the reference's order (n_colours then
                                 counts the runs) */
    int32_t lean;             /* 1: only the positions in shared memory, rest lengths and lambdas
                                 read in place in HBM (one CTA or two where a full-shared-memory
                                 layout would need a larger cluster); 2: the same on one CTA
                                 with the positions as float arrays and an index into the
                                 cloth's distinct inverse masses (pxb_context_set_lean_arrays) */
    int32_t phases;           /* barrier-separated phases per iteration: colours in a row that
                                 touch disjoint particles share one (one CTA only; else n_colours) */
} pxb_cloth_plan;

/* Plans a cloth without a context or a GPU: validates it exactly as pxb_cloth_add does and
 * fills *out. On failure the message goes to err (NUL-terminated, at most err_cap bytes). */
pxb_status pxb_cloth_plan_layout(const pxb_cloth_desc* desc, pxb_cloth_plan* out, char* err,
                                 uint32_t err_cap);
/* Replaces a live cloth's tunables (ClothComponent::cloth_mut()->params is edited live). */
pxb_status pxb_cloth_set_params(pxb_context* ctx, uint64_t id, const pxb_cloth_params* params);
/* Host edit of particle state between steps (all four fields of every particle). */
pxb_status pxb_cloth_write_particles(pxb_context* ctx, uint64_t id, const pxb_particle* particles,
                                     uint32_t n);
/* Reads particle state back (positions, prev positions, velocities, inv_mass). */
pxb_status pxb_cloth_read_particles(pxb_context* ctx, uint64_t id, pxb_particle* out, uint32_t n);
/* Reads the constraint lambdas left by the last substep, in the reference's list order. */
pxb_status pxb_cloth_read_lambdas(pxb_context* ctx, uint64_t id, float* stretch_out,
                                  uint32_t n_stretch, float* bend_out, uint32_t n_bend);
/* Sets this frame's anchor targets (3 floats per anchor, anchor-list order). The previous
 * targets become prev_world_position, as the reference's per-step epilogue leaves them
 * (cloth_solver.h:457). */
pxb_status pxb_cloth_set_anchor_targets(pxb_context* ctx, uint64_t id, const float* world_xyz,
                                        uint32_t n_anchors);
/* Reads the anchors' current (prev, world) targets back, reference layout. */
pxb_status pxb_cloth_read_anchors(pxb_context* ctx, uint64_t id, pxb_anchor* out, uint32_t n);
/* Cloth::time after the last step. */
pxb_status pxb_cloth_read_time(pxb_context* ctx, uint64_t id, float* time_out);

/* ------------------------------------------------------------------------------------------ */
/* Batched step: one solve_cloth per listed cloth, all in one device launch sequence.           */
/* ------------------------------------------------------------------------------------------ */

typedef struct pxb_cloth_step_desc {
    const uint64_t* cloths;       /* ids to advance */
    uint32_t n_cloths;
    const pxb_collider* colliders;          /* flat collider list */
    const uint32_t* collider_offsets;       /* n_cloths + 1 offsets; NULL = no colliders */
    float gravity[3];                       /* world gravity (PhysicsWorld::gravity_) */
    const pxb_gravity_source* sources;      /* flat gravity-source list, may be NULL */
    const uint32_t* source_offsets;         /* n_cloths + 1 offsets; NULL = no sources */
    uint32_t substeps;    /* solve_cloth's `substeps` (a cloth's params.substeps wins) */
    uint32_t iterations;  /* solve_cloth's `iterations` (a cloth's params.iterations wins) */
    float h;              /* step length, seconds */
} pxb_cloth_step_desc;

/* Per-cloth results of a step: the world AABB (Cloth::bounds) and max particle speed that the
 * caller's broadphase query and sleep gate read (world.h:1777-1779, 1837). */
typedef struct pxb_cloth_frame_result {
    float bounds_min[3];
    float bounds_max[3];
    float max_speed;
    float time;
} pxb_cloth_frame_result;

/* Advances every listed cloth by one call of solve_cloth, with gravity evaluated per cloth at
 * its mean particle position when it has gravity sources (PhysicsWorld::gravity_at(cloth_centre_),
 * world.h:1833, 2048-2076). Enqueued on the context stream; returns before completion. */
pxb_status pxb_cloths_step(pxb_context* ctx, const pxb_cloth_step_desc* step);
/* The same step replayed from a CUDA graph. The host prepares the step's inputs as
 * pxb_cloths_step does; the upload and every launch of the step (side-stream groups included)
 * are captured once and replayed while the step's shape stays the same (same cloths in the same
 * order, same collider and gravity-source counts, same kernel variant, no cloth added, removed
 * or re-parameterised, no internal buffer regrown). A new shape runs eagerly on its first call
 * and is captured on its second. Results are identical to pxb_cloths_step's. Must not be called
 * while the context stream is being captured by the caller. No counterpart in the reference. */
pxb_status pxb_cloths_step_graph(pxb_context* ctx, const pxb_cloth_step_desc* step);
/* Copies the last step's per-cloth results to host memory (synchronizes the stream). */
pxb_status pxb_cloths_read_results(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                   pxb_cloth_frame_result* out);
/* ------------------------------------------------------------------------------------------ */
/* A whole cloth frame: PhysicsWorld::step_cloths_ (physxcoopa/world.h:1749-1847)                */
/* ------------------------------------------------------------------------------------------ */

/* A rigid body's pose as the caller's world holds it (dynamics::Body::position / orientation,
 * quaternion x, y, z, w), indexed by pxb_anchor::body_index. An anchor resolves against it only
 * when `alive` is set and `generation` equals the anchor's body_generation (what
 * PhysicsWorld::get_body checks); otherwise it keeps its last target. 36 bytes. */
typedef struct pxb_body_pose {
    float position[3];
    float orientation[4];
    uint32_t generation;
    uint32_t alive;
} pxb_body_pose;

typedef struct pxb_cloth_frame_desc {
    const uint64_t* cloths;                 /* live, enabled cloths to advance this frame */
    uint32_t n_cloths;
    const pxb_body_pose* bodies;            /* may be NULL when no cloth has anchors */
    uint32_t n_bodies;
    const pxb_collider* colliders;          /* each cloth's gathered colliders, flat */
    const uint32_t* collider_offsets;       /* n_cloths + 1 offsets; NULL = no colliders */
    const uint8_t* collider_moving;         /* per cloth: a non-static collider of its list moves
                                               (world.h:1808-1812); NULL = none does */
    float gravity[3];
    const pxb_gravity_source* sources;
    const uint32_t* source_offsets;
    float fixed_dt;                         /* PhysicsConfig::fixed_dt */
    uint32_t cloth_substeps;                /* PhysicsConfig::cloth_substeps */
    uint32_t cloth_iterations;              /* PhysicsConfig::cloth_iterations */
    float dt;                               /* this frame's dt */
} pxb_cloth_frame_desc;

/* One cloth frame as PhysicsWorld::step_cloths_ runs it, for every listed cloth: the frame's
 * substep count (world.h:1753-1756); each anchor's target from its body's pose,
 * position + orientation * local_position (world.h:1765-1772); the sleep gate (a moved anchor or
 * a moving collider wakes the cloth; a sleeping cloth only carries its anchors' targets into their
 * previous targets, world.h:1815-1825); one batched solve of the awake cloths; then the sleep
 * bookkeeping on each solved cloth's max particle speed (below params.sleep_threshold for
 * params.sleep_time seconds: asleep, velocities zeroed, world.h:1831-1845). The collider gather
 * (broadphase) stays the caller's. Synchronous: it reads the solved cloths' results back.
 * dt must be positive (PhysicsWorld steps with its fixed dt).
 * awake_out (n_cloths entries, may be NULL) receives each cloth's awake flag after the frame. */
pxb_status pxb_cloths_step_frame(pxb_context* ctx, const pxb_cloth_frame_desc* frame, uint8_t* awake_out);

/* The cloth part of PhysicsWorld::world_state_hash (world.h:1334-1359): FNV-1a 64, continued
 * from `seed` (1469598103934665603, the FNV offset basis, when no bodies were mixed before), over
 * each listed cloth's particles in index order, position then velocity, the floats' bytes as they
 * lie in memory. The device gathers those bytes for every cloth in one launch; the chain itself,
 * serial by definition, runs on the host. Synchronous. */
pxb_status pxb_cloths_state_hash(pxb_context* ctx, const uint64_t* cloths, uint32_t n, uint64_t seed,
                                 uint64_t* hash_out);

/* A renderer's vertex buffer over Cloth::triangles (physxcoopa/cloth/cloth.h:293-299, the index
 * buffer a renderer draws): 6 floats per particle, cloths in list order, particles in index order
 * -- position, then the unit vertex normal, the sum of cross(b - a, c - a) over the particle's
 * triangles (make_grid_cloth's two per grid cell, cloth_builder.h:200-207) normalized, or zero
 * where that sum is zero. The reference tree has no normal pass (its renderer is outside it), so
 * this formula is the library's own. Refused for a cloth with no triangle list. `capacity` is in
 * floats. Synchronous. */
pxb_status pxb_cloths_read_render_buffer(pxb_context* ctx, const uint64_t* cloths, uint32_t n, float* out,
                                         size_t capacity);

/* Cloth::awake and Cloth::sleep_timer of the listed cloths (a new cloth is awake, timer 0). */
pxb_status pxb_cloths_read_sleep_state(pxb_context* ctx, const uint64_t* cloths, uint32_t n, uint8_t* awake_out,
                                       float* sleep_timer_out);

/* Copies positions of the listed cloths (3 floats per particle, cloths in list order) into
 * host memory `out` of `capacity` floats (synchronizes the stream). This is what a renderer or
 * a determinism hash reads back each frame. */
pxb_status pxb_cloths_read_positions(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                     float* out, size_t capacity);
/* Pipelined form for a renderer that draws frame k while frame k + 1 is simulated: snapshots
 * the same positions on the device (after every step enqueued so far) and copies them into
 * host `out` on a copy stream, returning at once, so the copy overlaps the next step. `out`
 * must stay valid until pxb_cloths_wait_positions returns, and should be pinned host memory
 * (cudaHostAlloc) for the copy to run asynchronously. Two snapshots may be in flight; a third
 * call first waits for the older one. */
pxb_status pxb_cloths_read_positions_async(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                           float* out, size_t capacity);
/* The same for the last step's per-cloth results (what pxb_cloths_read_results returns), copied
 * into host `out` (n records, pinned for an asynchronous copy) without waiting for the step, so
 * the caller can enqueue the next step at once; every listed cloth must have been in the last
 * (plain) step. Two copies may be in flight. */
pxb_status pxb_cloths_read_results_async(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                         pxb_cloth_frame_result* out);
/* Blocks until every copy started by pxb_cloths_read_positions_async or
 * pxb_cloths_read_results_async has landed, then checks the device error word. */
pxb_status pxb_cloths_wait_positions(pxb_context* ctx);
/* The same gather into DEVICE memory `out_device` (capacity floats), allocating nothing. No
 * counterpart in the reference. For callers that may not allocate device memory while they run
 * (a per-frame reader inside a fixed memory budget, or code where cudaMalloc / cudaFree would
 * synchronise the device or is not permitted): pxb_cloths_read_positions grows internal buffers
 * on demand, this never does. At most 4096 cloths per call (PXB_ERR_TOO_LARGE beyond); the
 * per-call cloth list lives in a 48 KB array compiled into the library, held on every GPU that
 * loads it until exit. A context's first call looks up that array's address (set-up) and
 * keeps it on the context: make it before any stream capture. The call list is assembled in a static host buffer under a
 * mutex (no allocation, no large stack frame), so concurrent host calls take turns. The registry must be current (a step since the last
 * add / remove / parameter change), else PXB_ERR_INVALID_ARGUMENT. Enqueued on the context
 * stream, returns before completion; calls that overlap on the GPU (other contexts or streams
 * of the same device) share the array and race -- serialise them. */
pxb_status pxb_cloths_gather_positions_device(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                              float* out_device, size_t capacity);

/* Drop-in single-cloth solve on HOST memory, the exact contract of cloth::solve_cloth: the cloth
 * described by `desc` is uploaded, advanced, and its particles / lambdas / anchors / time /
 * bounds written back to the caller's arrays. `particles`, `stretch`, `bend`, `anchors` are
 * updated in place through the non-const pointers; `time_inout` and `bounds_out` (6 floats) may
 * be NULL. Uses a per-context cache so repeated calls on the same arrays do not re-upload the
 * topology. */
pxb_status pxb_solve_cloth_host(pxb_context* ctx, const pxb_cloth_desc* desc,
                                pxb_particle* particles, pxb_constraint* stretch,
                                pxb_constraint* bend, pxb_anchor* anchors,
                                const pxb_collider* colliders, uint32_t n_colliders,
                                const float gravity[3], uint32_t substeps, uint32_t iterations,
                                float h, float* time_inout, float* bounds_out);

/* Kernel variant used by pxb_cloths_step: the block-size cap of the cloth kernel (0 = 512
 * threads, 1 = 768, 2 = 1024; a larger block has more warps to hide latency but fewer
 * registers per thread), for every layout class (clears the autotuner's per-class choices).
 * Results are identical across variants; only speed differs. */
pxb_status pxb_context_set_cloth_variant(pxb_context* ctx, int32_t variant);
/* Failure-path testing (no counterpart in the reference). Cloths beyond an 8-CTA cluster step on
 * every SM with a grid barrier between colours; each barrier wait is bounded (grid_wait_polls
 * polls of about 64 ns, default 2^22) and, when it runs out, records an error word, stops all
 * later barrier waits of the launch so it ends at once, and makes the next synchronising call
 * return PXB_ERR_DEVICE_STATUS (which clears the word). With `unreachable` set, no grid barrier
 * can complete, so that path runs on purpose; the cloth's state after such a step is
 * meaningless -- rewrite it (pxb_cloth_write_particles) or re-add the cloth. The context stays
 * usable: restore the defaults with (1 << 22, 0). */
pxb_status pxb_context_set_wait_test(pxb_context* ctx, uint32_t grid_wait_polls, uint32_t unreachable);
/* Launch form of pxb_cloths_step (no counterpart in the reference, whose step_cloths_ walks its
 * cloths one after another). Cloths are grouped by layout and launched largest first. Mode 1
 * (default): each group runs as a persistent kernel, as many CTAs (clusters) as the SMs hold,
 * each popping the group's next cloth from a device work queue (one atomic per cloth) until the
 * queue is empty. Mode 0: one CTA (cluster) per cloth, the hardware scheduler handing them out.
 * Results are identical; only speed differs. */
pxb_status pxb_context_set_launch_mode(pxb_context* ctx, int32_t mode);
/* Threads per CTA of one-CTA grid cloths (no counterpart in the reference). Mode 0: a cloth runs
 * with half the items of its largest colour in threads, up to the kernel variant's cap. Mode 1
 * (default): where shared memory lets an SM hold k CTAs of the cloth, it runs with at most 1/k of
 * the threads the variant's registers allow, so k CTAs share each SM (one projects while another
 * waits at a colour barrier). Results are identical; only speed differs. */
pxb_status pxb_context_set_thread_fit(pxb_context* ctx, int32_t mode);
/* Layout choice for cloths added from now on (no counterpart in the reference). With `enable`
 * (default), a sheet small enough to be held whole in one CTA's shared memory, but so large that
 * an SM then holds only one of its CTAs, takes the lean layout (positions alone in shared memory,
 * rest lengths and lambdas read in place in HBM) where that lets an SM hold two or more; with 0 it
 * is held whole. Results are identical; only speed differs. */
pxb_status pxb_context_set_lean_mid(pxb_context* ctx, int32_t enable);
/* Layout choice for cloths added from now on (no counterpart in the reference). With `enable`
 * (default), a grid cloth too large for one CTA's shared memory as float4 positions but small
 * enough as float arrays (12 bytes per particle plus a one-byte index into a table of its
 * distinct inverse masses; sheets up to 128 x 128) runs on one CTA in that form; with 0 it runs
 * on a cluster of two CTAs as before. Results are identical; only speed differs. */
pxb_status pxb_context_set_lean_arrays(pxb_context* ctx, int32_t enable);
/* Autotuner: times every kernel variant in both launch forms on `step` (the caller's real batch,
 * `trials` launches each after one warm-up) and keeps the fastest pair on the context. Then, one
 * layout class at a time (largest share of the batch first), it times the class's cloths at the
 * other two variants with the rest unchanged, alternating with the current choice, and keeps a
 * variant that is faster by more than 1 %. The listed
 * cloths' device state and host mirrors are saved first and restored after, so tuning does not
 * advance them. variant_out (may be NULL) receives variant + 3 * mode of the pair kept; ms_out
 * (may be NULL) six entries, milliseconds per step: variants 0-2 one CTA per cloth, then variants
 * 0-2 persistent. The threads a constraint colour runs with follow the block size (and the
 * thread fit, pxb_context_set_thread_fit); iterations are never fused between barriers (the
 * reference's Gauss-Seidel order needs one after every colour). */
pxb_status pxb_cloths_autotune(pxb_context* ctx, const pxb_cloth_step_desc* step, uint32_t trials,
                               int32_t* variant_out, float* ms_out);
/* Layout classes of the per-class block-size choice: class = 3 * kind + residency, kind 0 a sheet
 * held whole in shared memory, 1 the same with mesh / hull colliders, self-collision or general
 * topology, 2 general topology with its state in HBM, 3 / 4 lean float4 positions (plain /
 * extended), 5 / 6 lean float arrays (plain / extended); residency 0, 1, 2 for one, two, three
 * or more of the cloth's CTAs per SM by shared memory. */
#define PXB_TUNE_CLASSES 21
/* The kernel configuration in use: block-size variant (0-2: caps of 512 / 768 / 1024 threads),
 * launch mode, thread fit, and per layout class the variant it runs (PXB_TUNE_CLASSES entries;
 * may be NULL) with the layout slots the last plain step launched in it (may be NULL). */
pxb_status pxb_context_get_tuning(pxb_context* ctx, int32_t* variant, int32_t* launch_mode, int32_t* thread_fit,
                                  int32_t* class_variants, double* class_slots);

/* ------------------------------------------------------------------------------------------ */
/* Collision primitive: cloth::project_particle (physxcoopa/cloth/cloth_collision.h:386-420)    */
/* evaluated on the device for a batch of points (the collision stage of both solvers).         */
/* ------------------------------------------------------------------------------------------ */

/* For each of n points: projects it out of `collider` with standoff `thickness`. Writes the
 * corrected point, the normal and depth, and hit (1/0). motion_start_xyz (may be NULL) is each
 * point's position at the start of the substep, which enables the TriangleMesh swept crossing
 * test (cloth_collision.h:217-272). Host arrays; synchronous. */
pxb_status pxb_project_particles(pxb_context* ctx, const pxb_collider* collider, float thickness,
                                 const float* points_xyz, const float* motion_start_xyz,
                                 uint32_t n, float* points_out, float* normals_out,
                                 float* depths_out, int32_t* hit_out);

/* ------------------------------------------------------------------------------------------ */
/* Collider geometry: geometry::ConvexHull and geometry::TriangleMesh, registered once          */
/* ------------------------------------------------------------------------------------------ */

/* geometry::ConvexHull (physxcoopa/geometry/convex_hull.h:41-57), the arrays hull_vs_sphere
 * reads: vertices (xyz), face_planes (xyz = outward unit normal, w = offset), and face f's
 * vertex indices face_vertices[face_starts[f] .. face_starts[f + 1]), CCW about its normal. */
typedef struct pxb_hull_desc {
    const float* vertices;         /* 3 floats per vertex */
    uint32_t n_vertices;
    const float* face_planes;      /* 4 floats per face */
    uint32_t n_faces;
    const uint32_t* face_starts;   /* n_faces + 1 entries, starting at 0 */
    const uint32_t* face_vertices; /* face_starts[n_faces] entries */
} pxb_hull_desc;

/* geometry::TriangleMesh (physxcoopa/geometry/triangle_mesh.h:70-96) as its four-argument
 * constructor takes it: vertices, three indices per triangle and one face normal per triangle
 * (TriangleMesh::normals()). normals may be NULL: they are then computed the way
 * TriangleMesh::from_triangles does, normalize(cross(b - a, c - a)). Adjacency is not read by
 * cloth or strand collision. */
typedef struct pxb_mesh_desc {
    const float* vertices;   /* 3 floats per vertex */
    uint32_t n_vertices;
    const uint32_t* indices; /* 3 per triangle */
    uint32_t n_indices;
    const float* normals;    /* 3 floats per triangle, or NULL */
} pxb_mesh_desc;

/* Copies a hull to the device and returns its id (never 0) for pxb_collider::geometry. Each
 * step then poses it on the host (world vertices, face planes and edge normals, as
 * collision::world_posed_hull and hull_vs_sphere derive them) and every particle tests the
 * posed faces on the device. Refused: no faces, a face with no vertex or more than 160
 * (k_hull_clip_cap, sat_hull.h:157), an index out of range; PXB_ERR_TOO_LARGE beyond 4096 faces
 * or 65536 face-vertex entries. */
pxb_status pxb_geometry_create_hull(pxb_context* ctx, const pxb_hull_desc* desc, uint32_t* id_out);

/* Copies a triangle mesh to the device with its bounding-volume hierarchy, built on the host by
 * MeshBVH::build's rule (mesh_bvh.h: leaves of at most 4 triangles, median split on the widest
 * centroid axis), so the device visits candidate triangles in the reference's order and breaks
 * ties between equally near triangles the same way. An empty mesh (no triangles) is accepted and
 * never collides, like TriangleMesh::empty(). PXB_ERR_TOO_LARGE beyond 2^24 triangles. */
pxb_status pxb_geometry_create_mesh(pxb_context* ctx, const pxb_mesh_desc* desc, uint32_t* id_out);

/* Waits for the context's stream, then frees the geometry. A later step naming its id is refused
 * with PXB_ERR_INVALID_HANDLE. */
/* A height-grid mesh (TriangleMesh::from_height_grid over geometry::HeightGrid, height_grid.h,
 * triangle_mesh.h:210-215): nx x ny samples (at least 2 x 2; heights padded with zeros), sample
 * (i, j) at (i * cell_x, j * cell_y, heights[j * nx + i]), two triangles per cell. Mesh colliders
 * naming it are queried through the grid's block pyramid in the reference's order. Sides of at
 * most 32768 samples and at most 2^24 samples in all, else PXB_ERR_TOO_LARGE (the reference's
 * HeightGrid has no such limit). */
typedef struct pxb_height_grid_desc {
    uint32_t nx, ny;
    float cell_x, cell_y;
    const float* heights;
    uint32_t n_heights;
} pxb_height_grid_desc;
pxb_status pxb_geometry_create_height_grid(pxb_context* ctx, const pxb_height_grid_desc* desc, uint32_t* id_out);
pxb_status pxb_geometry_destroy(pxb_context* ctx, uint32_t id);

/* ------------------------------------------------------------------------------------------ */
/* Grid builders (host, setup time): cloth::make_grid_cloth / pin_static / build_tethers        */
/* (physxcoopa/cloth/cloth_builder.h:81-358). A built cloth lives in library host memory; view  */
/* it as a pxb_cloth_desc, edit it through the view's arrays, upload it with pxb_cloth_add.      */
/* ------------------------------------------------------------------------------------------ */

typedef struct pxb_host_cloth pxb_host_cloth;

/* cloth::GridClothDesc (physxcoopa/cloth/cloth_builder.h:52-64) plus a seeded jitter: when
 * jitter > 0 every particle is displaced by an independent uniform draw in [-jitter, jitter] per
 * axis (splitmix64 stream from jitter_seed) BEFORE rest lengths are captured, so the jittered
 * sheet starts unstrained. jitter = 0 reproduces make_grid_cloth exactly. */
typedef struct pxb_grid_cloth_desc {
    uint32_t columns;
    uint32_t rows;
    float width;
    float height;
    float center[3];
    float orientation[4]; /* (x, y, z, w) */
    float total_mass;
    int32_t shear;
    pxb_cloth_params params;
    float jitter;
    uint64_t jitter_seed;
} pxb_grid_cloth_desc;

pxb_status pxb_host_cloth_make_grid(const pxb_grid_cloth_desc* desc, pxb_host_cloth** out);

/* A cloth from an arbitrary triangle mesh (no reference builder; the reference's README names
 * "a builder and a batch colouring pass" as what an imported-mesh cloth needs). One particle per
 * vertex (mass total_mass / n_vertices, as make_grid_cloth spreads it); a stretch constraint per
 * distinct edge in first-appearance order (triangle by triangle, edges (0,1), (1,2), (2,0)); with
 * bend set, a bend constraint between the two opposite vertices of every edge exactly two
 * triangles share (skipped when it repeats a stretch edge or an earlier bend pair). Each list is
 * coloured greedily, first fit in list order, into particle-disjoint batches and stored batch by
 * batch. Triangles are the mesh's; columns and rows are 0. A self_distance left at 0 becomes
 * 0.6 x the mean edge length. */
typedef struct pxb_mesh_cloth_desc {
    const float* vertices;   /* xyz per vertex */
    uint32_t n_vertices;
    const uint32_t* indices; /* three per triangle */
    uint32_t n_indices;
    float total_mass;
    int32_t bend;
    pxb_cloth_params params;
} pxb_mesh_cloth_desc;
pxb_status pxb_host_cloth_make_mesh(const pxb_mesh_cloth_desc* desc, pxb_host_cloth** out);
pxb_status pxb_host_cloth_destroy(pxb_host_cloth* cloth);
/* cloth::pin_static (cloth_builder.h:271-292). Writes the number newly pinned to pinned_out. */
pxb_status pxb_host_cloth_pin_static(pxb_host_cloth* cloth, const float world_point[3],
                                     float radius, uint32_t* pinned_out);
/* cloth::pin_to_body (cloth_builder.h:235-258): pins every not-yet-pinned particle within
 * `radius` of world_point to the body (index, generation) at the given pose, recording each
 * anchor's position in the body's frame. Writes the number newly pinned to pinned_out. */
pxb_status pxb_host_cloth_pin_to_body(pxb_host_cloth* cloth, uint32_t body_index, uint32_t body_generation,
                                      const float body_position[3], const float body_orientation[4],
                                      const float world_point[3], float radius, uint32_t* pinned_out);
/* cloth::build_tethers (cloth_builder.h:308-358): geodesic Dijkstra over the stretch graph. */
pxb_status pxb_host_cloth_build_tethers(pxb_host_cloth* cloth);
/* cloth::build_tethers on the device: the same tethers, bit for bit. Dijkstra's float distances
 * are the unique fixpoint of dist[v] = min over neighbours u of dist[u] + |p_v - p_u| as long as
 * no edge vanishes in that sum (dist[u] + |p_v - p_u| == dist[u] for two distinct particles); the
 * device relaxes to that fixpoint in parallel and gives each particle the anchor of the neighbour
 * the reference's priority queue settles first among those reaching its distance (smallest
 * (dist, index)). When some edge does vanish the queue's order is no longer that, and the call
 * returns PXB_ERR_UNSUPPORTED with the tethers unchanged (use pxb_host_cloth_build_tethers).
 * Writes n_out tethers (at most n_particles) in particle order. */
pxb_status pxb_build_tethers_device(pxb_context* ctx, const pxb_particle* particles, uint32_t n_particles,
                                    const pxb_constraint* stretch, uint32_t n_stretch,
                                    const pxb_anchor* anchors, uint32_t n_anchors, float tether_scale,
                                    pxb_tether* out, uint32_t capacity, uint32_t* n_out);
/* The same on a host cloth's arrays, replacing its tethers. */
pxb_status pxb_host_cloth_build_tethers_device(pxb_context* ctx, pxb_host_cloth* cloth);
/* A view of the cloth's arrays; pointers stay valid until the next builder call on it. */
pxb_status pxb_host_cloth_view(pxb_host_cloth* cloth, pxb_cloth_desc* view_out);
/* Mutable pointers into the same arrays, for host edits before upload. */
pxb_status pxb_host_cloth_mutable(pxb_host_cloth* cloth, pxb_particle** particles,
                                  pxb_anchor** anchors, pxb_cloth_params** params);

/* ------------------------------------------------------------------------------------------ */
/* Hair strand sets: mirrors PhysicsWorld::add_strands / step_strands_ (world.h:632-650,       */
/* 1861-1957) and hair::solve_strands (physxcoopa/hair/strand_solver.h:121-327).                */
/* ------------------------------------------------------------------------------------------ */

/* Uploads a strand set built by make_strands (strand_builder.h:58-127): strands contiguous,
 * stretch constraints in the builder's even / odd batches. Refuses an empty set with
 * PXB_ERR_INVALID_ARGUMENT (add_strands does the same), another layout with
 * PXB_ERR_UNSUPPORTED, and a strand of more than 8192 particles with PXB_ERR_TOO_LARGE. Sets whose
 * strands all have at most 32 particles run one lane per particle; a set with a longer strand
 * runs the long-strand kernel (lanes stride over the particles, positions in shared memory). */
pxb_status pxb_strands_add(pxb_context* ctx, const pxb_strand_set_desc* desc, uint64_t* id_out);
pxb_status pxb_strands_remove(pxb_context* ctx, uint64_t id);
pxb_status pxb_strands_set_params(pxb_context* ctx, uint64_t id, const pxb_strand_params* params);
/* hair::set_strand_roots (strand_builder.h:139-149): every strand's previous root becomes its
 * current one, then the new targets are written (3 floats per strand; orientations, 4 floats
 * (x, y, z, w) per strand, may be NULL / shorter to keep the current ones). */
pxb_status pxb_strands_set_roots(pxb_context* ctx, uint64_t id, const float* positions,
                                 uint32_t n_positions, const float* orientations,
                                 uint32_t n_orientations);
pxb_status pxb_strands_write_particles(pxb_context* ctx, uint64_t id, const pxb_particle* particles,
                                       uint32_t n);
pxb_status pxb_strands_read_particles(pxb_context* ctx, uint64_t id, pxb_particle* out, uint32_t n);
/* Lambdas of the stretch constraints left by the last substep, reference list order. */
pxb_status pxb_strands_read_lambdas(pxb_context* ctx, uint64_t id, float* out, uint32_t n);
/* The strand records (root targets), reference layout. */
pxb_status pxb_strands_read_strands(pxb_context* ctx, uint64_t id, pxb_strand* out, uint32_t n);
pxb_status pxb_strands_read_time(pxb_context* ctx, uint64_t id, float* time_out);

typedef struct pxb_strand_step_desc {
    const uint64_t* sets;
    uint32_t n_sets;
    const pxb_collider* colliders;
    const uint32_t* collider_offsets;   /* n_sets + 1; NULL = no colliders */
    float gravity[3];
    const pxb_gravity_source* sources;
    const uint32_t* source_offsets;     /* n_sets + 1; NULL = no sources */
    uint32_t substeps;
    uint32_t iterations;
    float h;
} pxb_strand_step_desc;

/* Advances every listed set by one solve_strands, gravity evaluated at the centre of the set's
 * last bounds when it has sources (world.h:1941-1945). */
pxb_status pxb_strands_step(pxb_context* ctx, const pxb_strand_step_desc* step);
/* Per-set bounds, max particle speed and time after the last step (synchronizes). */
pxb_status pxb_strands_read_results(pxb_context* ctx, const uint64_t* sets, uint32_t n,
                                    pxb_cloth_frame_result* out);

typedef struct pxb_strand_frame_desc {
    const uint64_t* sets;                   /* live strand sets to advance this frame */
    uint32_t n_sets;
    const pxb_collider* colliders;          /* each set's gathered colliders, flat */
    const uint32_t* collider_offsets;       /* n_sets + 1 offsets; NULL = no colliders */
    const uint8_t* collider_moving;         /* per set: a non-static collider of its list moves
                                               (world.h:1905-1911); NULL = none does */
    float gravity[3];
    const pxb_gravity_source* sources;
    const uint32_t* source_offsets;
    float fixed_dt;                         /* PhysicsConfig::fixed_dt */
    uint32_t cloth_substeps;                /* PhysicsConfig::cloth_substeps */
    uint32_t cloth_iterations;              /* PhysicsConfig::cloth_iterations */
    float dt;                               /* this frame's dt */
} pxb_strand_frame_desc;

/* One strand frame as PhysicsWorld::step_strands_ runs it (world.h:1861-1957), for every listed
 * set: the frame's substep count; a root whose target moved since the last one (|root -
 * prev_root|^2 > 1e-6, set by pxb_strands_set_roots) or a moving collider wakes the set; a
 * sleeping set only carries its roots' targets into their previous targets; one batched solve
 * of the awake sets (gravity at each set's bounds centre when it has sources); then the sleep
 * bookkeeping on each solved set's max particle speed (below params.sleep_threshold for
 * params.sleep_time seconds: asleep, velocities zeroed). The collider gather (broadphase or the
 * set's allowlist) stays the caller's. Synchronous. dt must be positive. awake_out (n_sets
 * entries, may be NULL) receives each set's awake flag after the frame. */
pxb_status pxb_strands_step_frame(pxb_context* ctx, const pxb_strand_frame_desc* frame, uint8_t* awake_out);
/* StrandSet::awake and StrandSet::sleep_timer of the listed sets (a new set is awake, timer 0). */
pxb_status pxb_strands_read_sleep_state(pxb_context* ctx, const uint64_t* sets, uint32_t n, uint8_t* awake_out,
                                        float* sleep_timer_out);

/* Drop-in hair::solve_strands on HOST memory: the set described by `desc` is advanced and its
 * particles, stretch lambdas and time written back (bounds_out, 6 floats, may be NULL). */
pxb_status pxb_solve_strands_host(pxb_context* ctx, const pxb_strand_set_desc* desc,
                                  pxb_particle* particles, pxb_constraint* stretch,
                                  const pxb_collider* colliders, uint32_t n_colliders,
                                  const float gravity[3], uint32_t substeps, uint32_t iterations,
                                  float h, float* time_inout, float* bounds_out);

/* Builder: hair::make_strands (strand_builder.h:58-127) from n_strands polylines of counts[i]
 * points (3 floats each, packed), one root orientation (x, y, z, w) and particle mass per strand
 * (either may be NULL: identity / 0.001 kg). */
typedef struct pxb_host_strands pxb_host_strands;
pxb_status pxb_host_strands_make(uint32_t n_strands, const uint32_t* counts, const float* points,
                                 const float* root_orientations, const float* particle_masses,
                                 const pxb_strand_params* params, pxb_host_strands** out);
pxb_status pxb_host_strands_destroy(pxb_host_strands* set);
pxb_status pxb_host_strands_view(pxb_host_strands* set, pxb_strand_set_desc* view_out);
/* Fills `out` with the reference's StrandParams defaults (physxcoopa/hair/strand.h:96-147). */
void pxb_strand_params_default(pxb_strand_params* out);

/* ------------------------------------------------------------------------------------------ */
/* Warm-start network. No counterpart in the reference (physxcoopa has no learned component).  */
/* Per free vertex of a cloth, after integration: 24 features (predicted displacement, velocity*/
/* at the substep start, the strain vectors of its 6 triangulation edges) -> 64 -> SiLU -> 64 ->*/
/* SiLU -> 3, a displacement                                                                  */
/* added to the predicted position before a few constraint iterations; the solver falls back   */
/* to the plain iteration count when the residual stays above the cloth's threshold. BF16      */
/* weights and activations, FP32 accumulation, on the tensor cores.                            */
/* ------------------------------------------------------------------------------------------ */

#define PXB_MLP_INPUTS 24
#define PXB_MLP_HIDDEN 64
#define PXB_MLP_OUTPUTS 3

/* Weights row-major (out x in), as a linear layer stores them. Inputs are normalised as
 * (x - in_mean) * in_scale; outputs are multiplied by out_scale. */
typedef struct pxb_mlp_weights {
    float w1[PXB_MLP_HIDDEN][PXB_MLP_INPUTS];
    float b1[PXB_MLP_HIDDEN];
    float w2[PXB_MLP_HIDDEN][PXB_MLP_HIDDEN];
    float b2[PXB_MLP_HIDDEN];
    float w3[PXB_MLP_OUTPUTS][PXB_MLP_HIDDEN];
    float b3[PXB_MLP_OUTPUTS];
    float in_mean[PXB_MLP_INPUTS];
    float in_scale[PXB_MLP_INPUTS];
    float out_scale[PXB_MLP_OUTPUTS];
} pxb_mlp_weights;

/* Installs / reads the context's network. */
pxb_status pxb_mlp_set_weights(pxb_context* ctx, const pxb_mlp_weights* weights);
pxb_status pxb_mlp_get_weights(pxb_context* ctx, pxb_mlp_weights* out);
/* Runs the installed network on n host feature rows (n x 24 floats) into out (n x 3). */
pxb_status pxb_mlp_infer(pxb_context* ctx, const float* features, uint32_t n, float* out);

/* Training: fits the network to n rows (host memory: features n x 24, targets n x 3, e.g. from
 * pxb_cloths_record) by mean squared error in normalised units with Adam (FP32, cosine
 * learning-rate schedule over the epochs), seeded initialisation and shuffling. The
 * normalisation comes from the data (feature mean and inverse standard deviation, target root
 * mean square). Installs the result; *final_loss (optional) receives the last epoch's mean
 * loss. */
typedef struct pxb_mlp_train_desc {
    uint32_t epochs;
    uint32_t batch;          /* rows per optimiser step */
    float learning_rate;     /* peak Adam step size */
    uint64_t seed;
} pxb_mlp_train_desc;
pxb_status pxb_mlp_train(pxb_context* ctx, const float* features, const float* targets, uint64_t n,
                         const pxb_mlp_train_desc* desc, float* final_loss);
/* Loss and gradients of the installed network over n rows, as one training batch computes them
 * (FP32): loss = mean over rows and outputs of (y - target / out_scale)^2. Gradients fill the
 * weight and bias fields of *grads. */
pxb_status pxb_mlp_loss_gradients(pxb_context* ctx, const float* features, const float* targets, uint64_t n,
                                  float* loss, pxb_mlp_weights* grads);

/* Warm-started step: as pxb_cloths_step, but in every substep each free particle (not pinned,
 * not anchored) is first moved by the network's displacement, then warm_iterations run; when
 * the residual -- the max relative strain of the stretch constraints, max |len / rest - 1| -- is
 * still above the cloth's threshold, the substep restarts from the unmoved prediction with the
 * plain iteration count. warm_iterations == 0 runs the plain solve and only measures the
 * residual (no network needed), which is how a caller calibrates thresholds. */
typedef struct pxb_warm_start_desc {
    uint32_t warm_iterations;
    float residual_threshold;  /* used when thresholds is NULL */
    const float* thresholds;   /* optional, one per cloth of the step */
    /* Fallback: 0 restarts the substep from the unmoved prediction with the plain iteration
     * count (the plain solver's result exactly); 1 keeps iterating from the warm state,
     * warm_iterations at a time, until the residual is within the threshold or the plain count
     * is reached. */
    uint32_t continue_iterations;
} pxb_warm_start_desc;

typedef struct pxb_cloth_warm_result {
    float residual;      /* max over the step's substeps of the residual it ended with */
    uint32_t fallbacks;  /* substeps whose residual after the warm iterations was too high */
    uint32_t substeps;
    uint32_t extra_iterations; /* iterations run after the warm ones, over the step */
} pxb_cloth_warm_result;

pxb_status pxb_cloths_step_warm(pxb_context* ctx, const pxb_cloth_step_desc* step, const pxb_warm_start_desc* warm);
/* Results of the last pxb_cloths_step_warm, per listed cloth (synchronizes the stream). */
pxb_status pxb_cloths_read_warm_results(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                        pxb_cloth_warm_result* out);
/* Training rows from the plain solver: advances the listed cloths by one plain step and, during
 * substep `substep`, records for every free particle the network's 24 input features and the
 * displacement the plain iterations moved it by (3 floats). At most `capacity` rows are written
 * to features (capacity x 24) and targets (capacity x 3), cloths in list order, particles in
 * device layout order; *rows_out is the number written. */
pxb_status pxb_cloths_record(pxb_context* ctx, const pxb_cloth_step_desc* step, uint32_t substep,
                             float* features, float* targets, uint64_t capacity, uint64_t* rows_out);

/* ------------------------------------------------------------------------------------------ */
/* Diagnostics                                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* Measures the achievable shared-memory bandwidth of the whole device (bytes read + written
 * per second, one 1024-thread CTA per SM copying float4s between two shared buffers). The
 * cloth kernel is bound by this figure; benchmarks use it as the roofline denominator. */
pxb_status pxb_measure_smem_bandwidth(pxb_context* ctx, double* bytes_per_second);
/* Self-check of the solver's division on this device (no counterpart in the reference): the
 * constraint direction d / |d| is computed as three correctly rounded quotients from one
 * reciprocal (Markstein's method). mismatches[0] counts divisor significands (every one of the
 * 2^23, at three exponents) whose refined reciprocal is not the correctly rounded one;
 * mismatches[1] counts, over `samples` seeded random constraints (3 quotients each), quotients
 * that differ from IEEE division. Both must be 0. */
pxb_status pxb_check_quotients(pxb_context* ctx, uint64_t samples, uint64_t seed, uint64_t mismatches[2]);
/* The same division over whole significands: for divisor significands [b_first, b_first +
 * b_count) (of the 2^23) and every numerator significand, the number of quotients that differ
 * from IEEE division (the full sweep, b_first 0 and b_count 2^23, is every case the method's
 * rounding depends on; it takes a few minutes). */
pxb_status pxb_check_quotient_significands(pxb_context* ctx, uint32_t b_first, uint32_t b_count, uint64_t* mismatches);
/* Self-check of one whole constraint projection: the solver's form (packed two-lane FP32
 * arithmetic, shared reciprocal) against the reference's scalar IEEE operations on `samples`
 * seeded random endpoint pairs (ordinary, near-zero and subnormal coordinates, signed zeros,
 * pinned endpoints, compliances and lambdas). *mismatches counts projections differing in any
 * output bit; the first such input (8 floats: a xyzw, b xyzw) goes to first_bad when not NULL. */
pxb_status pxb_check_projections(pxb_context* ctx, uint64_t samples, uint64_t seed, uint64_t* mismatches,
                                 float* first_bad);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* PHYSXCOOPA_B200_H */
