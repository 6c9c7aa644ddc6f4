/*
 * xpbd_oracle.h -- CPU restatement of physxcoopa's XPBD cloth and hair substeps.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU path is compared against; nothing in
 * the shipped library links, loads or calls it. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it.
 *
 * Each function restates the reference algorithm stage by stage, in the reference's operation
 * order, in plain C99 single-precision arithmetic (compiled with -ffp-contract=off so no fused
 * multiply-add changes the rounding). Citations are to files of the physxcoopa tree.
 * The restatement is pinned against the reference's own headers compiled into oracle/_ref
 * (oracle/ref_driver.cpp) and against the known answers of the reference's tests.
 */
#ifndef PXB_XPBD_ORACLE_H
#define PXB_XPBD_ORACLE_H

#include <stdint.h>

#include "../include/physxcoopa_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A cloth in reference layout, mutable (the oracle advances it in place). */
typedef struct orc_cloth {
    pxb_particle* particles;
    uint32_t n_particles;
    pxb_constraint* stretch;
    uint32_t n_stretch;
    const pxb_batch* stretch_batches;
    uint32_t n_stretch_batches;
    pxb_constraint* bend;
    uint32_t n_bend;
    const pxb_batch* bend_batches;
    uint32_t n_bend_batches;
    const pxb_tether* tethers;
    uint32_t n_tethers;
    pxb_anchor* anchors;
    uint32_t n_anchors;
    const uint32_t* triangles;
    uint32_t n_triangle_indices;
    uint32_t columns;
    uint32_t rows;
    pxb_cloth_params params;
    float time;
    const float* stretch_batch_compliance; /* optional */
    const float* bend_batch_compliance;    /* optional */
    float bounds_min[3];
    float bounds_max[3];
} orc_cloth;

/* cloth::solve_cloth (cloth_solver.h:158-460), serial dispatch. Returns 0, or -1 for a
 * collider of unknown shape type. */
int orc_solve_cloth(orc_cloth* c, const pxb_collider* colliders, uint32_t n_colliders,
                    const float gravity[3], uint32_t substeps, uint32_t iterations, float h);

/* Collider geometry, registered under the ids pxb_collider::geometry names (1..1023). The hull
 * is kept as given and posed per call, as collision::world_posed_hull does; the mesh gets a
 * MeshBVH built by orc_bvh_build. */
int orc_geometry_set_hull(uint32_t id, const pxb_hull_desc* desc);
int orc_geometry_set_mesh(uint32_t id, const pxb_mesh_desc* desc);
/* A TriangleMesh::from_height_grid over geometry::HeightGrid(nx, ny, (cell_x, cell_y), heights)
 * (height_grid.h), queried through the grid's block pyramid as the reference does. */
int orc_geometry_set_height_grid(uint32_t id, int nx, int ny, float cell_x, float cell_y, const float* heights,
                                 uint32_t n_heights);
void orc_geometry_clear(void);

/* One MeshBVH node (mesh_bvh.h): bounds, children (left < 0 for a leaf) and the leaf's range of
 * the triangle order. */
typedef struct orc_bvh_node {
    float mn[3], mx[3];
    int32_t left, right;
    uint32_t tri_start, tri_count;
} orc_bvh_node;

/* MeshBVH::build (mesh_bvh.h) over n_tris triangles: writes the nodes (at most 2 * n_tris, root
 * first, in creation order) and the triangle order, returns the node count. In
 * oracle/xpbd_oracle_bvh.cpp: the split is std::nth_element, as in the reference. */
uint32_t orc_bvh_build(const float* vertices, const uint32_t* indices, uint32_t n_tris,
                       orc_bvh_node* nodes, uint32_t* order);

/* cloth::project_particle (cloth_collision.h:386-420). Returns 1 on hit, 0 on miss, -1 for an
 * unknown shape type. motion_start may be NULL. */
int orc_project_particle(const pxb_collider* collider, float thickness, float p[3],
                         float normal_out[3], float* depth_out, const float* motion_start);

/* PhysicsWorld::gravity_at (world.h:1186-1190 over field_at_ world.h:2048-2068). */
void orc_gravity_at(const float gravity[3], const pxb_gravity_source* sources,
                    uint32_t n_sources, const float p[3], float out[3]);

/* PhysicsWorld::cloth_centre_ (world.h:2072-2076): sequential mean particle position. */
void orc_cloth_centre(const pxb_particle* particles, uint32_t n, float out[3]);

/* The per-cloth body of PhysicsWorld::step_cloths_ that concerns the solver (world.h:1832-1834):
 * gravity = sources ? gravity_at(cloth_centre_) : gravity, then solve_cloth. */
int orc_step_cloth(orc_cloth* c, const pxb_collider* colliders, uint32_t n_colliders,
                   const float gravity[3], const pxb_gravity_source* sources,
                   uint32_t n_sources, uint32_t substeps, uint32_t iterations, float h);

/* A strand set in reference layout, mutable. rest_local / rest_offset: 3 floats per particle. */
typedef struct orc_strand_set {
    pxb_particle* particles;
    uint32_t n_particles;
    pxb_constraint* stretch;
    uint32_t n_stretch;
    const pxb_batch* stretch_batches;
    uint32_t n_stretch_batches;
    const float* rest_local;
    const float* rest_offset;
    pxb_strand* strands;
    uint32_t n_strands;
    pxb_strand_params params;
    float time;
    float bounds_min[3];
    float bounds_max[3];
} orc_strand_set;

/* hair::solve_strands (strand_solver.h:121-327). Returns 0, or -1 for a collider of unknown
 * shape type. */
int orc_solve_strands(orc_strand_set* s, const pxb_collider* colliders, uint32_t n_colliders,
                      const float gravity[3], uint32_t substeps, uint32_t iterations, float h);

/* The per-set body of PhysicsWorld::step_strands_ that concerns the solver (world.h:1941-1945):
 * gravity = sources ? gravity_at(bounds centre) : gravity, then solve_strands. */
int orc_step_strands(orc_strand_set* s, const pxb_collider* colliders, uint32_t n_colliders,
                     const float gravity[3], const pxb_gravity_source* sources,
                     uint32_t n_sources, uint32_t substeps, uint32_t iterations, float h);

/* hair::set_strand_roots (strand_builder.h:139-149); orientations may be NULL. */
void orc_set_strand_roots(orc_strand_set* s, const float* positions, uint32_t n_positions,
                          const float* orientations, uint32_t n_orientations);

/* cloth::max_particle_speed (cloth.h:330-336). */
float orc_max_particle_speed(const pxb_particle* particles, uint32_t n);

/* The substep count PhysicsWorld::step_cloths_ derives from a frame dt (world.h:1753-1757). */
uint32_t orc_frame_substeps(float dt, float fixed_dt, uint32_t cloth_substeps);

/* PhysicsWorld::step_cloths_'s per-cloth body (world.h:1762-1845) without the collider gather:
 * anchors from the bodies' poses, the sleep gate, the solve (orc_step_cloth with the frame's
 * substeps), the sleep bookkeeping. *awake / *sleep_timer are Cloth::awake / sleep_timer, read and
 * written. Returns 1 when the cloth was solved, 0 when it slept, -1 as orc_solve_cloth. */
int orc_world_step_cloth(orc_cloth* c, const pxb_body_pose* bodies, uint32_t n_bodies, int collider_moving,
                         const pxb_collider* colliders, uint32_t n_colliders, const float gravity[3],
                         const pxb_gravity_source* sources, uint32_t n_sources, float fixed_dt,
                         uint32_t cloth_substeps, uint32_t cloth_iterations, float dt, int* awake,
                         float* sleep_timer);

/* PhysicsWorld::step_strands_'s per-set body (world.h:1861-1957) without the collider gather: a
 * root that moved since the last target (|root - prev_root|^2 > k_epsilon) or a moving collider
 * wakes the set; a sleeping set only carries its roots' targets into their previous targets; an
 * awake set is solved (orc_step_strands with the frame's substeps, gravity at the bounds centre
 * when there are sources), then the sleep bookkeeping on its max particle speed. *awake /
 * *sleep_timer are StrandSet::awake / sleep_timer, read and written. Returns 1 when the set was
 * solved, 0 when it slept, -1 as orc_solve_strands. */
int orc_world_step_strands(orc_strand_set* s, int collider_moving, const pxb_collider* colliders,
                           uint32_t n_colliders, const float gravity[3], const pxb_gravity_source* sources,
                           uint32_t n_sources, float fixed_dt, uint32_t cloth_substeps,
                           uint32_t cloth_iterations, float dt, int* awake, float* sleep_timer);

#ifdef __cplusplus
}
#endif

#endif /* PXB_XPBD_ORACLE_H */
