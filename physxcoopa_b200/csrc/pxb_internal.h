// pxb_internal.h -- host/device shared definitions of the B200 cloth / strand solver.
//
// Device data layout of one grid cloth (all in HBM, staged into shared memory per step):
//
//   layout index   l = y * S + (x % 4) * Q + x / 4,   Q = ceil(columns / 4), S = 4 * Q
//
// i.e. every row is split into the four "x mod 4" classes, each padded to Q slots. Slots with
// x >= columns are ghosts: pinned (inv_mass 0), never touched by a constraint, excluded from
// every reduction. In this order each of the 16 constraint colours of a make_grid_cloth sheet
// (cloth_builder.h:128-194) reads and writes CONTIGUOUS float4 runs, so a warp's shared-memory
// accesses are bank-conflict free for every colour.
//
// A colour is a list of affine segments. Item i of a segment is row r = i / per_row (computed
// as umulhi(i, magic) with magic = ceil(2^32 / per_row), checked exact on the host for every
// item), column k = i - r * per_row, and joins layout slots
//   la = a_base + r * row_stride + k,  lb = la + d
// reading its rest length from slot rest_base + i and, when the colour is compliant, its lambda
// from slot lam_base + i. The host derives the segments from the reference's own constraint
// lists and refuses the fast path unless they reproduce those lists exactly.
#ifndef PXB_INTERNAL_H
#define PXB_INTERNAL_H

#include <stdint.h>

#define PXB_MAX_COLOURS 16
#define PXB_MAX_SEGS 64
#define PXB_MAX_COLLIDERS_PER_CLOTH 64
#define PXB_EPSILON 1e-6f  // util::k_epsilon (physxcoopa/util/math.h:19)

// Error word bits a kernel may raise (never traps; the host reads them after the step).
#define PXB_DEVERR_BAD_INDEX 0x1u
#define PXB_DEVERR_TMA_TIMEOUT 0x2u
#define PXB_DEVERR_QUEUE_TIMEOUT 0x4u
#define PXB_DEVERR_MMA_TIMEOUT 0x8u

// 16-byte aligned: the kernel reads a descriptor as two 16-byte words.
struct alignas(16) PxbSeg {
    int32_t count;      // items (rows * per_row)
    uint32_t magic;     // ceil(2^32 / per_row): row of item i = umulhi(i, magic); 0 when per_row is 1
    int32_t per_row;    // items per row
    int32_t a_base;     // layout slot of item 0's `a`
    int32_t row_stride; // layout distance between rows
    int32_t d;          // lb - la
    int32_t rest_base;  // rest-length slot of item 0
    int32_t lam_base;   // lambda slot of item 0, or -1 when the colour has zero compliance
};

#define PXB_MAX_RANKS 8

// One CTA of a cloth's thread-block cluster: it holds rows [row0, row0 + n_rows) of the layout,
// its own colour segments (every item's `a` endpoint in its rows; `b` there or in the next
// rank's rows), rest lengths and lambdas. A cloth that fits one CTA has one rank.
struct PxbRank {
    int32_t row0, n_rows;
    int32_t seg_begin;                        // first segment of this rank in `segs`
    int32_t colour_seg[PXB_MAX_COLOURS + 1];  // colour c = segs[seg_begin + colour_seg[c] ...)
    int32_t rest_off, n_rest_pad;             // this rank's rest slots in `rest` (multiple of 4)
    int32_t lam_off, n_lam;                   // this rank's lambda slots in `lam_out`
    int32_t smem_bytes;                       // dynamic shared memory of this rank
};

// Static per-cloth description, device resident, written at registration.
struct PxbClothDev {
    float4* pos;            // [n_layout] xyz + inv_mass
    float4* vel;            // [n_layout] xyz + (1 real particle, 0 ghost)
    float4* prv;            // [n_layout] prev_position (start of the last substep)
    const float* rest;      // rest lengths, rank after rank
    float* lam_out;         // lambdas left by the last substep, rank after rank
    const int32_t* anchor_of;   // [n_layout] anchor record index or -1
    const int2* tether;         // [n_layout] (anchor layout slot or -1, max_length bits)
    float* anchors;             // [n_anchors * 8] prev xyz, pad, world xyz, pad
    const PxbSeg* segs;         // all ranks' segments
    PxbRank rank[PXB_MAX_RANKS];
    int32_t n_ranks;            // CTAs per cloth (cluster size)
    int32_t rows_per_rank;      // rows of every rank but the last
    int32_t n_colours;
    uint32_t cross_mask;        // bit c: colour c joins particles of different rows
    int32_t n_layout;
    int32_t n_real;
    int32_t columns, rows, Q, S;
    int32_t n_anchors;
    int32_t smem_bytes;         // max over ranks
    int32_t threads;            // block size this cloth runs with
    int32_t aero_grid;          // triangles are exactly make_grid_cloth's (cloth_builder.h:200-207)
    uint32_t stretch_mask;      // bit c: colour c comes from the stretch list
    uint32_t sync_mask;         // one CTA: bit c set = a CTA barrier after colour c (clear: colours
                                // c and c + 1 touch disjoint particles and run as one phase)
    const float* edge_rest;     // [6][n_layout] rest length to the grid neighbour (+x, -x, +y,
                                // -y, +x+y, -x-y), 0 where no stretch constraint joins them
    float4* disp;               // [n_layout] warm-start displacement scratch
    // Self-collision (one-CTA cloths): the spatial hash's bucket count (hash_bucket_count of the
    // particle count) and where in dynamic shared memory its tables live: PXB_SELF_WORDS words
    // from self_hash_off, in the rest-length region when they fit there (self_restage: the rest
    // lengths are staged again afterwards), else after the lambda region.
    int32_t self_buckets;
    int32_t self_hash_off;
    int32_t self_restage;
    // 0: grid layout (colour segments above). 1: general topology (any other mesh): one row of
    // `columns` = n particles, constraints as runs of PxbRun, aerodynamics over the triangle
    // index below; always one CTA. 2: the same with the state left in HBM (positions, rest
    // lengths and endpoints read in place, lambdas in list_scratch) for cloths whose state
    // exceeds one CTA's shared memory.
    int32_t topology;
    const struct PxbRun* runs;  // [n_runs], solved in order, one block barrier after each
    const int32_t* tri_off;     // [n_layout + 1] a slot's entries in tri_ent (ascending triangle)
    const int4* tri_ent;        // one entry per triangle corner: the triangle's three corner slots
    int32_t n_runs;
    int32_t list_items_pad;     // items padded to 4: rest lengths are rest[0, pad), the packed
                                // endpoint slots (a | b << 16) rest[pad, 2 * pad) as uint32 bits,
                                // or with more than kListNarrowSlots slots (a, b) pairs in
                                // rest[pad, 3 * pad)
    float* list_scratch;        // topology 2: lambdas / parked velocities in HBM, max(pad, 3 n_layout)
    int32_t ref_columns;        // Cloth::columns as given: self-collision's 1-ring exemption reads it
    // 1: a lean grid cloth: only positions in shared memory, its rest lengths and lambdas read in
    // place in HBM (rest + rank.rest_off, lam_out + rank.lam_off), velocities too; one or two CTAs.
    // 2: the same on one CTA with the positions held as float arrays (x and y as float2, z) and one byte
    // per slot indexing wtab, the cloth's distinct inverse masses in ascending bit order
    // (n_wtab <= PXB_MAX_WTAB of them); n_wtab == 0 reads the inverse masses in place from
    // pos[].w in HBM instead (a cloth with more distinct values than the table holds).
    int32_t lean;
    int32_t n_wtab;
    const float* wtab;
};

#define PXB_MAX_WTAB 256

// General-topology cloths: endpoint slots packed as a | b << 16 in one word while the layout has at
// most 65535 slots; beyond, as two words (a, b) (only in HBM: such a cloth never fits shared memory).
constexpr int kListNarrowSlots = 65535;
constexpr int kListMaxSlots = 1 << 24;

// A run of a general-topology cloth: consecutive items of one reference batch, no two of which
// share a particle, so its items are projected in parallel between two block barriers.
struct alignas(16) PxbRun {
    int32_t count;      // items (at least 1)
    int32_t item_base;  // first item's rest / endpoint slot
    int32_t lam_base;   // first item's lambda slot, or -1 when the batch has zero compliance
    float compliance;   // the batch's compliance; alpha = compliance / (hs * hs)
};

// Words of the self-collision tables: bucket ends (buckets + 1), the sorted particle indices (n)
// and a block-scan scratch (32).
#define PXB_SELF_WORDS(buckets, n) ((buckets) + 1 + (n) + 32)

// Warm-start controls of one cloth for one step (pxb_cloths_step_warm / pxb_cloths_record).
struct PxbWarmStep {
    float tau;              // fall back when the residual after warm_iters exceeds this
    int32_t warm_iters;     // iterations after the network's displacement; 0 = plain solve
    int32_t record;         // record training rows during substep record_substep
    int32_t record_substep;
    float* rec_x;           // [rows][24] features of every layout slot
    float* rec_y;           // [rows][4] displacement made by the plain iterations, free flag
    int64_t rec_row0;       // this cloth's first row
    int32_t continue_iters; // fallback: 0 restarts with the plain count, 1 keeps iterating
    int32_t pad0;
};

struct PxbWarmResult {
    float residual;         // max over the step's substeps of the final residual
    int32_t fallbacks;      // substeps that fell back to the plain iteration count
    int32_t substeps;
    int32_t extra_iterations;  // iterations beyond warm_iters, summed over the substeps
};

// One anchor target pair as the device keeps it (ClothAnchor::prev_world_position /
// world_position, cloth.h:152-159), 32 bytes.
struct PxbAnchorRec {
    float prev[3];
    float pad0;
    float world[3];
    float pad1;
};

// Collider snapshot with its world-space derived quantities precomputed on the host by the
// same formulas the reference evaluates per call (shape.h:160-188, obb.h:31-36).
struct PxbPose {
    float center[3];
    float ax[3], ay[3], az[3];  // box axes
    float ca[3], cb[3];         // capsule segment
    float t1[3];                // capsule on-axis fallback normal (orthonormal_basis)
};
struct PxbDevCollider {
    int32_t type;
    int32_t enabled;
    int32_t two_pose;       // swept Box / Capsule: probe both poses, keep the deeper
    int32_t swept_sphere;
    float radius;           // sphere radius or capsule radius
    float he[3];
    float sweep[3];
    float bmin[3], bmax[3];
    PxbPose pose[2];
    // ConvexHull: geo = this step's posed hull (see PxbHullStage), geo_count = faces,
    //   geo_aux = face-vertex entries.
    // TriangleMesh: geo = triangles in hierarchy order (PxbMeshTri), nodes = the hierarchy
    //   (PxbMeshNode, root first), geo_count = nodes (0: empty mesh), geo_aux = its depth;
    //   q / qi / origin / scale are project_at_pose_'s rot, inverse(rot), mesh_origin and scale
    //   (cloth_collision.h:209-213), evaluated on the host.
    int32_t geo_count;
    int32_t geo_aux;
    float q[4], qi[4];
    float origin[3];
    float scale;
    const float4* geo;
    const float4* nodes;
};

// Posed hull of one step, float4 records from PxbDevCollider::geo (F faces, V face-vertex entries):
//   [0, F)            world face normal xyz, w = its plane offset dot(n, first vertex)
//   [F, 2F)           x = first entry of the face (as int bits), y = its vertex count
//   [2F, 2F + V)      world position of each face-vertex entry
//   [2F + V, 2F + 2V) outward in-plane normal of the edge from that entry to the next
#define PXB_HULL_MAX_FACE_VERTICES 160  // k_hull_clip_cap (sat_hull.h:157)
#define PXB_HULL_MAX_FACES 4096
#define PXB_HULL_MAX_ENTRIES 65536

// Mesh hierarchy node: a = (min xyz, left child or -1 - first triangle for a leaf), b = (max xyz,
// right child or the leaf's triangle count), int fields as bits.
struct alignas(16) PxbMeshNode {
    float mn[3];
    int32_t left;
    float mx[3];
    int32_t right;
};
// Triangle in hierarchy order: the three vertices and TriangleMesh::triangle_normal, w unused.
struct alignas(16) PxbMeshTri {
    float v[3][4];
    float n[4];
};
#define PXB_MESH_MAX_DEPTH 60
#define PXB_MESH_MAX_TRIANGLES (1u << 24)

// Per cloth, per step, computed on the host (the prologue of solve_cloth, cloth_solver.h:162-194).
struct PxbClothStep {
    float hs, inv_hs, damping_factor, max_velocity, max_velocity2;
    float thickness, friction, air_drag, air_lift;
    float base_accel[3];     // used when n_sources == 0
    float gravity[3];        // world gravity (for the source field)
    float gravity_scale;
    float external_acceleration[3];
    float wind[3];
    float alpha[PXB_MAX_COLOURS];
    int32_t steps, iters, aero;
    int32_t col_begin, col_count, src_begin, src_count;
    int32_t write_lambdas;
    float self_distance;     // ClothParams::self_distance when self-collision runs, else 0
    int32_t self_collision;  // self_collision && self_distance > k_epsilon (cloth_solver.h:170)
    uint32_t grid_wait_polls;   // whole-GPU path: polls of a grid-barrier wait before it gives up
    uint32_t grid_extra_arrivals;  // 0; a test sets it so no grid barrier can complete
};

// One registered strand set on the device. Particles are strand-major, 32 slots per strand
// (slot = strand * 32 + k, k < count[strand] <= 32), or, when some strand is longer, each strand
// padded to a multiple of 32 slots from base[strand]; slot k's rest length and lambda are the
// stretch constraint (k, k + 1)'s.
struct PxbStrandDev {
    float4* pos;               // xyz + inv_mass
    float4* vel;
    float4* prv;
    const float4* rest_local;  // StrandSet::rest_local
    const float4* rest_offset; // StrandSet::rest_offset
    const float* rest;
    const float* wshape;       // pow(1 - k / (count - 1), global_shape_falloff), host-evaluated
    float* lam;
    const int32_t* count;
    const float* roots;        // 16 floats per strand: root pos, root q, pad, prev pos, prev q, pad
    int* bounds_next;          // 7 order-preserving keys reduced by the step
    float* bounds_prev;        // last decoded bounds: min xyz, max xyz, max speed^2
    float* bounds_out;         // where this step's decoded bounds go (same buffer, stream-ordered)
    int32_t n_strands;
    // 0: every strand has at most 32 particles, slot = strand * 32 + k (strand_step_kernel).
    // 1: some strand is longer: slot = base[strand] + k, strands padded to multiples of 32, solved
    //    by strand_long_kernel, `warps` strands per block, each with pad_count slots of shared memory.
    int32_t long_mode;
    const int32_t* base;
    int32_t pad_count;
    int32_t warps;
};

// Per set, per step: the prologue of solve_strands (strand_solver.h:127-155) on the host.
struct PxbStrandStep {
    float hs, inv_hs, alpha, damping_factor, max_velocity, max_speed2;
    float air_drag, wind_turbulence, turbulence_amp, thickness, friction;
    float global_per_substep, local_per_substep, time;
    float accel[3], gravity[3], gravity_scale, external_acceleration[3], wind[3];
    int32_t steps, iters, global_shape_on, local_shape_on;
    int32_t col_begin, col_count, src_begin, src_count;
};

// Inter-CTA state of one whole-GPU cloth launch (zeroed before the launch).
struct PxbGridSync {
    unsigned int count;      // barrier arrivals so far
    unsigned int gen;        // barriers completed
    float base_accel[3];     // gravity (+ external) selected for this step
    unsigned int keys[7];    // order-preserving keys: bounds min xyz, max xyz, max speed^2
    unsigned int pad[4];
};

struct PxbFrameResult {
    float bounds_min[3];
    float bounds_max[3];
    float max_speed;
    float time;
};

static_assert(sizeof(PxbSeg) == 32 && alignof(PxbSeg) == 16, "segment descriptor layout");
static_assert(sizeof(PxbClothStep) == 200, "per-step record size is part of the staging contract");
static_assert(sizeof(PxbDevCollider) == 312, "collider snapshot size is part of the staging contract");
static_assert(sizeof(PxbMeshNode) == 32 && sizeof(PxbMeshTri) == 64, "mesh record layout");

#endif  // PXB_INTERNAL_H
