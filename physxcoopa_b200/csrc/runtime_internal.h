// runtime_internal.h -- host-side state behind the C-ABI handles.
#ifndef PXB_RUNTIME_INTERNAL_H
#define PXB_RUNTIME_INTERNAL_H

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct TopologyEdge {
    uint32_t a, b;
    float rest;
};

// One registered cloth: host mirrors of what the reference keeps on the Cloth (params, time,
// anchors, tethers) plus the device-side description and its allocation.
struct ClothEntry {
    bool alive = false;
    bool grid = false;  // beyond a cluster: solved by every SM from global memory
    bool lean = false;  // only positions in shared memory (PxbClothDev::lean), one CTA or two
    bool soa = false;   // lean on one CTA with the positions as float arrays (PxbClothDev::lean 2)
    uint32_t generation = 0;
    uint32_t n_particles = 0;
    int cols = 0, rows = 0, Q = 0, S = 0, n_layout = 0;
    int n_colours = 0;
    std::vector<PxbSeg> segs;              // every rank's device segments, rank after rank
    std::vector<int> colour_is_bend;
    // One CTA of the cloth's cluster (see PxbRank); the host keeps the same fields.
    struct Rank {
        int row0 = 0, n_rows = 0, seg_begin = 0;
        std::vector<int> colour_seg;       // relative to seg_begin, n_colours + 1 entries
        int rest_off = 0, n_rest_pad = 0, lam_off = 0, n_lam = 0, smem = 0;
    };
    std::vector<Rank> ranks;
    uint32_t cross_mask = 0;
    std::vector<int32_t> colour_batch;     // colour -> reference batch index in its list
    std::vector<int32_t> rest_ref;         // global rest slot -> stretch index, or n_stretch + bend index (-1 padding)
    int n_rest_total = 0;
    int n_lam = 0;                         // lambda slots over all ranks
    int threads = 64;
    int warm_smem = 0;  // dynamic shared memory of the warm-start kernel (max over ranks)
    bool awake = true;        // Cloth::awake (cloth.h:312), kept by pxb_cloths_step_frame
    float sleep_timer = 0.0f; // Cloth::sleep_timer (cloth.h:313)
    bool self_ok = false;  // self-collision can run (one CTA, hash tables fit in shared memory)
    int self_smem = 0;     // dynamic shared memory with self-collision on
    int aero_grid = 0;
    // General topology (PxbClothDev::topology 1): runs in solve order, each run's batch (bend
    // flag, batch index) for its compliance, the packed endpoints of every item, and the
    // per-slot triangle index.
    bool list = false;
    bool list_gmem = false;  // its state exceeds one CTA's shared memory: solved in HBM (topology 2)
    int ref_columns = 0;     // Cloth::columns as given (self-collision's 1-ring exemption)
    std::vector<PxbRun> runs;
    std::vector<int2> run_batch;
    std::vector<uint64_t> item_ends;  // per item: a slot | b slot << 32
    int list_items_pad = 0;
    std::vector<int32_t> tri_off;
    std::vector<int4> tri_ent;
    uint32_t n_triangle_indices = 0;
    uint32_t n_stretch = 0, n_bend = 0, n_stretch_batches = 0, n_bend_batches = 0;
    std::vector<float> stretch_batch_comp, bend_batch_comp;
    std::vector<TopologyEdge> topology;
    std::vector<pxb_tether> tethers;
    std::vector<pxb_anchor> anchors;
    std::vector<PxbAnchorRec> anchor_recs;
    pxb_cloth_params params{};
    float time = 0.0f;
    PxbClothDev dev{};
    void* dmem = nullptr;
    size_t dbytes = 0;
    PxbFrameResult result{};
    bool has_result = false;
    int32_t last_slot = -1;  // launch slot in the last step (pxb_context::last_step)
    PxbWarmResult warm_result{};
    bool has_warm_result = false;
};

// General-topology endpoints stored as two words per item (more than 65535 layout slots).
inline bool list_wide(const ClothEntry& e) { return e.list && e.n_layout > kListNarrowSlots; }

// One registered strand set (hair::StrandSet mirrors + device buffers).
struct StrandEntry {
    bool alive = false;
    uint32_t generation = 0;
    uint32_t n_particles = 0, n_strands = 0, n_stretch = 0;
    std::vector<uint32_t> first, count;
    std::vector<int32_t> base;             // first device slot of each strand (PxbStrandDev)
    size_t n_slots = 0;                    // device slots over all strands
    std::vector<pxb_strand> records;       // root targets, host mirror
    std::vector<int32_t> stretch_slot;     // stretch list index -> device slot
    std::vector<TopologyEdge> topology;
    pxb_strand_params params{};
    float time = 0.0f;
    void* dmem = nullptr;
    PxbStrandDev dev{};
    float bounds[7] = {0, 0, 0, 0, 0, 0, 0};
    bool has_result = false;
    bool awake = true;         // StrandSet::awake (pxb_strands_step_frame)
    float sleep_timer = 0.0f;  // StrandSet::sleep_timer
};

// One registered collider geometry (pxb_geometry_create_hull / _mesh); id = index + 1.
struct GeometryEntry {
    bool alive = false;
    int type = 0;  // PXB_SHAPE_CONVEX_HULL or PXB_SHAPE_TRIANGLE_MESH
    // hull: host copy, posed on the host at every step
    std::vector<float> vertices;        // xyz
    std::vector<float> planes;          // xyzw
    std::vector<uint32_t> starts;       // faces + 1
    std::vector<uint32_t> face_vertices;
    // mesh: device copy of the hierarchy (PxbMeshNode) and triangles in its order (PxbMeshTri)
    void* dmem = nullptr;
    const float4* d_nodes = nullptr;
    const float4* d_tris = nullptr;  // a height grid: its record (see GridTris in pxb_device_math.cuh)
    int n_nodes = 0, depth = 0;
    bool grid = false;               // TriangleMesh::from_height_grid
};

// The colliders of one step as the device reads them: the records plus the hulls posed for this
// step (one block per distinct geometry and pose, shared by every record naming it).
struct ColliderStage {
    std::vector<size_t> hull_block;   // per record: offset of its posed hull in float4s, or SIZE_MAX
    std::vector<size_t> block_start;  // distinct posed hulls
    std::vector<uint32_t> block_record;
    std::vector<uint8_t> geo;         // per record: an enabled mesh or hull naming a geometry
    size_t n_float4 = 0;
    // Whether records [begin, begin + count) include a mesh or hull: such a launch needs the
    // kernel instantiated with those branches.
    bool any_geometry(uint32_t begin, uint32_t count) const {
        for (uint32_t k = begin; k < begin + count && k < geo.size(); ++k)
            if (geo[k]) return true;
        return false;
    }
    pxb_status plan(pxb_context* ctx, const pxb_collider* c, uint32_t n);
    size_t bytes() const { return n_float4 * 16; }
    // Writes the device records (out) and the posed hulls (host_geo, to be copied to dev_geo).
    void fill(const pxb_context* ctx, const pxb_collider* c, uint32_t n, PxbDevCollider* out, float4* host_geo,
              const float4* dev_geo) const;
};

// pxb_solve_cloth_host keeps the registration it made for a caller's arrays.
struct HostSolveCache {
    const pxb_particle* particles;
    uint64_t id;
};

struct pxb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t staged = nullptr;
    // Side streams for launch groups that run side by side: forked from `stream` after the
    // step's upload, joined back before anything else is queued on it.
    static constexpr int kSideStreams = 8;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kSideStreams] = {};
    uint32_t* d_err = nullptr;
    // whole-GPU path: polls of a grid-barrier wait before it expires, and the test setting that
    // makes every grid barrier unreachable (pxb_context_set_wait_test)
    uint32_t grid_wait_polls = 1u << 22;
    uint32_t grid_extra_arrivals = 0;
    std::string error;
    uint64_t launches = 0;
    std::vector<ClothEntry> cloths;
    bool registry_dirty = true;
    uint64_t registry_epoch = 0;  // advances with every change to the registry or a cloth's layout
    DevBuf d_registry, d_stage, d_results, d_gather, d_gather_meta, d_scratch;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    std::vector<uint64_t> last_step;  // ids of the last step, in launch-slot order
    // warm-start network: host copy of the weights and the packed device blob
    bool has_mlp = false;
    pxb_mlp_weights mlp{};
    DevBuf d_mlp, d_mlp_io;
    int n_sms = 148;
    bool results_fresh = false;
    std::vector<HostSolveCache> host_cache;
    std::vector<StrandEntry> strand_sets;
    std::vector<HostSolveCache> strand_cache;
    std::vector<GeometryEntry> geometries;
    const GeometryEntry* lookup_geometry(uint32_t id) const {
        return id >= 1 && id <= geometries.size() && geometries[id - 1].alive ? &geometries[id - 1] : nullptr;
    }
    int cloth_variant = 0;  // kernel block-size cap, see pxb_kernels.h (autotuned or set)
    int launch_mode = 1;    // 1: persistent CTAs popping a work queue per launch group; 0: one CTA per cloth
    // 1: a one-CTA grid cloth whose shared memory lets an SM hold k of its CTAs launches with
    // 1/k of the threads the kernel's register file allows, so k CTAs are resident at once;
    // 0: it launches with its own thread count (half its largest colour, up to the cap)
    int thread_fit = 1;
    // Block-size variant per layout class (PXB_TUNE_CLASSES: kernel instantiation x how many of
    // the cloth's CTAs shared memory lets an SM hold), stored + 1 (0: cloth_variant); set by the
    // autotuner. The last plain step records the layout slots each class launched.
    int class_variant[PXB_TUNE_CLASSES] = {};
    double class_work[PXB_TUNE_CLASSES] = {};
    bool soa_layouts = true;  // cloths added from now on may take the float-array lean layout
    bool lean_mid = true;     // ... and the lean layout where it lets an SM hold more of their CTAs
    unsigned char* gather_scratch = nullptr;  // pxb_cloths_gather_positions_device's static scratch
    DevBuf d_tune;          // cloth state saved across an autotune
    // Pipelined position read-back (pxb_cloths_read_positions_async): two device snapshots,
    // each gathered on `stream` and copied to the host on `copy_stream`, which waits for it.
    cudaStream_t copy_stream = nullptr;
    DevBuf d_snap[2], d_snap_meta[2];
    cudaEvent_t snap_ready[2] = {}, snap_copied[2] = {};
    bool snap_busy[2] = {false, false};
    int snap_next = 0;
    DevBuf d_res_snap[2];  // pxb_cloths_read_results_async: slots, times, gathered records
    cudaEvent_t res_ready[2] = {}, res_copied[2] = {};
    bool res_busy[2] = {false, false};
    int res_next = 0;

    ~pxb_context() {
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        for (int k = 0; k < 2; ++k) {
            for (DevBuf* b : {&d_snap[k], &d_snap_meta[k], &d_res_snap[k]})
                if (b->p) cudaFree(b->p);
            for (cudaEvent_t ev : {snap_ready[k], snap_copied[k], res_ready[k], res_copied[k]})
                if (ev) cudaEventDestroy(ev);
        }
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        for (ClothEntry& e : cloths)
            if (e.alive && e.dmem) cudaFree(e.dmem);
        for (StrandEntry& e : strand_sets)
            if (e.alive && e.dmem) cudaFree(e.dmem);
        for (GeometryEntry& g : geometries)
            if (g.alive && g.dmem) cudaFree(g.dmem);
        for (DevBuf* b : {&d_registry, &d_stage, &d_results, &d_gather, &d_gather_meta, &d_scratch, &d_tune, &d_mlp, &d_mlp_io, &d_wresults, &d_rec, &d_grid, &d_frame})
            if (b->p) cudaFree(b->p);
        if (pinned) cudaFreeHost(pinned);
        if (d_err) cudaFree(d_err);
        if (staged) cudaEventDestroy(staged);
        if (fork) cudaEventDestroy(fork);
        for (int k = 0; k < kSideStreams; ++k) {
            if (join[k]) cudaEventDestroy(join[k]);
            if (side[k]) cudaStreamDestroy(side[k]);
        }
        if (stream) cudaStreamDestroy(stream);
    }

    pxb_status fail(pxb_status s, const char* fmt, ...);
    pxb_status cuda(cudaError_t e, const char* what);
    pxb_status grow(DevBuf& b, size_t bytes, const char* what);
    pxb_status grow_pinned(size_t bytes);
    ClothEntry* lookup(uint64_t id);
    void refresh_layout(ClothEntry& e);
    pxb_status upload_mlp();
    pxb_status upload_segments(ClothEntry& e);
    pxb_status upload_particles(ClothEntry& e, const pxb_particle* particles);
    pxb_status upload_anchor_records(ClothEntry& e);
    pxb_status add_cloth(const pxb_cloth_desc* d, uint64_t* id_out);
    pxb_status sync_registry();
    // Warm-start / recording controls of a step (null: the plain kernel).
    struct WarmCfg {
        int warm_iters = 0;
        float tau = 0.0f;
        const float* taus = nullptr;      // per cloth, overrides tau
        int record = 0, record_substep = 0;
        float* rec_x = nullptr;           // device rows, cloth k from rec_row0[k]
        float* rec_y = nullptr;
        const int64_t* rec_row0 = nullptr;
        int continue_iters = 0;
    };
    pxb_status step_cloths(const pxb_cloth_step_desc* sd, const WarmCfg* warm = nullptr, bool use_graph = false);
    // the captured step (pxb_cloths_step_graph)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<uint64_t> graph_key, graph_pending;
    int graph_kernels = 0;
    void drop_graph();
    DevBuf d_wresults, d_rec, d_grid;
    DevBuf d_frame;  // pxb_cloths_step_frame: anchor records to scatter, cloths whose velocities to zero
    bool warm_fresh = false;
    bool last_step_warm = false;
    pxb_status fetch_warm_results();
    pxb_status check_device_error();
    pxb_status fetch_results();
    StrandEntry* lookup_strands(uint64_t id);
    pxb_status upload_strand_records(StrandEntry& e);
    pxb_status upload_strand_shape(StrandEntry& e);
};

// Collider snapshot -> device record with the reference's per-call world-space quantities.
void pxb_make_dev_collider(const pxb_collider& c, PxbDevCollider& o);

#endif  // PXB_RUNTIME_INTERNAL_H
