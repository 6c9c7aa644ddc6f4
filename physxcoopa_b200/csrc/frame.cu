// frame.cu -- pxb_cloths_step_frame / pxb_strands_step_frame: one cloth or strand frame as
// PhysicsWorld::step_cloths_ (physxcoopa/world.h:1749-1847) and step_strands_ (:1861-1957) run
// it, minus the collider gather, which stays the caller's.
//
// The per-cloth glue is evaluated on the host with the reference's formulas (anchor targets,
// the sleep gate and timer are a few floats per cloth); every changed anchor record goes to the
// device in one upload and one scatter launch, the awake cloths are solved in one batched step,
// and the cloths that fall asleep get their velocities zeroed by one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "host_math.h"
#include "pxb_internal.h"
#include "runtime_internal.h"

namespace {

struct AnchorWrite {
    PxbAnchorRec* dst;
    PxbAnchorRec rec;
};

struct VelZero {
    float4* vel;
    int32_t n;
    int32_t pad;
};

__global__ void scatter_anchor_records_kernel(const AnchorWrite* __restrict__ w, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) *w[i].dst = w[i].rec;
}

// Cloth::particles[i].velocity = 0 for every particle (world.h:1840); the slot's w (real particle
// or ghost) is kept.
__global__ void zero_velocities_kernel(const VelZero* __restrict__ z) {
    const VelZero c = z[blockIdx.y];
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < c.n; l += gridDim.x * blockDim.x) {
        const float4 v = c.vel[l];
        c.vel[l] = make_float4(0.0f, 0.0f, 0.0f, v.w);
    }
}

}  // namespace

extern "C" {

pxb_status pxb_cloths_step_frame(pxb_context* ctx, const pxb_cloth_frame_desc* fd, uint8_t* awake_out) {
    using namespace pxb::hm;
    if (!ctx || !fd || (fd->n_cloths && !fd->cloths)) return PXB_ERR_INVALID_ARGUMENT;
    const uint32_t n = fd->n_cloths;
    if (fd->n_bodies && !fd->bodies) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null bodies");
    // PhysicsWorld steps with its fixed, positive dt; a frame of no time is refused here rather
    // than half-run (the reference would still run its sleep bookkeeping on it)
    if (!(fd->dt > 0.0f)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "a frame needs dt > 0");
    std::vector<ClothEntry*> ents(n);
    for (uint32_t k = 0; k < n; ++k) {
        ents[k] = ctx->lookup(fd->cloths[k]);
        if (!ents[k]) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id %llu is not live", (unsigned long long)fd->cloths[k]);
        if (fd->collider_offsets && fd->collider_offsets[k + 1] < fd->collider_offsets[k])
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider offsets decrease");
        if (fd->source_offsets && fd->source_offsets[k + 1] < fd->source_offsets[k])
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "source offsets decrease");
    }
    if (fd->collider_offsets && fd->collider_offsets[n] && !fd->colliders)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null colliders");
    if (fd->source_offsets && fd->source_offsets[n] && !fd->sources)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null sources");

    // Substeps per frame, holding the internal substep at fixed_dt / cloth_substeps (world.h:1753-1756).
    const float internal_h =
        std::max(fd->fixed_dt / static_cast<float>(std::max(1u, fd->cloth_substeps)), 1e-6f);
    const uint32_t frame_substeps =
        std::clamp<uint32_t>(static_cast<uint32_t>(std::lround(fd->dt / internal_h)), 1u, 16u);

    // --- anchors from the bodies' live poses, then the sleep gate (world.h:1762-1825) ---
    std::vector<AnchorWrite> writes;
    std::vector<uint32_t> solve;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry& e = *ents[k];
        bool moved = false;
        for (size_t a = 0; a < e.anchors.size(); ++a) {
            pxb_anchor& A = e.anchors[a];
            const pxb_body_pose* b = nullptr;
            if (fd->bodies && A.body_index < fd->n_bodies && fd->bodies[A.body_index].alive &&
                fd->bodies[A.body_index].generation == A.body_generation)
                b = &fd->bodies[A.body_index];
            const V3 world = ld(A.world_position);
            const V3 target = b ? add(ld(b->position), qrot(ldq(b->orientation), ld(A.local_position))) : world;
            const V3 delta = sub(target, world);
            if (dot(delta, delta) > 1e-6f) moved = true;
            st(A.world_position, target);
            st(e.anchor_recs[a].world, target);
        }
        if (moved || (fd->collider_moving && fd->collider_moving[k])) {
            e.awake = true;
            e.sleep_timer = 0.0f;
        }
        if (!e.awake) {
            // the lerp's start stays where the sheet is, or waking would snap it (world.h:1819-1823)
            for (size_t a = 0; a < e.anchors.size(); ++a) {
                std::memcpy(e.anchors[a].prev_world_position, e.anchors[a].world_position, 12);
                std::memcpy(e.anchor_recs[a].prev, e.anchor_recs[a].world, 12);
            }
        } else {
            solve.push_back(k);
        }
        PxbAnchorRec* recs = reinterpret_cast<PxbAnchorRec*>(e.dev.anchors);  // 8 floats per anchor
        for (size_t a = 0; a < e.anchor_recs.size(); ++a) writes.push_back(AnchorWrite{recs + a, e.anchor_recs[a]});
    }
    if (!writes.empty()) {
        if (pxb_status s = ctx->grow(ctx->d_frame, sizeof(AnchorWrite) * writes.size(), "frame anchors")) return s;
        if (pxb_status s = ctx->cuda(cudaMemcpyAsync(ctx->d_frame.p, writes.data(), sizeof(AnchorWrite) * writes.size(),
                                                     cudaMemcpyHostToDevice, ctx->stream),
                                     "upload anchor targets"))
            return s;
        const int nw = static_cast<int>(writes.size());
        scatter_anchor_records_kernel<<<(nw + 255) / 256, 256, 0, ctx->stream>>>(
            static_cast<const AnchorWrite*>(ctx->d_frame.p), nw);
        if (pxb_status s = ctx->cuda(cudaGetLastError(), "launch anchor scatter")) return s;
        ++ctx->launches;
        // the buffer is reused below: let the scatter read it first
        if (pxb_status s = ctx->cuda(cudaStreamSynchronize(ctx->stream), "anchor scatter")) return s;
    }

    // --- one batched solve of the awake cloths (world.h:1827-1829) ---
    if (!solve.empty()) {
        std::vector<uint64_t> ids;
        std::vector<pxb_collider> cols;
        std::vector<uint32_t> coff(1, 0);
        std::vector<pxb_gravity_source> srcs;
        std::vector<uint32_t> soff(1, 0);
        for (uint32_t k : solve) {
            ids.push_back(fd->cloths[k]);
            if (fd->collider_offsets)
                for (uint32_t c = fd->collider_offsets[k]; c < fd->collider_offsets[k + 1]; ++c) cols.push_back(fd->colliders[c]);
            coff.push_back(static_cast<uint32_t>(cols.size()));
            if (fd->source_offsets)
                for (uint32_t c = fd->source_offsets[k]; c < fd->source_offsets[k + 1]; ++c) srcs.push_back(fd->sources[c]);
            soff.push_back(static_cast<uint32_t>(srcs.size()));
        }
        pxb_cloth_step_desc sd;
        std::memset(&sd, 0, sizeof(sd));
        sd.cloths = ids.data();
        sd.n_cloths = static_cast<uint32_t>(ids.size());
        sd.colliders = cols.empty() ? nullptr : cols.data();
        sd.collider_offsets = coff.data();
        std::memcpy(sd.gravity, fd->gravity, 12);
        sd.sources = srcs.empty() ? nullptr : srcs.data();
        sd.source_offsets = soff.data();
        sd.substeps = frame_substeps;
        sd.iterations = fd->cloth_iterations;
        sd.h = fd->dt;
        if (pxb_status s = ctx->step_cloths(&sd)) return s;
        {
            if (pxb_status s = ctx->fetch_results()) return s;
            // --- sleep bookkeeping on the solved cloths' max particle speed (world.h:1831-1845) ---
            std::vector<VelZero> zero;
            for (uint32_t k : solve) {
                ClothEntry& e = *ents[k];
                if (e.result.max_speed < e.params.sleep_threshold) {
                    e.sleep_timer += fd->dt;
                    if (e.sleep_timer >= e.params.sleep_time) {
                        e.awake = false;
                        zero.push_back(VelZero{e.dev.vel, e.n_layout, 0});
                        e.result.max_speed = 0.0f;
                    }
                } else {
                    e.sleep_timer = 0.0f;
                }
            }
            if (!zero.empty()) {
                if (pxb_status s = ctx->grow(ctx->d_frame, sizeof(VelZero) * zero.size(), "frame sleep")) return s;
                if (pxb_status s = ctx->cuda(cudaMemcpyAsync(ctx->d_frame.p, zero.data(), sizeof(VelZero) * zero.size(),
                                                             cudaMemcpyHostToDevice, ctx->stream),
                                             "upload sleeping cloths"))
                    return s;
                zero_velocities_kernel<<<dim3(8, static_cast<unsigned>(zero.size())), 256, 0, ctx->stream>>>(
                    static_cast<const VelZero*>(ctx->d_frame.p));
                if (pxb_status s = ctx->cuda(cudaGetLastError(), "launch velocity zeroing")) return s;
                ++ctx->launches;
                if (pxb_status s = ctx->cuda(cudaStreamSynchronize(ctx->stream), "velocity zeroing")) return s;
            }
        }
    }
    if (awake_out)
        for (uint32_t k = 0; k < n; ++k) awake_out[k] = ents[k]->awake ? 1 : 0;
    return ctx->check_device_error();
}

pxb_status pxb_strands_step_frame(pxb_context* ctx, const pxb_strand_frame_desc* fd, uint8_t* awake_out) {
    using namespace pxb::hm;
    if (!ctx || !fd || (fd->n_sets && !fd->sets)) return PXB_ERR_INVALID_ARGUMENT;
    const uint32_t n = fd->n_sets;
    if (!(fd->dt > 0.0f)) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "a frame needs dt > 0");
    std::vector<StrandEntry*> ents(n);
    for (uint32_t k = 0; k < n; ++k) {
        ents[k] = ctx->lookup_strands(fd->sets[k]);
        if (!ents[k]) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id %llu is not live", (unsigned long long)fd->sets[k]);
        if (fd->collider_offsets && fd->collider_offsets[k + 1] < fd->collider_offsets[k])
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider offsets decrease");
        if (fd->source_offsets && fd->source_offsets[k + 1] < fd->source_offsets[k])
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "source offsets decrease");
    }
    if (fd->collider_offsets && fd->collider_offsets[n] && !fd->colliders)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null colliders");
    if (fd->source_offsets && fd->source_offsets[n] && !fd->sources)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null sources");

    // substeps per frame (world.h:1862-1866), as for cloth
    const float internal_h =
        std::max(fd->fixed_dt / static_cast<float>(std::max(1u, fd->cloth_substeps)), 1e-6f);
    const uint32_t frame_substeps =
        std::clamp<uint32_t>(static_cast<uint32_t>(std::lround(fd->dt / internal_h)), 1u, 16u);

    // --- root-moved wake and the sleep gate (world.h:1873-1878, 1928-1940) ---
    std::vector<uint32_t> solve;
    for (uint32_t k = 0; k < n; ++k) {
        StrandEntry& e = *ents[k];
        if (e.n_strands == 0) continue;  // an empty set is skipped (world.h:1871)
        bool root_moved = false;
        for (uint32_t s = 0; s < e.n_strands && !root_moved; ++s) {
            const V3 delta = sub(ld(e.records[s].root_position), ld(e.records[s].prev_root_position));
            if (dot(delta, delta) > 1e-6f) root_moved = true;
        }
        if (root_moved || (fd->collider_moving && fd->collider_moving[k])) {
            e.awake = true;
            e.sleep_timer = 0.0f;
        }
        if (!e.awake) {
            // the root lerp starts where the groom is, or waking would snap it (world.h:1932-1939)
            for (pxb_strand& r : e.records) {
                std::memcpy(r.prev_root_position, r.root_position, 12);
                std::memcpy(r.prev_root_orientation, r.root_orientation, 16);
            }
            if (pxb_status s = ctx->upload_strand_records(e)) return s;
        } else {
            solve.push_back(k);
        }
    }

    // --- one batched solve of the awake sets (world.h:1942-1945) ---
    if (!solve.empty()) {
        std::vector<uint64_t> ids;
        std::vector<pxb_collider> cols;
        std::vector<uint32_t> coff(1, 0);
        std::vector<pxb_gravity_source> srcs;
        std::vector<uint32_t> soff(1, 0);
        for (uint32_t k : solve) {
            ids.push_back(fd->sets[k]);
            if (fd->collider_offsets)
                for (uint32_t c = fd->collider_offsets[k]; c < fd->collider_offsets[k + 1]; ++c) cols.push_back(fd->colliders[c]);
            coff.push_back(static_cast<uint32_t>(cols.size()));
            if (fd->source_offsets)
                for (uint32_t c = fd->source_offsets[k]; c < fd->source_offsets[k + 1]; ++c) srcs.push_back(fd->sources[c]);
            soff.push_back(static_cast<uint32_t>(srcs.size()));
        }
        pxb_strand_step_desc sd;
        std::memset(&sd, 0, sizeof(sd));
        sd.sets = ids.data();
        sd.n_sets = static_cast<uint32_t>(ids.size());
        sd.colliders = cols.empty() ? nullptr : cols.data();
        sd.collider_offsets = coff.data();
        std::memcpy(sd.gravity, fd->gravity, 12);
        sd.sources = srcs.empty() ? nullptr : srcs.data();
        sd.source_offsets = soff.data();
        sd.substeps = frame_substeps;
        sd.iterations = fd->cloth_iterations;
        sd.h = fd->dt;
        if (pxb_status s = pxb_strands_step(ctx, &sd)) return s;
        std::vector<pxb_cloth_frame_result> res(ids.size());
        if (pxb_status s = pxb_strands_read_results(ctx, ids.data(), static_cast<uint32_t>(ids.size()), res.data()))
            return s;
        // --- sleep bookkeeping on each solved set's max particle speed (world.h:1947-1955) ---
        std::vector<VelZero> zero;
        for (size_t j = 0; j < solve.size(); ++j) {
            StrandEntry& e = *ents[solve[j]];
            if (res[j].max_speed < e.params.sleep_threshold) {
                e.sleep_timer += fd->dt;
                if (e.sleep_timer >= e.params.sleep_time) {
                    e.awake = false;
                    zero.push_back(VelZero{e.dev.vel, static_cast<int32_t>(e.n_slots), 0});
                    e.bounds[6] = 0.0f;  // the speed the next read reports
                }
            } else {
                e.sleep_timer = 0.0f;
            }
        }
        if (!zero.empty()) {
            if (pxb_status s = ctx->grow(ctx->d_frame, sizeof(VelZero) * zero.size(), "frame sleep")) return s;
            if (pxb_status s = ctx->cuda(cudaMemcpyAsync(ctx->d_frame.p, zero.data(), sizeof(VelZero) * zero.size(),
                                                         cudaMemcpyHostToDevice, ctx->stream),
                                         "upload sleeping sets"))
                return s;
            zero_velocities_kernel<<<dim3(8, static_cast<unsigned>(zero.size())), 256, 0, ctx->stream>>>(
                static_cast<const VelZero*>(ctx->d_frame.p));
            if (pxb_status s = ctx->cuda(cudaGetLastError(), "launch velocity zeroing")) return s;
            ++ctx->launches;
            if (pxb_status s = ctx->cuda(cudaStreamSynchronize(ctx->stream), "velocity zeroing")) return s;
        }
    }
    if (awake_out)
        for (uint32_t k = 0; k < n; ++k) awake_out[k] = ents[k]->awake ? 1 : 0;
    return ctx->check_device_error();
}

pxb_status pxb_strands_read_sleep_state(pxb_context* ctx, const uint64_t* sets, uint32_t n, uint8_t* awake_out,
                                        float* sleep_timer_out) {
    if (!ctx || (n && !sets)) return PXB_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < n; ++k) {
        const StrandEntry* e = ctx->lookup_strands(sets[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id %llu is not live", (unsigned long long)sets[k]);
        if (awake_out) awake_out[k] = e->awake ? 1 : 0;
        if (sleep_timer_out) sleep_timer_out[k] = e->sleep_timer;
    }
    return PXB_OK;
}

pxb_status pxb_cloths_read_sleep_state(pxb_context* ctx, const uint64_t* cloths, uint32_t n, uint8_t* awake_out,
                                       float* sleep_timer_out) {
    if (!ctx || (n && !cloths)) return PXB_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < n; ++k) {
        const ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id %llu is not live", (unsigned long long)cloths[k]);
        if (awake_out) awake_out[k] = e->awake ? 1 : 0;
        if (sleep_timer_out) sleep_timer_out[k] = e->sleep_timer;
    }
    return PXB_OK;
}

}  // extern "C"
