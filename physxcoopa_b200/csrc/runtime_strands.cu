// runtime_strands.cu -- host runtime of the strand-set half of the C-ABI.
//
// A set is accepted on the device path when its layout is make_strands' (strand_builder.h:
// 58-127): strands contiguous in `particles`, stretch constraint (k-1, k) of each strand in the
// even batch when k-1 is even and in the odd batch otherwise, batches in that order. Device
// slots are strand-major with 32 per strand (one warp per strand, lane = particle).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "host_math.h"
#include "pxb_internal.h"
#include "pxb_kernels.h"
#include "runtime_internal.h"

using namespace pxb;

namespace {
size_t al256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
constexpr float kReferenceStep = 1.0f / 60.0f;  // hair::k_reference_step (strand_solver.h:63)
}  // namespace

StrandEntry* pxb_context::lookup_strands(uint64_t id) {
    const uint32_t index = static_cast<uint32_t>(id & 0xffffffffu);
    const uint32_t gen = static_cast<uint32_t>(id >> 32);
    if (index >= strand_sets.size()) return nullptr;
    StrandEntry& e = strand_sets[index];
    if (!e.alive || e.generation != gen) return nullptr;
    return &e;
}

pxb_status pxb_context::upload_strand_records(StrandEntry& e) {
    std::vector<float> r(16 * static_cast<size_t>(e.n_strands), 0.0f);
    for (uint32_t s = 0; s < e.n_strands; ++s) {
        const pxb_strand& q = e.records[s];
        float* o = &r[16 * static_cast<size_t>(s)];
        std::memcpy(o, q.root_position, 12);
        std::memcpy(o + 3, q.root_orientation, 16);
        std::memcpy(o + 8, q.prev_root_position, 12);
        std::memcpy(o + 11, q.prev_root_orientation, 16);
    }
    pxb_status s = cuda(cudaMemcpyAsync(const_cast<float*>(e.dev.roots), r.data(), 4 * r.size(),
                                        cudaMemcpyHostToDevice, stream), "upload roots");
    if (s) return s;
    return cuda(cudaStreamSynchronize(stream), "upload roots");
}

// The per-particle global-shape falloff pow(1 - k / (count - 1), falloff) (strand_solver.h:
// 227-229), evaluated on the host with the same single-precision operations as the reference.
pxb_status pxb_context::upload_strand_shape(StrandEntry& e) {
    std::vector<float> w(e.n_slots, 0.0f);
    for (uint32_t s = 0; s < e.n_strands; ++s) {
        const uint32_t n = e.count[s];
        if (n < 2) continue;
        const float inv_last = 1.0f / static_cast<float>(n - 1);
        for (uint32_t k = 1; k < n; ++k) {
            const float along = static_cast<float>(k) * inv_last;
            w[e.base[s] + k] = std::pow(1.0f - along, e.params.global_shape_falloff);
        }
    }
    pxb_status st = cuda(cudaMemcpyAsync(const_cast<float*>(e.dev.wshape), w.data(), 4 * w.size(),
                                         cudaMemcpyHostToDevice, stream), "upload shape weights");
    if (st) return st;
    return cuda(cudaStreamSynchronize(stream), "upload shape weights");
}

// Longest strand the device path takes: its positions and lambdas (20 B per particle) sit in one
// warp's share of shared memory.
constexpr uint32_t kMaxStrandParticles = 8192;

static pxb_status strands_upload_particles(pxb_context* ctx, StrandEntry& e, const pxb_particle* particles) {
    const size_t S = e.n_slots;
    std::vector<float4> pos(S, make_float4(0, 0, 0, 0)), vel(S, make_float4(0, 0, 0, 0)),
        prv(S, make_float4(0, 0, 0, 0));
    for (uint32_t s = 0; s < e.n_strands; ++s)
        for (uint32_t k = 0; k < e.count[s]; ++k) {
            const pxb_particle& p = particles[e.first[s] + k];
            const size_t l = e.base[s] + k;
            pos[l] = make_float4(p.position[0], p.position[1], p.position[2], p.inv_mass);
            vel[l] = make_float4(p.velocity[0], p.velocity[1], p.velocity[2], 0.0f);
            prv[l] = make_float4(p.prev_position[0], p.prev_position[1], p.prev_position[2], 0.0f);
        }
    pxb_status st = ctx->cuda(cudaMemcpyAsync(e.dev.pos, pos.data(), 16 * S, cudaMemcpyHostToDevice, ctx->stream), "upload strand pos");
    if (!st) st = ctx->cuda(cudaMemcpyAsync(e.dev.vel, vel.data(), 16 * S, cudaMemcpyHostToDevice, ctx->stream), "upload strand vel");
    if (!st) st = ctx->cuda(cudaMemcpyAsync(e.dev.prv, prv.data(), 16 * S, cudaMemcpyHostToDevice, ctx->stream), "upload strand prv");
    if (!st) st = ctx->cuda(cudaStreamSynchronize(ctx->stream), "upload strand particles");
    return st;
}

static pxb_status strands_add(pxb_context* ctx, const pxb_strand_set_desc* d, uint64_t* id_out) {
    if (!d || !id_out) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null argument");
    if (d->n_particles == 0 || d->n_strands == 0 || !d->particles || !d->strands)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "an empty strand set is refused (add_strands does the same)");
    if (!d->rest_local || !d->rest_offset || (d->n_stretch && !d->stretch) ||
        (d->n_stretch_batches && !d->stretch_batches))
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "null array with a nonzero count");
    StrandEntry e;
    e.n_particles = d->n_particles;
    e.n_strands = d->n_strands;
    e.n_stretch = d->n_stretch;
    uint32_t next = 0;
    for (uint32_t s = 0; s < d->n_strands; ++s) {
        const pxb_strand& q = d->strands[s];
        if (q.first != next) return ctx->fail(PXB_ERR_UNSUPPORTED, "strands are not contiguous (make_strands layout)");
        if (q.count > kMaxStrandParticles)
            return ctx->fail(PXB_ERR_TOO_LARGE, "strand %u has %u particles; the device path holds %u", s, q.count,
                             kMaxStrandParticles);
        e.first.push_back(q.first);
        e.count.push_back(q.count);
        next += q.count;
    }
    // slots: 32 per strand while every strand fits a warp's lanes; else each strand padded to a
    // multiple of 32 (the long-strand kernel's layout)
    uint32_t longest = 0;
    for (uint32_t c : e.count) longest = std::max(longest, c);
    const bool long_mode = longest > 32;
    for (uint32_t s = 0; s < d->n_strands; ++s) {
        e.base.push_back(static_cast<int32_t>(e.n_slots));
        e.n_slots += long_mode ? std::max<size_t>(32, (e.count[s] + 31) & ~31u) : 32;
    }
    if (next != d->n_particles) return ctx->fail(PXB_ERR_UNSUPPORTED, "particles outside the strands");
    // make_strands' stretch lists: even (k-1 even) constraints of every strand, then odd ones.
    std::vector<std::pair<uint32_t, uint32_t>> want;
    std::vector<int32_t> slot;
    for (int parity = 0; parity < 2; ++parity)
        for (uint32_t s = 0; s < d->n_strands; ++s)
            for (uint32_t k = 1; k < e.count[s]; ++k)
                if (static_cast<int>((k - 1) % 2) == parity) {
                    want.push_back({e.first[s] + k - 1, e.first[s] + k});
                    slot.push_back(e.base[s] + static_cast<int32_t>(k) - 1);
                }
    if (want.size() != d->n_stretch) return ctx->fail(PXB_ERR_UNSUPPORTED, "stretch list is not make_strands'");
    size_t n_even = 0;
    for (uint32_t s = 0; s < d->n_strands; ++s) n_even += e.count[s] / 2;
    std::vector<pxb_batch> batches;
    if (n_even) batches.push_back({0u, static_cast<uint32_t>(n_even)});
    if (want.size() > n_even) batches.push_back({static_cast<uint32_t>(n_even), static_cast<uint32_t>(want.size())});
    if (batches.size() != d->n_stretch_batches) return ctx->fail(PXB_ERR_UNSUPPORTED, "stretch batches are not make_strands'");
    for (size_t b = 0; b < batches.size(); ++b)
        if (batches[b].begin != d->stretch_batches[b].begin || batches[b].end != d->stretch_batches[b].end)
            return ctx->fail(PXB_ERR_UNSUPPORTED, "stretch batches are not make_strands'");
    for (size_t k = 0; k < want.size(); ++k)
        if (d->stretch[k].a != want[k].first || d->stretch[k].b != want[k].second)
            return ctx->fail(PXB_ERR_UNSUPPORTED, "stretch list is not make_strands'");
    e.stretch_slot = slot;
    e.topology.resize(d->n_stretch);
    for (uint32_t k = 0; k < d->n_stretch; ++k) e.topology[k] = {d->stretch[k].a, d->stretch[k].b, d->stretch[k].rest_length};
    e.records.assign(d->strands, d->strands + d->n_strands);
    e.params = d->params;
    e.time = d->time;

    // --- device buffers ---
    const size_t S = e.n_slots;
    size_t off = 0;
    auto take = [&](size_t b) { const size_t o = off; off += al256(std::max<size_t>(b, 16)); return o; };
    const size_t o_pos = take(16 * S), o_vel = take(16 * S), o_prv = take(16 * S), o_rl = take(16 * S),
                 o_ro = take(16 * S), o_rest = take(4 * S), o_w = take(4 * S), o_lam = take(4 * S),
                 o_cnt = take(4 * static_cast<size_t>(e.n_strands)), o_base = take(4 * static_cast<size_t>(e.n_strands)),
                 o_roots = take(64 * static_cast<size_t>(e.n_strands)),
                 o_keys = take(32), o_bounds = take(32);
    cudaError_t ce = cudaMalloc(&e.dmem, off);
    if (ce != cudaSuccess) return ctx->cuda(ce, "cudaMalloc(strands)");
    char* base = static_cast<char*>(e.dmem);
    e.dev.pos = reinterpret_cast<float4*>(base + o_pos);
    e.dev.vel = reinterpret_cast<float4*>(base + o_vel);
    e.dev.prv = reinterpret_cast<float4*>(base + o_prv);
    e.dev.rest_local = reinterpret_cast<const float4*>(base + o_rl);
    e.dev.rest_offset = reinterpret_cast<const float4*>(base + o_ro);
    e.dev.rest = reinterpret_cast<const float*>(base + o_rest);
    e.dev.wshape = reinterpret_cast<const float*>(base + o_w);
    e.dev.lam = reinterpret_cast<float*>(base + o_lam);
    e.dev.count = reinterpret_cast<const int32_t*>(base + o_cnt);
    e.dev.roots = reinterpret_cast<const float*>(base + o_roots);
    e.dev.bounds_next = reinterpret_cast<int*>(base + o_keys);
    e.dev.bounds_prev = reinterpret_cast<float*>(base + o_bounds);
    e.dev.bounds_out = e.dev.bounds_prev;
    e.dev.n_strands = static_cast<int32_t>(e.n_strands);
    e.dev.base = reinterpret_cast<const int32_t*>(base + o_base);
    e.dev.long_mode = long_mode ? 1 : 0;
    e.dev.pad_count = static_cast<int32_t>((longest + 31) & ~31u);
    // strands per block: as many as fit 96 KB of shared memory (20 B per slot), 1 to 8
    e.dev.warps = static_cast<int32_t>(std::min<uint32_t>(8, std::max<uint32_t>(1, 98304 / (20 * std::max(32u, (longest + 31) & ~31u)))));
    std::vector<float4> rl(S, make_float4(0, 0, 0, 0)), ro(S, make_float4(0, 0, 0, 0));
    std::vector<float> rest(S, 0.0f);
    std::vector<int32_t> cnt(e.count.begin(), e.count.end());
    for (uint32_t s = 0; s < e.n_strands; ++s)
        for (uint32_t k = 0; k < e.count[s]; ++k) {
            const size_t i = e.first[s] + k, l = e.base[s] + k;
            rl[l] = make_float4(d->rest_local[3 * i], d->rest_local[3 * i + 1], d->rest_local[3 * i + 2], 0.0f);
            ro[l] = make_float4(d->rest_offset[3 * i], d->rest_offset[3 * i + 1], d->rest_offset[3 * i + 2], 0.0f);
        }
    for (uint32_t k = 0; k < d->n_stretch; ++k) rest[slot[k]] = d->stretch[k].rest_length;
    // bounds the first step reads for a gravity source: compute_bounds over the particles
    float b[8] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f,
                  -3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < d->n_particles; ++i)
        for (int c = 0; c < 3; ++c) {
            const float x = d->particles[i].position[c];
            b[c] = x < b[c] ? x : b[c];
            b[3 + c] = b[3 + c] < x ? x : b[3 + c];
        }
    pxb_status st = PXB_OK;
    auto up = [&](size_t o, const void* src, size_t bytes) {
        if (!st && bytes) st = ctx->cuda(cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload strands");
    };
    up(o_rl, rl.data(), 16 * S);
    up(o_ro, ro.data(), 16 * S);
    up(o_rest, rest.data(), 4 * S);
    up(o_cnt, cnt.data(), 4 * cnt.size());
    up(o_base, e.base.data(), 4 * e.base.size());
    up(o_bounds, b, 32);
    if (!st) st = ctx->cuda(cudaMemsetAsync(base + o_lam, 0, 4 * S, ctx->stream), "zero lambdas");
    if (!st) st = ctx->upload_strand_records(e);
    if (!st) st = ctx->upload_strand_shape(e);
    if (!st) st = strands_upload_particles(ctx, e, d->particles);
    if (st) {
        cudaFree(e.dmem);
        return st;
    }
    std::memcpy(e.bounds, b, sizeof(e.bounds));
    uint32_t index = 0;
    while (index < ctx->strand_sets.size() && ctx->strand_sets[index].alive) ++index;
    if (index == ctx->strand_sets.size()) ctx->strand_sets.emplace_back();
    e.generation = ctx->strand_sets[index].generation + 1;
    e.alive = true;
    ctx->strand_sets[index] = std::move(e);
    *id_out = (static_cast<uint64_t>(ctx->strand_sets[index].generation) << 32) | index;
    return PXB_OK;
}

extern "C" {

void pxb_strand_params_default(pxb_strand_params* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    // hair::StrandParams defaults (physxcoopa/hair/strand.h:96-147)
    out->stretch_compliance = 0.0f;
    out->global_shape = 0.22f;
    out->global_shape_falloff = 1.6f;
    out->local_shape = 0.35f;
    out->damping = 0.08f;
    out->thickness = 0.01f;
    out->friction = 0.4f;
    out->gravity_scale = 1.0f;
    out->max_velocity = 50.0f;
    out->wind_turbulence = 0.1f;
    out->air_drag = 0.6f;
    out->substeps = 0;
    out->iterations = 0;
    out->sleep_threshold = 0.02f;
    out->sleep_time = 0.6f;
    out->layer = 0;
}

pxb_status pxb_strands_add(pxb_context* ctx, const pxb_strand_set_desc* desc, uint64_t* id_out) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    return strands_add(ctx, desc, id_out);
}

pxb_status pxb_strands_remove(pxb_context* ctx, uint64_t id) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    cudaStreamSynchronize(ctx->stream);
    cudaFree(e->dmem);
    const uint32_t gen = e->generation;
    *e = StrandEntry();
    e->generation = gen;
    return PXB_OK;
}

pxb_status pxb_strands_set_params(pxb_context* ctx, uint64_t id, const pxb_strand_params* params) {
    if (!ctx || !params) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    const float old_falloff = e->params.global_shape_falloff;
    e->params = *params;
    if (old_falloff != params->global_shape_falloff) return ctx->upload_strand_shape(*e);
    return PXB_OK;
}

pxb_status pxb_strands_set_roots(pxb_context* ctx, uint64_t id, const float* positions, uint32_t n_positions,
                                 const float* orientations, uint32_t n_orientations) {
    if (!ctx || (n_positions && !positions) || (n_orientations && !orientations)) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    const uint32_t n = std::min(e->n_strands, n_positions);
    for (uint32_t i = 0; i < n; ++i) {
        pxb_strand& s = e->records[i];
        std::memcpy(s.prev_root_position, s.root_position, 12);
        std::memcpy(s.prev_root_orientation, s.root_orientation, 16);
        std::memcpy(s.root_position, positions + 3 * static_cast<size_t>(i), 12);
        if (i < n_orientations) std::memcpy(s.root_orientation, orientations + 4 * static_cast<size_t>(i), 16);
    }
    return ctx->upload_strand_records(*e);
}

pxb_status pxb_strands_write_particles(pxb_context* ctx, uint64_t id, const pxb_particle* particles, uint32_t n) {
    if (!ctx || !particles) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    if (n != e->n_particles) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "particle count mismatch");
    return strands_upload_particles(ctx, *e, particles);
}

pxb_status pxb_strands_read_particles(pxb_context* ctx, uint64_t id, pxb_particle* out, uint32_t n) {
    if (!ctx || !out) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    if (n != e->n_particles) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "particle count mismatch");
    const size_t S = e->n_slots;
    std::vector<float4> pos(S), vel(S), prv(S);
    pxb_status st = ctx->cuda(cudaMemcpyAsync(pos.data(), e->dev.pos, 16 * S, cudaMemcpyDeviceToHost, ctx->stream), "read strand pos");
    if (!st) st = ctx->cuda(cudaMemcpyAsync(vel.data(), e->dev.vel, 16 * S, cudaMemcpyDeviceToHost, ctx->stream), "read strand vel");
    if (!st) st = ctx->cuda(cudaMemcpyAsync(prv.data(), e->dev.prv, 16 * S, cudaMemcpyDeviceToHost, ctx->stream), "read strand prv");
    if (!st) st = ctx->check_device_error();
    if (st) return st;
    for (uint32_t s = 0; s < e->n_strands; ++s)
        for (uint32_t k = 0; k < e->count[s]; ++k) {
            const size_t l = e->base[s] + k;
            pxb_particle& p = out[e->first[s] + k];
            p.position[0] = pos[l].x; p.position[1] = pos[l].y; p.position[2] = pos[l].z;
            p.inv_mass = pos[l].w;
            p.velocity[0] = vel[l].x; p.velocity[1] = vel[l].y; p.velocity[2] = vel[l].z;
            p.prev_position[0] = prv[l].x; p.prev_position[1] = prv[l].y; p.prev_position[2] = prv[l].z;
        }
    return PXB_OK;
}

pxb_status pxb_strands_read_lambdas(pxb_context* ctx, uint64_t id, float* out, uint32_t n) {
    if (!ctx || (n && !out)) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    if (n != e->n_stretch) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "lambda count mismatch");
    std::vector<float> lam(e->n_slots);
    pxb_status st = ctx->cuda(cudaMemcpyAsync(lam.data(), e->dev.lam, 4 * lam.size(), cudaMemcpyDeviceToHost, ctx->stream), "read lambdas");
    if (!st) st = ctx->check_device_error();
    if (st) return st;
    for (uint32_t k = 0; k < n; ++k) out[k] = lam[e->stretch_slot[k]];
    return PXB_OK;
}

pxb_status pxb_strands_read_strands(pxb_context* ctx, uint64_t id, pxb_strand* out, uint32_t n) {
    if (!ctx || (n && !out)) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    if (n != e->n_strands) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "strand count mismatch");
    std::memcpy(out, e->records.data(), sizeof(pxb_strand) * n);
    return PXB_OK;
}

pxb_status pxb_strands_read_time(pxb_context* ctx, uint64_t id, float* time_out) {
    if (!ctx || !time_out) return PXB_ERR_INVALID_ARGUMENT;
    StrandEntry* e = ctx->lookup_strands(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    *time_out = e->time;
    return PXB_OK;
}

pxb_status pxb_strands_step(pxb_context* ctx, const pxb_strand_step_desc* sd) {
    if (!ctx || !sd || (sd->n_sets && !sd->sets)) return PXB_ERR_INVALID_ARGUMENT;
    if (!(sd->h > 0.0f) || sd->n_sets == 0) return PXB_OK;  // solve_strands no-op (strand_solver.h:125)
    const uint32_t n = sd->n_sets;
    const uint32_t n_col = sd->collider_offsets ? sd->collider_offsets[n] : 0;
    const uint32_t n_src = sd->source_offsets ? sd->source_offsets[n] : 0;
    for (uint32_t k = 0; k < n_col; ++k) {
        const pxb_collider& c = sd->colliders[k];
        if (!c.enabled) continue;
        if (c.type < 0 || c.type > PXB_SHAPE_CONVEX_HULL || (c.type == PXB_SHAPE_CAPSULE && (c.capsule_axis < 0 || c.capsule_axis > 2)))
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider %u is malformed", k);
    }
    std::vector<StrandEntry*> ents(n);
    for (uint32_t k = 0; k < n; ++k) {
        ents[k] = ctx->lookup_strands(sd->sets[k]);
        if (!ents[k]) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
    }
    ColliderStage cstage;
    if (pxb_status s = cstage.plan(ctx, sd->colliders, n_col)) return s;
    // colliders, sources and posed hulls go up once for all sets
    const size_t b_cols = sizeof(PxbDevCollider) * std::max<uint32_t>(n_col, 1);
    const size_t o_geo = al256(b_cols) + al256(sizeof(pxb_gravity_source) * std::max<uint32_t>(n_src, 1));
    const size_t total = o_geo + al256(cstage.bytes());
    if (pxb_status s = ctx->grow(ctx->d_scratch, total, "strand step staging")) return s;
    std::vector<unsigned char> host(total, 0);
    char* db = static_cast<char*>(ctx->d_scratch.p);
    cstage.fill(ctx, sd->colliders, n_col, reinterpret_cast<PxbDevCollider*>(host.data()),
                reinterpret_cast<float4*>(host.data() + o_geo), reinterpret_cast<const float4*>(db + o_geo));
    if (n_src) std::memcpy(host.data() + al256(b_cols), sd->sources, sizeof(pxb_gravity_source) * n_src);
    if (pxb_status s = ctx->cuda(cudaMemcpyAsync(db, host.data(), total, cudaMemcpyHostToDevice, ctx->stream), "upload strand step")) return s;
    if (pxb_status s = ctx->cuda(cudaStreamSynchronize(ctx->stream), "upload strand step")) return s;
    const pxb::hm::V3 g = pxb::hm::ld(sd->gravity);
    for (uint32_t k = 0; k < n; ++k) {
        StrandEntry& e = *ents[k];
        const pxb_strand_params& Pm = e.params;
        PxbStrandStep p;
        std::memset(&p, 0, sizeof(p));
        // solve_strands prologue (strand_solver.h:127-155), evaluated as the reference does
        const uint32_t steps = std::max<uint32_t>(1, Pm.substeps ? Pm.substeps : sd->substeps);
        const uint32_t iters = std::max<uint32_t>(1, Pm.iterations ? Pm.iterations : sd->iterations);
        const float hs = sd->h / static_cast<float>(steps);
        const float inv_hs = 1.0f / hs;
        p.hs = hs;
        p.inv_hs = inv_hs;
        p.steps = static_cast<int32_t>(steps);
        p.iters = static_cast<int32_t>(iters);
        p.alpha = Pm.stretch_compliance * inv_hs * inv_hs;
        const pxb::hm::V3 acc = pxb::hm::add(pxb::hm::mul(g, Pm.gravity_scale), pxb::hm::ld(Pm.external_acceleration));
        pxb::hm::st(p.accel, acc);
        pxb::hm::st(p.gravity, g);
        p.gravity_scale = Pm.gravity_scale;
        std::memcpy(p.external_acceleration, Pm.external_acceleration, 12);
        p.max_velocity = Pm.max_velocity;
        p.max_speed2 = Pm.max_velocity * Pm.max_velocity;
        const float substep_fraction = hs / kReferenceStep;
        auto clamp01 = [](float x) { return std::min(std::max(x, 0.0f), 1.0f); };
        p.global_per_substep = 1.0f - std::pow(1.0f - clamp01(Pm.global_shape), substep_fraction);
        p.local_per_substep = 1.0f - std::pow(1.0f - clamp01(Pm.local_shape), substep_fraction);
        p.global_shape_on = Pm.global_shape > 0.0f ? 1 : 0;
        p.local_shape_on = Pm.local_shape > 0.0f ? 1 : 0;
        p.damping_factor = 1.0f / (1.0f + Pm.damping * hs);
        p.air_drag = Pm.air_drag;
        p.wind_turbulence = Pm.wind_turbulence;
        p.turbulence_amp = Pm.wind_turbulence * pxb::hm::length(pxb::hm::ld(Pm.wind));
        std::memcpy(p.wind, Pm.wind, 12);
        p.thickness = Pm.thickness;
        p.friction = Pm.friction;
        p.time = e.time;
        p.col_begin = sd->collider_offsets ? static_cast<int32_t>(sd->collider_offsets[k]) : 0;
        p.col_count = sd->collider_offsets ? static_cast<int32_t>(sd->collider_offsets[k + 1] - sd->collider_offsets[k]) : 0;
        p.src_begin = sd->source_offsets ? static_cast<int32_t>(sd->source_offsets[k]) : 0;
        p.src_count = sd->source_offsets ? static_cast<int32_t>(sd->source_offsets[k + 1] - sd->source_offsets[k]) : 0;
        cudaError_t le = launch_strand_step(e.dev, p, reinterpret_cast<const PxbDevCollider*>(db),
                                            reinterpret_cast<const pxb_gravity_source*>(db + al256(b_cols)),
                                            ctx->stream,
                                            cstage.any_geometry(static_cast<uint32_t>(p.col_begin),
                                                                static_cast<uint32_t>(p.col_count)));
        if (le != cudaSuccess) return ctx->cuda(le, "launch strand_step");
        ctx->launches += 3;
        for (uint32_t q = 0; q < steps; ++q) e.time += hs;  // StrandSet::time (strand_solver.h:323)
        e.has_result = false;
    }
    // The staging buffer is reused by the next call: let these launches finish reading it.
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "strand step");
}

pxb_status pxb_strands_read_results(pxb_context* ctx, const uint64_t* sets, uint32_t n, pxb_cloth_frame_result* out) {
    if (!ctx || (n && (!sets || !out))) return PXB_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < n; ++k) {
        StrandEntry* e = ctx->lookup_strands(sets[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "strand set id is not live");
        if (!e->has_result) {
            float b[8];
            pxb_status st = ctx->cuda(cudaMemcpyAsync(b, e->dev.bounds_prev, 32, cudaMemcpyDeviceToHost, ctx->stream), "read strand bounds");
            if (!st) st = ctx->check_device_error();
            if (st) return st;
            std::memcpy(e->bounds, b, sizeof(e->bounds));
            e->has_result = true;
        }
        std::memcpy(out[k].bounds_min, e->bounds, 12);
        std::memcpy(out[k].bounds_max, e->bounds + 3, 12);
        out[k].max_speed = std::sqrt(e->bounds[6]);
        out[k].time = e->time;
    }
    return PXB_OK;
}

pxb_status pxb_solve_strands_host(pxb_context* ctx, const pxb_strand_set_desc* desc, pxb_particle* particles,
                                  pxb_constraint* stretch, const pxb_collider* colliders, uint32_t n_colliders,
                                  const float gravity[3], uint32_t substeps, uint32_t iterations, float h,
                                  float* time_inout, float* bounds_out) {
    if (!ctx || !desc || !gravity) return PXB_ERR_INVALID_ARGUMENT;
    if (desc->n_particles == 0 || desc->n_strands == 0 || !(h > 0.0f)) return PXB_OK;
    HostSolveCache* hit = nullptr;
    for (HostSolveCache& c : ctx->strand_cache) {
        StrandEntry* e = c.particles == desc->particles ? ctx->lookup_strands(c.id) : nullptr;
        if (!e) continue;
        bool same = e->n_particles == desc->n_particles && e->n_strands == desc->n_strands && e->n_stretch == desc->n_stretch;
        for (uint32_t k = 0; same && k < desc->n_stretch; ++k)
            same = e->topology[k].a == desc->stretch[k].a && e->topology[k].b == desc->stretch[k].b &&
                   e->topology[k].rest == desc->stretch[k].rest_length;
        if (same) { hit = &c; break; }
        pxb_strands_remove(ctx, c.id);
        c.particles = nullptr;
    }
    uint64_t id = 0;
    pxb_status st;
    if (!hit) {
        if ((st = strands_add(ctx, desc, &id))) return st;
        ctx->strand_cache.push_back(HostSolveCache{desc->particles, id});
    } else {
        id = hit->id;
        StrandEntry* e = ctx->lookup_strands(id);
        if ((st = pxb_strands_set_params(ctx, id, &desc->params))) return st;
        if ((st = strands_upload_particles(ctx, *e, desc->particles))) return st;
        e->records.assign(desc->strands, desc->strands + desc->n_strands);
        if ((st = ctx->upload_strand_records(*e))) return st;
        e->time = desc->time;
    }
    StrandEntry* e = ctx->lookup_strands(id);
    if (time_inout) e->time = *time_inout;
    // the bounds a gravity source would read come from the caller's set (StrandSet::bounds);
    // without sources they are not read.
    const uint32_t offs[2] = {0, n_colliders};
    pxb_strand_step_desc sd{};
    sd.sets = &id;
    sd.n_sets = 1;
    sd.colliders = colliders;
    sd.collider_offsets = offs;
    std::memcpy(sd.gravity, gravity, 12);
    sd.substeps = substeps;
    sd.iterations = iterations;
    sd.h = h;
    if ((st = pxb_strands_step(ctx, &sd))) return st;
    if ((st = pxb_strands_read_particles(ctx, id, particles, desc->n_particles))) return st;
    if (stretch) {
        std::vector<float> lam(desc->n_stretch);
        if ((st = pxb_strands_read_lambdas(ctx, id, lam.data(), desc->n_stretch))) return st;
        for (uint32_t k = 0; k < desc->n_stretch; ++k) stretch[k].lambda = lam[k];
    }
    if (time_inout) *time_inout = e->time;
    if (bounds_out) {
        pxb_cloth_frame_result r;
        if ((st = pxb_strands_read_results(ctx, &id, 1, &r))) return st;
        std::memcpy(bounds_out, r.bounds_min, 12);
        std::memcpy(bounds_out + 3, r.bounds_max, 12);
    }
    return PXB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Builders: make_strands (strand_builder.h:58-127)
// ------------------------------------------------------------------------------------------

struct pxb_host_strands {
    std::vector<pxb_particle> particles;
    std::vector<pxb_constraint> stretch;
    std::vector<pxb_batch> batches;
    std::vector<float> rest_local, rest_offset;
    std::vector<pxb_strand> strands;
    pxb_strand_params params{};
};

extern "C" pxb_status pxb_host_strands_make(uint32_t n_strands, const uint32_t* counts, const float* points,
                                            const float* root_orientations, const float* particle_masses,
                                            const pxb_strand_params* params, pxb_host_strands** out) {
    if (!out || !params || (n_strands && (!counts || !points))) return PXB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* set = new (std::nothrow) pxb_host_strands();
    if (!set) return PXB_ERR_OUT_OF_MEMORY;
    set->params = *params;
    std::vector<pxb_constraint> even, odd;
    size_t off = 0;
    for (uint32_t i = 0; i < n_strands; ++i) {
        const float* pts = points + 3 * off;
        const uint32_t n = counts[i];
        off += n;
        if (n < 2) continue;  // fewer than two points is skipped
        pxb_strand s{};
        s.first = static_cast<uint32_t>(set->particles.size());
        s.count = n;
        std::memcpy(s.root_position, pts, 12);
        const float q_id[4] = {0.0f, 0.0f, 0.0f, 1.0f};
        std::memcpy(s.root_orientation, root_orientations ? root_orientations + 4 * static_cast<size_t>(i) : q_id, 16);
        std::memcpy(s.prev_root_position, s.root_position, 12);
        std::memcpy(s.prev_root_orientation, s.root_orientation, 16);
        const pxb::hm::Q4 q = pxb::hm::ldq(s.root_orientation);
        // glm::inverse(q) = conjugate(q) / dot(q, q)
        const float qq = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
        const pxb::hm::Q4 to_root{-q.x / qq, -q.y / qq, -q.z / qq, q.w / qq};
        const float mass = particle_masses ? particle_masses[i] : 0.001f;
        const float inv_mass = mass > 0.0f ? 1.0f / mass : 1.0f;
        const pxb::hm::V3 root = pxb::hm::ld(pts);
        for (uint32_t k = 0; k < n; ++k) {
            pxb_particle p{};
            std::memcpy(p.position, pts + 3 * k, 12);
            std::memcpy(p.prev_position, p.position, 12);
            p.inv_mass = k == 0 ? 0.0f : inv_mass;
            set->particles.push_back(p);
            const pxb::hm::V3 rl = pxb::hm::qrot(to_root, pxb::hm::sub(pxb::hm::ld(pts + 3 * k), root));
            set->rest_local.insert(set->rest_local.end(), {rl.x, rl.y, rl.z});
            const pxb::hm::V3 ro = k == 0 ? pxb::hm::V3{0.0f, 0.0f, 0.0f}
                                          : pxb::hm::sub(pxb::hm::ld(pts + 3 * k), pxb::hm::ld(pts + 3 * (k - 1)));
            set->rest_offset.insert(set->rest_offset.end(), {ro.x, ro.y, ro.z});
            if (k > 0) {
                pxb_constraint c{};
                c.a = s.first + k - 1;
                c.b = s.first + k;
                c.rest_length = pxb::hm::length(pxb::hm::sub(pxb::hm::ld(pts + 3 * k), pxb::hm::ld(pts + 3 * (k - 1))));
                ((k - 1) % 2 == 0 ? even : odd).push_back(c);
            }
        }
        set->strands.push_back(s);
    }
    set->stretch = even;
    set->stretch.insert(set->stretch.end(), odd.begin(), odd.end());
    if (!even.empty()) set->batches.push_back({0u, static_cast<uint32_t>(even.size())});
    if (!odd.empty()) set->batches.push_back({static_cast<uint32_t>(even.size()), static_cast<uint32_t>(even.size() + odd.size())});
    *out = set;
    return PXB_OK;
}

extern "C" pxb_status pxb_host_strands_destroy(pxb_host_strands* set) {
    delete set;
    return PXB_OK;
}

extern "C" pxb_status pxb_host_strands_view(pxb_host_strands* set, pxb_strand_set_desc* v) {
    if (!set || !v) return PXB_ERR_INVALID_ARGUMENT;
    std::memset(v, 0, sizeof(*v));
    v->particles = set->particles.data();
    v->n_particles = static_cast<uint32_t>(set->particles.size());
    v->stretch = set->stretch.data();
    v->n_stretch = static_cast<uint32_t>(set->stretch.size());
    v->stretch_batches = set->batches.data();
    v->n_stretch_batches = static_cast<uint32_t>(set->batches.size());
    v->rest_local = set->rest_local.data();
    v->rest_offset = set->rest_offset.data();
    v->strands = set->strands.data();
    v->n_strands = static_cast<uint32_t>(set->strands.size());
    v->params = set->params;
    v->time = 0.0f;
    return PXB_OK;
}

