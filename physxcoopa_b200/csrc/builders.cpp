// builders.cpp -- setup-time host builders of cloths (C-ABI pxb_host_cloth_*).
//
// Restates the reference's cloth construction so a cloth built here is the one the reference
// would build, array for array and bit for bit:
//   make_grid_cloth   physxcoopa/cloth/cloth_builder.h:81-219
//   pin_static        physxcoopa/cloth/cloth_builder.h:271-292
//   build_tethers     physxcoopa/cloth/cloth_builder.h:308-358
// plus one documented extension, a seeded jitter applied before rest lengths are captured, and
// pxb_host_cloth_make_mesh, a builder for arbitrary triangle meshes the reference does not have.
// These run once at setup, on the host (they allocate freely), never per frame.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <queue>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "host_math.h"

struct pxb_host_cloth {
    std::vector<pxb_particle> particles;
    std::vector<pxb_constraint> stretch;
    std::vector<pxb_batch> stretch_batches;
    std::vector<pxb_constraint> bend;
    std::vector<pxb_batch> bend_batches;
    std::vector<pxb_tether> tethers;
    std::vector<pxb_anchor> anchors;
    std::vector<uint32_t> triangles;
    std::vector<float> stretch_batch_compliance;  // filled when params.has_shear_compliance
    uint32_t columns = 0;
    uint32_t rows = 0;
    pxb_cloth_params params{};
    float time = 0.0f;
};

using pxb::hm::V3;

namespace {

// splitmix64 stream -> uniform float in [-amp, amp], 24-bit resolution.
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

V3 pos_of(const pxb_particle& p) { return V3{p.position[0], p.position[1], p.position[2]}; }

}  // namespace

extern "C" {

void pxb_cloth_params_default(pxb_cloth_params* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    // cloth::ClothParams defaults (physxcoopa/cloth/cloth.h:171-255)
    out->stretch_compliance = 0.0f;
    out->bend_compliance = 5e-5f;
    out->damping = 0.05f;
    out->thickness = 0.03f;
    out->friction = 0.5f;
    out->gravity_scale = 1.0f;
    out->max_velocity = 100.0f;
    out->wind_turbulence = 0.0f;
    out->air_drag = 0.02f;
    out->air_lift = 0.02f;
    out->self_collision = 0;
    out->self_distance = 0.0f;
    out->tether_scale = 1.02f;
    out->substeps = 0;
    out->iterations = 0;
    out->sleep_threshold = 0.05f;
    out->sleep_time = 0.5f;
    out->layer = 0;
    out->has_shear_compliance = 0;
    out->shear_compliance = 0.0f;
}

pxb_status pxb_host_cloth_make_grid(const pxb_grid_cloth_desc* desc, pxb_host_cloth** out) {
    if (!desc || !out) return PXB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* c = new (std::nothrow) pxb_host_cloth();
    if (!c) return PXB_ERR_OUT_OF_MEMORY;
    const uint32_t cols = std::max<uint32_t>(2, desc->columns);
    const uint32_t rows = std::max<uint32_t>(2, desc->rows);
    c->columns = cols;
    c->rows = rows;
    c->params = desc->params;

    const uint32_t count = cols * rows;
    const float eps = 1e-6f;
    const float particle_mass =
        (desc->total_mass > eps) ? desc->total_mass / static_cast<float>(count) : 0.0f;
    const float inv_mass = (particle_mass > eps) ? 1.0f / particle_mass : 0.0f;
    const float dx = desc->width / static_cast<float>(cols - 1);
    const float dy = desc->height / static_cast<float>(rows - 1);
    const pxb::hm::Q4 orient{desc->orientation[0], desc->orientation[1], desc->orientation[2],
                             desc->orientation[3]};
    const V3 center{desc->center[0], desc->center[1], desc->center[2]};

    // --- particles (cloth_builder.h:100-112), then the seeded jitter extension ---
    c->particles.resize(count);
    for (uint32_t y = 0; y < rows; ++y) {
        for (uint32_t x = 0; x < cols; ++x) {
            const V3 local{static_cast<float>(x) * dx - desc->width * 0.5f,
                           static_cast<float>(y) * dy - desc->height * 0.5f, 0.0f};
            const V3 p = pxb::hm::add(center, pxb::hm::qrot(orient, local));
            pxb_particle& q = c->particles[y * cols + x];
            q.position[0] = p.x; q.position[1] = p.y; q.position[2] = p.z;
            std::memcpy(q.prev_position, q.position, sizeof(q.position));
            q.velocity[0] = q.velocity[1] = q.velocity[2] = 0.0f;
            q.inv_mass = inv_mass;
        }
    }
    if (desc->jitter > 0.0f) {
        Jitter j{desc->jitter_seed};
        for (pxb_particle& q : c->particles) {
            q.position[0] += j.next(desc->jitter);
            q.position[1] += j.next(desc->jitter);
            q.position[2] += j.next(desc->jitter);
            std::memcpy(q.prev_position, q.position, sizeof(q.position));
        }
    }

    auto index_of = [cols](uint32_t x, uint32_t y) { return y * cols + x; };
    auto emit = [c](std::vector<pxb_constraint>& list, uint32_t a, uint32_t b) {
        pxb_constraint k;
        k.a = a;
        k.b = b;
        k.rest_length = pxb::hm::length(pxb::hm::sub(pos_of(c->particles[a]), pos_of(c->particles[b])));
        k.lambda = 0.0f;
        list.push_back(k);
    };
    auto close_batch = [](std::vector<pxb_constraint>& list, std::vector<pxb_batch>& batches,
                          uint32_t begin) {
        const uint32_t end = static_cast<uint32_t>(list.size());
        if (end > begin) batches.push_back(pxb_batch{begin, end});
    };
    std::vector<int> stretch_is_shear;
    auto close_stretch = [&](uint32_t begin, int shear) {
        const size_t before = c->stretch_batches.size();
        close_batch(c->stretch, c->stretch_batches, begin);
        if (c->stretch_batches.size() > before) stretch_is_shear.push_back(shear);
    };

    // --- structural, horizontal then vertical, by parity (cloth_builder.h:128-147) ---
    for (uint32_t parity = 0; parity < 2; ++parity) {
        const uint32_t begin = static_cast<uint32_t>(c->stretch.size());
        for (uint32_t y = 0; y < rows; ++y)
            for (uint32_t x = parity; x + 1 < cols; x += 2) emit(c->stretch, index_of(x, y), index_of(x + 1, y));
        close_stretch(begin, 0);
    }
    for (uint32_t parity = 0; parity < 2; ++parity) {
        const uint32_t begin = static_cast<uint32_t>(c->stretch.size());
        for (uint32_t y = parity; y + 1 < rows; y += 2)
            for (uint32_t x = 0; x < cols; ++x) emit(c->stretch, index_of(x, y), index_of(x, y + 1));
        close_stretch(begin, 0);
    }
    // --- shear, both diagonals by column parity (cloth_builder.h:153-172) ---
    if (desc->shear) {
        for (uint32_t parity = 0; parity < 2; ++parity) {
            const uint32_t begin = static_cast<uint32_t>(c->stretch.size());
            for (uint32_t y = 0; y + 1 < rows; ++y)
                for (uint32_t x = parity; x + 1 < cols; x += 2)
                    emit(c->stretch, index_of(x, y), index_of(x + 1, y + 1));
            close_stretch(begin, 1);
        }
        for (uint32_t parity = 0; parity < 2; ++parity) {
            const uint32_t begin = static_cast<uint32_t>(c->stretch.size());
            for (uint32_t y = 0; y + 1 < rows; ++y)
                for (uint32_t x = parity; x + 1 < cols; x += 2)
                    emit(c->stretch, index_of(x + 1, y), index_of(x, y + 1));
            close_stretch(begin, 1);
        }
    }
    // --- bend, two apart, modulo 4 (cloth_builder.h:177-194) ---
    for (uint32_t phase = 0; phase < 4; ++phase) {
        const uint32_t begin = static_cast<uint32_t>(c->bend.size());
        for (uint32_t y = 0; y < rows; ++y)
            for (uint32_t x = phase; x + 2 < cols; x += 4) emit(c->bend, index_of(x, y), index_of(x + 2, y));
        close_batch(c->bend, c->bend_batches, begin);
    }
    for (uint32_t phase = 0; phase < 4; ++phase) {
        const uint32_t begin = static_cast<uint32_t>(c->bend.size());
        for (uint32_t y = phase; y + 2 < rows; y += 4)
            for (uint32_t x = 0; x < cols; ++x) emit(c->bend, index_of(x, y), index_of(x, y + 2));
        close_batch(c->bend, c->bend_batches, begin);
    }
    // --- triangles (cloth_builder.h:199-207) ---
    c->triangles.reserve(static_cast<size_t>(cols - 1) * (rows - 1) * 6);
    for (uint32_t y = 0; y + 1 < rows; ++y) {
        for (uint32_t x = 0; x + 1 < cols; ++x) {
            const uint32_t i00 = index_of(x, y), i10 = index_of(x + 1, y);
            const uint32_t i01 = index_of(x, y + 1), i11 = index_of(x + 1, y + 1);
            c->triangles.insert(c->triangles.end(), {i00, i10, i11, i00, i11, i01});
        }
    }
    // --- self-collision distance default (cloth_builder.h:213-215) ---
    if (c->params.self_distance <= 0.0f) c->params.self_distance = 0.6f * std::min(dx, dy);
    // --- per-batch compliance extension: shear batches get their own compliance ---
    if (c->params.has_shear_compliance) {
        c->stretch_batch_compliance.resize(c->stretch_batches.size());
        for (size_t b = 0; b < c->stretch_batches.size(); ++b)
            c->stretch_batch_compliance[b] =
                stretch_is_shear[b] ? c->params.shear_compliance : c->params.stretch_compliance;
    }
    *out = c;
    return PXB_OK;
}

pxb_status pxb_host_cloth_make_mesh(const pxb_mesh_cloth_desc* desc, pxb_host_cloth** out) {
    if (!desc || !out) return PXB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const uint32_t n = desc->n_vertices;
    if (n == 0 || !desc->vertices || desc->n_indices % 3 != 0 || (desc->n_indices && !desc->indices))
        return PXB_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < desc->n_indices; ++k)
        if (desc->indices[k] >= n) return PXB_ERR_INVALID_ARGUMENT;
    auto* c = new (std::nothrow) pxb_host_cloth();
    if (!c) return PXB_ERR_OUT_OF_MEMORY;
    c->params = desc->params;
    // --- particles: mass spread evenly (the rule of cloth_builder.h:95-98) ---
    const float eps = 1e-6f;
    const float particle_mass = (desc->total_mass > eps) ? desc->total_mass / static_cast<float>(n) : 0.0f;
    const float inv_mass = (particle_mass > eps) ? 1.0f / particle_mass : 0.0f;
    c->particles.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        pxb_particle& q = c->particles[i];
        std::memcpy(q.position, desc->vertices + 3 * static_cast<size_t>(i), sizeof(q.position));
        std::memcpy(q.prev_position, q.position, sizeof(q.position));
        q.velocity[0] = q.velocity[1] = q.velocity[2] = 0.0f;
        q.inv_mass = inv_mass;
    }
    auto key = [](uint32_t a, uint32_t b) {
        return a < b ? (static_cast<uint64_t>(a) << 32 | b) : (static_cast<uint64_t>(b) << 32 | a);
    };
    auto make = [c](uint32_t a, uint32_t b) {
        pxb_constraint k;
        k.a = a;
        k.b = b;
        k.rest_length = pxb::hm::length(pxb::hm::sub(pos_of(c->particles[a]), pos_of(c->particles[b])));
        k.lambda = 0.0f;
        return k;
    };
    // --- distinct edges in first-appearance order, with the vertices opposite them ---
    std::vector<pxb_constraint> stretch, bend;
    std::vector<std::vector<uint32_t>> opposite;
    std::unordered_map<uint64_t, uint32_t> edge_of;
    const uint32_t nt = desc->n_indices / 3;
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t* v = desc->indices + 3 * static_cast<size_t>(t);
        for (int e = 0; e < 3; ++e) {
            const uint32_t a = v[e], b = v[(e + 1) % 3], o = v[(e + 2) % 3];
            if (a == b) continue;
            auto it = edge_of.find(key(a, b));
            if (it == edge_of.end()) {
                it = edge_of.emplace(key(a, b), static_cast<uint32_t>(stretch.size())).first;
                stretch.push_back(make(a, b));
                opposite.emplace_back();
            }
            opposite[it->second].push_back(o);
        }
    }
    if (desc->bend) {
        std::unordered_map<uint64_t, uint32_t> bend_of;
        for (size_t e = 0; e < stretch.size(); ++e) {
            if (opposite[e].size() != 2) continue;
            const uint32_t a = opposite[e][0], b = opposite[e][1];
            if (a == b || edge_of.count(key(a, b)) || bend_of.count(key(a, b))) continue;
            bend_of.emplace(key(a, b), static_cast<uint32_t>(bend.size()));
            bend.push_back(make(a, b));
        }
    }
    // --- greedy first-fit colouring, then the list stored batch by batch ---
    auto colour = [n](const std::vector<pxb_constraint>& list, std::vector<pxb_constraint>& sorted,
                      std::vector<pxb_batch>& batches) {
        std::vector<std::vector<uint8_t>> used;  // used[b][particle]
        std::vector<uint32_t> batch_of(list.size());
        for (size_t k = 0; k < list.size(); ++k) {
            size_t b = 0;
            while (b < used.size() && (used[b][list[k].a] || used[b][list[k].b])) ++b;
            if (b == used.size()) used.emplace_back(n, 0);
            used[b][list[k].a] = used[b][list[k].b] = 1;
            batch_of[k] = static_cast<uint32_t>(b);
        }
        sorted.clear();
        batches.clear();
        for (size_t b = 0; b < used.size(); ++b) {
            const uint32_t begin = static_cast<uint32_t>(sorted.size());
            for (size_t k = 0; k < list.size(); ++k)
                if (batch_of[k] == b) sorted.push_back(list[k]);
            batches.push_back(pxb_batch{begin, static_cast<uint32_t>(sorted.size())});
        }
    };
    colour(stretch, c->stretch, c->stretch_batches);
    colour(bend, c->bend, c->bend_batches);
    c->triangles.assign(desc->indices, desc->indices + desc->n_indices);
    if (c->params.self_distance <= 0.0f && !stretch.empty()) {
        float sum = 0.0f;
        for (const pxb_constraint& k : stretch) sum += k.rest_length;
        c->params.self_distance = 0.6f * (sum / static_cast<float>(stretch.size()));
    }
    *out = c;
    return PXB_OK;
}

pxb_status pxb_host_cloth_destroy(pxb_host_cloth* cloth) {
    delete cloth;
    return PXB_OK;
}

pxb_status pxb_host_cloth_pin_static(pxb_host_cloth* c, const float world_point[3], float radius,
                                     uint32_t* pinned_out) {
    if (!c || !world_point) return PXB_ERR_INVALID_ARGUMENT;
    const float r2 = radius * radius;
    const V3 wp{world_point[0], world_point[1], world_point[2]};
    uint32_t pinned = 0;
    for (uint32_t i = 0; i < c->particles.size(); ++i) {
        pxb_particle& p = c->particles[i];
        if (p.inv_mass == 0.0f) continue;
        const V3 d = pxb::hm::sub(pos_of(p), wp);
        if (pxb::hm::dot(d, d) > r2) continue;
        p.inv_mass = 0.0f;
        p.velocity[0] = p.velocity[1] = p.velocity[2] = 0.0f;
        pxb_anchor a{};
        a.particle = i;
        a.body_index = 0xFFFFFFFFu;  // dynamics::BodyId{}: invalid -> static pin
        a.body_generation = 0;
        std::memcpy(a.world_position, p.position, sizeof(a.world_position));
        std::memcpy(a.prev_world_position, p.position, sizeof(a.prev_world_position));
        c->anchors.push_back(a);
        ++pinned;
    }
    if (pinned_out) *pinned_out = pinned;
    return PXB_OK;
}

// cloth::pin_to_body (cloth_builder.h:235-258): the anchor's local position is
// inverse(orientation) * (p - body position), glm::inverse of a quaternion being its conjugate
// over its squared length.
pxb_status pxb_host_cloth_pin_to_body(pxb_host_cloth* c, uint32_t body_index, uint32_t body_generation,
                                      const float body_position[3], const float body_orientation[4],
                                      const float world_point[3], float radius, uint32_t* pinned_out) {
    if (!c || !body_position || !body_orientation || !world_point) return PXB_ERR_INVALID_ARGUMENT;
    const float r2 = radius * radius;
    const pxb::hm::Q4 q = pxb::hm::ldq(body_orientation);
    const float qq = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    const pxb::hm::Q4 inv_rot{-q.x / qq, -q.y / qq, -q.z / qq, q.w / qq};
    const V3 bp = pxb::hm::ld(body_position);
    const V3 wp{world_point[0], world_point[1], world_point[2]};
    uint32_t pinned = 0;
    for (uint32_t i = 0; i < c->particles.size(); ++i) {
        pxb_particle& p = c->particles[i];
        if (p.inv_mass == 0.0f) continue;  // already pinned by an earlier anchor
        const V3 d = pxb::hm::sub(pos_of(p), wp);
        if (pxb::hm::dot(d, d) > r2) continue;
        p.inv_mass = 0.0f;
        p.velocity[0] = p.velocity[1] = p.velocity[2] = 0.0f;
        pxb_anchor a{};
        a.particle = i;
        a.body_index = body_index;
        a.body_generation = body_generation;
        pxb::hm::st(a.local_position, pxb::hm::qrot(inv_rot, pxb::hm::sub(pos_of(p), bp)));
        std::memcpy(a.world_position, p.position, sizeof(a.world_position));
        std::memcpy(a.prev_world_position, p.position, sizeof(a.prev_world_position));
        c->anchors.push_back(a);
        ++pinned;
    }
    if (pinned_out) *pinned_out = pinned;
    return PXB_OK;
}

pxb_status pxb_host_cloth_build_tethers(pxb_host_cloth* c) {
    if (!c) return PXB_ERR_INVALID_ARGUMENT;
    c->tethers.clear();
    if (c->anchors.empty() || c->particles.empty()) return PXB_OK;
    const size_t n = c->particles.size();
    // Adjacency over the stretch graph, in list order (cloth_builder.h:316-320).
    std::vector<std::vector<uint32_t>> adjacency(n);
    for (const pxb_constraint& k : c->stretch) {
        adjacency[k.a].push_back(k.b);
        adjacency[k.b].push_back(k.a);
    }
    const float inf = std::numeric_limits<float>::max();
    std::vector<float> dist(n, inf);
    std::vector<uint32_t> source(n, 0);
    using Entry = std::pair<float, uint32_t>;
    std::priority_queue<Entry, std::vector<Entry>, std::greater<Entry>> frontier;
    for (const pxb_anchor& a : c->anchors) {
        dist[a.particle] = 0.0f;
        source[a.particle] = a.particle;
        frontier.push({0.0f, a.particle});
    }
    while (!frontier.empty()) {
        const Entry top = frontier.top();
        frontier.pop();
        if (top.first > dist[top.second]) continue;
        for (uint32_t next : adjacency[top.second]) {
            const float edge = pxb::hm::length(
                pxb::hm::sub(pos_of(c->particles[next]), pos_of(c->particles[top.second])));
            const float candidate = top.first + edge;
            if (candidate >= dist[next]) continue;
            dist[next] = candidate;
            source[next] = source[top.second];
            frontier.push({candidate, next});
        }
    }
    const float scale = std::max(1.0f, c->params.tether_scale);
    for (uint32_t i = 0; i < n; ++i) {
        if (c->particles[i].inv_mass == 0.0f) continue;
        if (dist[i] >= inf) continue;
        c->tethers.push_back(pxb_tether{i, source[i], dist[i] * scale});
    }
    return PXB_OK;
}

pxb_status pxb_host_cloth_build_tethers_device(pxb_context* ctx, pxb_host_cloth* c) {
    if (!ctx || !c) return PXB_ERR_INVALID_ARGUMENT;
    std::vector<pxb_tether> t(c->particles.size());
    uint32_t k = 0;
    const pxb_status s = pxb_build_tethers_device(
        ctx, c->particles.data(), static_cast<uint32_t>(c->particles.size()), c->stretch.data(),
        static_cast<uint32_t>(c->stretch.size()), c->anchors.data(), static_cast<uint32_t>(c->anchors.size()),
        c->params.tether_scale, t.data(), static_cast<uint32_t>(t.size()), &k);
    if (s) return s;  // the cloth keeps its tethers
    t.resize(k);
    c->tethers.swap(t);
    return PXB_OK;
}

pxb_status pxb_host_cloth_view(pxb_host_cloth* c, pxb_cloth_desc* v) {
    if (!c || !v) return PXB_ERR_INVALID_ARGUMENT;
    std::memset(v, 0, sizeof(*v));
    v->particles = c->particles.data();
    v->n_particles = static_cast<uint32_t>(c->particles.size());
    v->stretch = c->stretch.data();
    v->n_stretch = static_cast<uint32_t>(c->stretch.size());
    v->stretch_batches = c->stretch_batches.data();
    v->n_stretch_batches = static_cast<uint32_t>(c->stretch_batches.size());
    v->bend = c->bend.data();
    v->n_bend = static_cast<uint32_t>(c->bend.size());
    v->bend_batches = c->bend_batches.data();
    v->n_bend_batches = static_cast<uint32_t>(c->bend_batches.size());
    v->tethers = c->tethers.data();
    v->n_tethers = static_cast<uint32_t>(c->tethers.size());
    v->anchors = c->anchors.data();
    v->n_anchors = static_cast<uint32_t>(c->anchors.size());
    v->triangles = c->triangles.data();
    v->n_triangle_indices = static_cast<uint32_t>(c->triangles.size());
    v->columns = c->columns;
    v->rows = c->rows;
    v->params = c->params;
    v->time = c->time;
    v->stretch_batch_compliance =
        c->stretch_batch_compliance.empty() ? nullptr : c->stretch_batch_compliance.data();
    v->bend_batch_compliance = nullptr;
    return PXB_OK;
}

pxb_status pxb_host_cloth_mutable(pxb_host_cloth* c, pxb_particle** particles,
                                  pxb_anchor** anchors, pxb_cloth_params** params) {
    if (!c) return PXB_ERR_INVALID_ARGUMENT;
    if (particles) *particles = c->particles.data();
    if (anchors) *anchors = c->anchors.data();
    if (params) *params = &c->params;
    return PXB_OK;
}

}  // extern "C"
