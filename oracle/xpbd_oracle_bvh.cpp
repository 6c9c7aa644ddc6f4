/*
 * xpbd_oracle_bvh.cpp -- the oracle's MeshBVH::build (physxcoopa/geometry/mesh_bvh.h).
 *
 * TEST INFRASTRUCTURE ONLY, part of the oracle (see xpbd_oracle.h). C++ because the reference
 * partitions with std::nth_element, whose placement of equal and unequal keys within each half
 * is the standard library's; calling the same function keeps the oracle's triangle order, and
 * so the order its queries visit triangles in, the reference's. Compiled with
 * -ffp-contract=off like the rest of the oracle.
 */
#include <algorithm>
#include <limits>
#include <vector>

#include "xpbd_oracle.h"

namespace {

struct Builder {
    std::vector<float> tmin, tmax, cen;  // 3 per triangle
    uint32_t* order;
    orc_bvh_node* nodes;
    uint32_t n_nodes = 0;

    int32_t build(size_t start, size_t end) {
        float mn[3], mx[3];
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::numeric_limits<float>::max();
            mx[k] = std::numeric_limits<float>::lowest();
        }
        for (size_t i = start; i < end; ++i) {  // AABB::merge: glm::min / glm::max
            const uint32_t t = order[i];
            for (int k = 0; k < 3; ++k) {
                if (tmin[3 * t + k] < mn[k]) mn[k] = tmin[3 * t + k];
                if (mx[k] < tmax[3 * t + k]) mx[k] = tmax[3 * t + k];
            }
        }
        const size_t count = end - start;
        const int32_t idx = static_cast<int32_t>(n_nodes++);
        orc_bvh_node& nd = nodes[idx];
        for (int k = 0; k < 3; ++k) {
            nd.mn[k] = mn[k];
            nd.mx[k] = mx[k];
        }
        nd.left = -1;
        nd.right = -1;
        nd.tri_start = 0;
        nd.tri_count = 0;
        if (count <= 4) {  // k_leaf_threshold
            nd.tri_start = static_cast<uint32_t>(start);
            nd.tri_count = static_cast<uint32_t>(count);
            return idx;
        }
        const float ext[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
        int axis = 0;
        if (ext[1] > ext[axis]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        const size_t mid = start + count / 2;
        std::nth_element(order + start, order + mid, order + end,
                         [&](uint32_t a, uint32_t b) { return cen[3 * a + axis] < cen[3 * b + axis]; });
        const int32_t left = build(start, mid);
        const int32_t right = build(mid, end);
        nodes[idx].left = left;
        nodes[idx].right = right;
        return idx;
    }
};

}  // namespace

extern "C" uint32_t orc_bvh_build(const float* v, const uint32_t* idx, uint32_t n_tris, orc_bvh_node* nodes,
                                  uint32_t* order) {
    if (n_tris == 0) return 0;
    Builder b;
    b.order = order;
    b.nodes = nodes;
    b.tmin.resize(3 * n_tris);
    b.tmax.resize(3 * n_tris);
    b.cen.resize(3 * n_tris);
    for (uint32_t t = 0; t < n_tris; ++t) {
        order[t] = t;
        const float* p0 = &v[3 * idx[3 * t]];
        const float* p1 = &v[3 * idx[3 * t + 1]];
        const float* p2 = &v[3 * idx[3 * t + 2]];
        for (int k = 0; k < 3; ++k) {
            // glm::min(v0, glm::min(v1, v2)): min(a, b) = b < a ? b : a
            const float m12 = p2[k] < p1[k] ? p2[k] : p1[k];
            b.tmin[3 * t + k] = m12 < p0[k] ? m12 : p0[k];
            const float x12 = p1[k] < p2[k] ? p2[k] : p1[k];
            b.tmax[3 * t + k] = p0[k] < x12 ? x12 : p0[k];
            b.cen[3 * t + k] = (p0[k] + p1[k] + p2[k]) * (1.0f / 3.0f);
        }
    }
    b.build(0, n_tris);
    return b.n_nodes;
}
