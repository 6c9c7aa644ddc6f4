// facade_check.cpp -- the C++ drop-in facade (include/physxcoopa_b200.hpp) against the
// reference's own code: a grid cloth and a strand set built by the reference's builders are
// advanced by the reference's solve_cloth / solve_strands on one copy and by the facade on the
// device on another; every particle must come out equal. Exit status 0 on success.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include <physxcoopa/cloth/cloth_builder.h>
#include <physxcoopa/cloth/cloth_solver.h>
#include <physxcoopa/hair/strand_builder.h>
#include <physxcoopa/hair/strand_solver.h>

#include "../../include/physxcoopa_b200.hpp"

namespace px = coopa::physx;

static int compare(const char* what, const std::vector<px::cloth::ClothParticle>& a,
                   const std::vector<px::cloth::ClothParticle>& b) {
    int bad = 0;
    float worst = 0.0f;
    for (size_t i = 0; i < a.size(); ++i) {
        for (int c = 0; c < 3; ++c) {
            const float d = std::fabs(a[i].position[c] - b[i].position[c]);
            worst = d > worst ? d : worst;
            if (a[i].position[c] != b[i].position[c] || a[i].velocity[c] != b[i].velocity[c]) ++bad;
        }
    }
    std::printf("%s: %zu particles, %d differing components, max |dp| %.3g\n", what, a.size(), bad, worst);
    return bad;
}

int main() {
    pxb::b200::Device dev(0);
    // --- cloth: a 24x24 sheet pinned at two corners, draped over a sphere ---
    px::cloth::GridClothDesc g;
    g.columns = 24;
    g.rows = 24;
    g.width = 1.15f;
    g.height = 1.15f;
    g.center = glm::vec3(0.0f, 0.0f, 1.0f);
    px::cloth::Cloth ref = px::cloth::make_grid_cloth(g);
    px::cloth::pin_static(ref, glm::vec3(-0.575f, 0.575f, 1.0f), 0.01f);
    px::cloth::pin_static(ref, glm::vec3(0.575f, 0.575f, 1.0f), 0.01f);
    px::cloth::build_tethers(ref);
    px::cloth::Cloth mine = ref;
    px::collision::Shape ball = px::collision::Shape::make_sphere(0.3f);
    px::cloth::ClothCollider col;
    col.shape = &ball;
    col.position = glm::vec3(0.0f, 0.0f, 0.5f);
    col.bounds = px::collision::world_bounds(ball, col.position, col.orientation);
    const std::vector<px::cloth::ClothCollider> cols = {col};
    px::cloth::ClothSolverScratch s1, s2;
    for (int i = 0; i < 120; ++i) {
        px::cloth::solve_cloth(ref, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s1);
        // the reference's own signature: only the namespace differs from the line above
        pxb::b200::solve_cloth(mine, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s2);
    }
    int bad = compare("cloth 24x24, 120 frames", ref.particles, mine.particles);
    bad += ref.time != mine.time;
    bad += ref.bounds.min != mine.bounds.min || ref.bounds.max != mine.bounds.max;

    // --- hair: straight strands falling onto a sphere, no local shape (exact path) ---
    std::vector<px::hair::StrandDesc> descs;
    for (int s = 0; s < 16; ++s) {
        px::hair::StrandDesc d;
        for (int k = 0; k < 12; ++k) d.points.push_back(glm::vec3(0.05f * k, 0.01f * s, 0.6f));
        descs.push_back(d);
    }
    px::hair::StrandParams hp;
    hp.local_shape = 0.0f;
    px::hair::StrandSet href = px::hair::make_strands(descs, hp);
    px::hair::StrandSet hmine = href;
    px::hair::StrandSolverScratch h1, h2;
    for (int i = 0; i < 90; ++i) {
        px::hair::solve_strands(href, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 4, 1.0f / 60.0f, h1);
        pxb::b200::solve_strands(hmine, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 4, 1.0f / 60.0f, h2);
    }
    bad += compare("strands 16x12, 90 frames", href.particles, hmine.particles);
    // strands longer than a warp's 32 lanes, beside short ones (the long-strand kernel)
    std::vector<px::hair::StrandDesc> ldescs;
    for (int s = 0; s < 6; ++s) {
        px::hair::StrandDesc d;
        for (int k = 0; k < 20 + 23 * s; ++k) d.points.push_back(glm::vec3(0.02f * k, 0.01f * s, 0.6f));
        ldescs.push_back(d);
    }
    px::hair::StrandSet lhref = px::hair::make_strands(ldescs, hp);
    px::hair::StrandSet lhmine = lhref;
    for (int i = 0; i < 60; ++i) {
        px::hair::solve_strands(lhref, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 4, 1.0f / 60.0f, h1);
        pxb::b200::solve_strands(dev, lhmine, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 4, 1.0f / 60.0f, h2);
    }
    bad += compare("strands of 20 to 135 particles, 60 frames", lhref.particles, lhmine.particles);

    // --- cloth onto a triangle-mesh floor with a convex-hull rock, both the reference's own
    //     objects (TriangleMesh::from_triangles, build_convex_hull) ---
    std::vector<glm::vec3> fv = {glm::vec3(-2.0f, -2.0f, 0.0f), glm::vec3(2.0f, -2.0f, 0.0f),
                                 glm::vec3(2.0f, 2.0f, 0.0f), glm::vec3(-2.0f, 2.0f, 0.0f),
                                 glm::vec3(0.0f, 0.0f, 0.15f)};
    std::vector<uint32_t> fi = {0, 1, 4, 1, 2, 4, 2, 3, 4, 3, 0, 4};  // a low pyramid
    const px::geometry::TriangleMesh floor = px::geometry::TriangleMesh::from_triangles(fv, fi);
    std::vector<glm::vec3> rock_pts;
    for (int k = 0; k < 8; ++k)
        rock_pts.push_back(glm::vec3(k & 1 ? 0.2f : -0.2f, k & 2 ? 0.12f : -0.12f, k & 4 ? 0.1f : -0.1f));
    rock_pts.push_back(glm::vec3(0.0f, 0.0f, 0.22f));
    px::geometry::ConvexHull rock;
    if (!px::geometry::build_convex_hull(rock_pts.data(), rock_pts.size(), rock)) return 2;
    px::collision::Shape floor_shape = px::collision::Shape::make_mesh(&floor);
    px::collision::Shape rock_shape = px::collision::Shape::make_hull(&rock, 1.2f);
    floor_shape.enabled = rock_shape.enabled = true;
    px::cloth::ClothCollider fc, rc;
    fc.shape = &floor_shape;
    fc.bounds = px::collision::world_bounds(floor_shape, fc.position, fc.orientation);
    rc.shape = &rock_shape;
    rc.position = glm::vec3(0.1f, -0.05f, 0.25f);
    rc.orientation = glm::quat(0.9659258f, 0.0f, 0.0f, 0.2588190f);
    rc.bounds = px::collision::world_bounds(rock_shape, rc.position, rc.orientation);
    const std::vector<px::cloth::ClothCollider> geo_cols = {fc, rc};
    px::cloth::GridClothDesc g2;
    g2.columns = 16;
    g2.rows = 16;
    g2.width = 1.2f;
    g2.height = 1.2f;
    g2.center = glm::vec3(0.0f, 0.0f, 0.8f);
    px::cloth::Cloth gref = px::cloth::make_grid_cloth(g2);
    px::cloth::Cloth gmine = gref;
    for (int i = 0; i < 150; ++i) {
        px::cloth::solve_cloth(gref, geo_cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s1);
        pxb::b200::solve_cloth(dev, gmine, geo_cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s2);
    }
    bad += compare("cloth 16x16 on a mesh floor and a hull, 150 frames", gref.particles, gmine.particles);

    // --- the same sheet onto a heightfield terrain (TriangleMesh::from_height_grid) ---
    std::vector<float> hts(30 * 26);
    for (int j = 0; j < 26; ++j)
        for (int i = 0; i < 30; ++i)
            hts[j * 30 + i] = 0.08f * std::sin(0.4f * static_cast<float>(i)) * std::cos(0.3f * static_cast<float>(j));
    const px::geometry::TriangleMesh terrain = px::geometry::TriangleMesh::from_height_grid(
        std::make_shared<const px::geometry::HeightGrid>(30, 26, glm::vec2(0.07f, 0.07f), hts));
    px::collision::Shape terrain_shape = px::collision::Shape::make_mesh(&terrain);
    terrain_shape.enabled = true;
    px::cloth::ClothCollider tc;
    tc.shape = &terrain_shape;
    tc.position = glm::vec3(-1.0f, -0.9f, 0.0f);
    tc.bounds = px::collision::world_bounds(terrain_shape, tc.position, tc.orientation);
    const std::vector<px::cloth::ClothCollider> terrain_cols = {tc};
    px::cloth::Cloth tref = px::cloth::make_grid_cloth(g2);
    px::cloth::Cloth tmine = tref;
    for (int i = 0; i < 150; ++i) {
        px::cloth::solve_cloth(tref, terrain_cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s1);
        pxb::b200::solve_cloth(dev, tmine, terrain_cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s2);
    }
    bad += compare("cloth 16x16 on a height-grid terrain, 150 frames", tref.particles, tmine.particles);

    // --- a cloth of no grid structure: the 24x24 sheet's lists shuffled and each walked as one
    //     serial batch, its triangles wound the other way, columns cleared (no 1-ring exemption),
    //     self-collision on: the reference's solve_cloth walks any such cloth ---
    px::cloth::GridClothDesc g3;
    g3.columns = 24;
    g3.rows = 24;
    g3.width = 1.15f;
    g3.height = 1.15f;
    g3.center = glm::vec3(0.0f, 0.0f, 1.0f);
    px::cloth::Cloth lref = px::cloth::make_grid_cloth(g3);
    px::cloth::pin_static(lref, glm::vec3(-0.575f, 0.575f, 1.0f), 0.01f);
    px::cloth::pin_static(lref, glm::vec3(0.575f, 0.575f, 1.0f), 0.01f);
    px::cloth::build_tethers(lref);
    uint64_t lcg = 12345u;
    for (std::size_t k = lref.stretch.size(); k > 1; --k) {  // seeded Fisher-Yates
        lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
        std::swap(lref.stretch[k - 1], lref.stretch[(lcg >> 33) % k]);
    }
    lref.stretch_batches = {px::cloth::ConstraintBatch{0, static_cast<uint32_t>(lref.stretch.size())}};
    lref.bend_batches = {px::cloth::ConstraintBatch{0, static_cast<uint32_t>(lref.bend.size())}};
    for (std::size_t t = 0; t + 2 < lref.triangles.size(); t += 3) std::swap(lref.triangles[t + 1], lref.triangles[t + 2]);
    lref.columns = 0;
    lref.rows = 0;
    lref.params.self_collision = true;
    lref.params.self_distance = 0.12f;
    px::cloth::Cloth lmine = lref;
    for (int i = 0; i < 40; ++i) {
        px::cloth::solve_cloth(lref, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s1);
        // the dispatcher overload's signature (cloth_solver.h:158-161); the device ignores it
        pxb::b200::solve_cloth(lmine, cols, glm::vec3(0.0f, 0.0f, -9.81f), 4, 10, 1.0f / 60.0f, s2,
                               [](uint32_t n, auto&& fn) { fn(0u, n); });
    }
    bad += compare("general-topology cloth (shuffled serial lists, self-collision), 40 frames", lref.particles,
                   lmine.particles);
    std::printf(bad ? "facade MISMATCH\n" : "facade ok\n");
    return bad ? 1 : 0;
}
