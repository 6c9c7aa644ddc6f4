// runtime.cu -- host runtime of the C-ABI (include/physxcoopa_b200.h): contexts, the cloth
// registry, the per-step host prologue, launches and read-backs.
//
// The registry mirrors PhysicsWorld's cloth slots (add_cloth / remove_cloth, world.h:552-596):
// generational ids, state resident on the device between steps. A cloth whose constraint lists
// are exactly make_grid_cloth's (cloth_builder.h:81-219) has its colours expressed as affine
// segments over the class-permuted layout described in pxb_internal.h, every segment pair checked
// against the reference lists before upload; any other cloth takes the general layout
// (build_list: the reference's batch walk cut into runs of particle-disjoint items).
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <unordered_map>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/physxcoopa_b200.h"
#include "host_math.h"
#include "pxb_internal.h"
#include "pxb_kernels.h"
#include "runtime_internal.h"

using namespace pxb;

// ------------------------------------------------------------------------------------------
// Context helpers
// ------------------------------------------------------------------------------------------

pxb_status pxb_context::fail(pxb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    error = buf;
    return s;
}

pxb_status pxb_context::cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PXB_OK;
    return fail(e == cudaErrorMemoryAllocation ? PXB_ERR_OUT_OF_MEMORY : PXB_ERR_CUDA,
                "%s: %s", what, cudaGetErrorString(e));
}

pxb_status pxb_context::grow(DevBuf& b, size_t bytes, const char* what) {
    if (b.bytes >= bytes) return PXB_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = std::max<size_t>(bytes, 256);
    want = want + want / 2;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) return cuda(e, what);
    b.bytes = want;
    return PXB_OK;
}

pxb_status pxb_context::grow_pinned(size_t bytes) {
    if (pinned_bytes >= bytes) return PXB_OK;
    if (pinned) {
        cudaEventSynchronize(staged);
        cudaFreeHost(pinned);
    }
    pinned = nullptr;
    pinned_bytes = 0;
    size_t want = bytes + bytes / 2 + 4096;
    cudaError_t e = cudaHostAlloc(&pinned, want, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda(e, "cudaHostAlloc(staging)");
    pinned_bytes = want;
    return PXB_OK;
}

ClothEntry* pxb_context::lookup(uint64_t id) {
    const uint32_t index = static_cast<uint32_t>(id & 0xffffffffu);
    const uint32_t gen = static_cast<uint32_t>(id >> 32);
    if (index >= cloths.size()) return nullptr;
    ClothEntry& e = cloths[index];
    if (!e.alive || e.generation != gen) return nullptr;
    return &e;
}

namespace {

// ------------------------------------------------------------------------------------------
// Grid recognition and colour segments
// ------------------------------------------------------------------------------------------

// Number of k >= 0 with 4k + c + need < cols.
int count_k(int cols, int c, int need) {
    const int top = cols - 1 - c - need;
    return top < 0 ? 0 : top / 4 + 1;
}

// A segment as recognised: `count` live items in rows of `per_row`.
struct HostSeg {
    int count, per_row, a_base, row_stride, d;
};

struct ColourSpec {
    bool bend;
    std::vector<HostSeg> segs;
    int total() const {
        int t = 0;
        for (const HostSeg& s : segs) t += s.count;
        return t;
    }
};

HostSeg seg(int rows_n, int per_row, int a_base, int row_stride, int d) {
    return HostSeg{rows_n * per_row, per_row, a_base, row_stride, d};
}

// Runs of contiguous layout slots covering the real x of a row: classes 0..3 in order, a run
// continuing into the next class while the current class is full (count == Q).
void class_runs(int cols, int Q, std::vector<std::pair<int, int>>& runs) {
    runs.clear();
    int c = 0;
    while (c < 4) {
        const int cnt = count_k(cols, c, 0);
        if (cnt == 0) break;
        int start = c, len = cnt;
        while (c < 3 && count_k(cols, c, 0) == Q && count_k(cols, c + 1, 0) > 0) {
            ++c;
            len += count_k(cols, c, 0);
        }
        runs.push_back({start * Q, len});
        ++c;
    }
}

// The 16 colours of make_grid_cloth in its batch order (cloth_builder.h:128-194), as segments.
void grid_colours(int cols, int rows, bool shear, int Q, int S, std::vector<ColourSpec>& out) {
    out.clear();
    std::vector<std::pair<int, int>> runs;
    class_runs(cols, Q, runs);
    auto H = [&](int p) {
        ColourSpec cs{false, {}};
        for (int c = p; c < 4; c += 2) {
            const int cnt = count_k(cols, c, 1);
            if (cnt > 0) cs.segs.push_back(seg(rows, cnt, c * Q, S, c < 3 ? Q : 1 - 3 * Q));
        }
        return cs;
    };
    auto V = [&](int p, int step, int need, int d, bool bend) {
        ColourSpec cs{bend, {}};
        const int top = rows - 1 - p - need;
        const int nr = top < 0 ? 0 : top / step + 1;
        if (nr > 0)
            for (auto& r : runs) cs.segs.push_back(seg(nr, r.second, p * S + r.first, step * S, d));
        return cs;
    };
    auto D1 = [&](int p) {  // "\" (x,y)-(x+1,y+1)
        ColourSpec cs{false, {}};
        for (int c = p; c < 4; c += 2) {
            const int cnt = count_k(cols, c, 1);
            if (cnt > 0) cs.segs.push_back(seg(rows - 1, cnt, c * Q, S, c < 3 ? S + Q : S + 1 - 3 * Q));
        }
        return cs;
    };
    auto D2 = [&](int p) {  // "/" (x+1,y)-(x,y+1)
        ColourSpec cs{false, {}};
        for (int c = p; c < 4; c += 2) {
            const int cnt = count_k(cols, c, 1);
            if (cnt == 0) continue;
            if (c < 3) cs.segs.push_back(seg(rows - 1, cnt, (c + 1) * Q, S, S - Q));
            else cs.segs.push_back(seg(rows - 1, cnt, 1, S, S + 3 * Q - 1));
        }
        return cs;
    };
    auto BH = [&](int ph) {
        ColourSpec cs{true, {}};
        const int cnt = count_k(cols, ph, 2);
        if (cnt > 0) cs.segs.push_back(seg(rows, cnt, ph * Q, S, ph < 2 ? 2 * Q : 1 - 2 * Q));
        return cs;
    };
    std::vector<ColourSpec> all;
    all.push_back(H(0));
    all.push_back(H(1));
    all.push_back(V(0, 2, 1, S, false));
    all.push_back(V(1, 2, 1, S, false));
    if (shear) {
        all.push_back(D1(0));
        all.push_back(D1(1));
        all.push_back(D2(0));
        all.push_back(D2(1));
    }
    for (int ph = 0; ph < 4; ++ph) all.push_back(BH(ph));
    for (int ph = 0; ph < 4; ++ph) all.push_back(V(ph, 4, 2, 2 * S, true));
    for (auto& cs : all)
        if (cs.total() > 0) out.push_back(std::move(cs));
}

int particle_of_slot(int l, int cols, int rows, int Q, int S) {
    if (l < 0 || l >= rows * S) return -1;
    const int y = l / S;
    const int j = l - y * S;
    const int cls = j / Q;
    const int x = 4 * (j - cls * Q) + cls;
    if (cls > 3 || x >= cols) return -1;
    return y * cols + x;
}

int slot_of_particle(int i, int cols, int Q, int S) {
    const int y = i / cols, x = i - y * cols;
    return y * S + (x & 3) * Q + (x >> 2);
}

// Tries to express the cloth's lists as the grid colours; fills `out` and the slot -> reference
// constraint map (stretch index, or n_stretch + bend index).
bool recognise_grid(const pxb_cloth_desc* d, int Q, int S, std::vector<ColourSpec>& out,
                    std::vector<int32_t>& rest_ref, std::vector<int32_t>& colour_batch) {
    const int cols = static_cast<int>(d->columns), rows = static_cast<int>(d->rows);
    if (d->n_stretch == 0 && d->n_bend == 0 && d->n_stretch_batches == 0 && d->n_bend_batches == 0) {
        // a grid of free particles (every constraint list cleared): no colour to solve
        out.clear();
        rest_ref.clear();
        colour_batch.clear();
        return true;
    }
    for (int shear = 1; shear >= 0; --shear) {
        std::vector<ColourSpec> cs;
        grid_colours(cols, rows, shear != 0, Q, S, cs);
        int n_str = 0, n_bend = 0;
        for (auto& c : cs) (c.bend ? n_bend : n_str)++;
        if (n_str != static_cast<int>(d->n_stretch_batches) || n_bend != static_cast<int>(d->n_bend_batches))
            continue;
        bool ok = true;
        std::vector<int32_t> by_a(d->n_particles, -1);
        std::vector<int32_t> refs;
        std::vector<int32_t> cb;
        int si = 0, bi = 0;
        for (auto& c : cs) {
            const pxb_batch bt = c.bend ? d->bend_batches[bi] : d->stretch_batches[si];
            const pxb_constraint* list = c.bend ? d->bend : d->stretch;
            const uint32_t n_list = c.bend ? d->n_bend : d->n_stretch;
            cb.push_back(c.bend ? bi : si);
            if (c.bend) ++bi; else ++si;
            if (bt.begin > bt.end || bt.end > n_list ||
                static_cast<int>(bt.end - bt.begin) != c.total()) { ok = false; break; }
            for (uint32_t k = bt.begin; k < bt.end; ++k) by_a[list[k].a] = static_cast<int32_t>(k);
            for (const HostSeg& s : c.segs) {
                for (int i = 0; i < s.count && ok; ++i) {
                    const int r = i / s.per_row, k = i - r * s.per_row;
                    const int la = s.a_base + r * s.row_stride + k, lb = la + s.d;
                    const int pa = particle_of_slot(la, cols, rows, Q, S), pb = particle_of_slot(lb, cols, rows, Q, S);
                    if (pa < 0 || pb < 0) { ok = false; break; }
                    const int32_t ref = by_a[pa];
                    if (ref < static_cast<int32_t>(bt.begin) || ref >= static_cast<int32_t>(bt.end) ||
                        list[ref].b != static_cast<uint32_t>(pb)) { ok = false; break; }
                    refs.push_back(c.bend ? static_cast<int32_t>(d->n_stretch) + ref : ref);
                }
            }
            for (uint32_t k = bt.begin; k < bt.end; ++k) by_a[list[k].a] = -1;
            if (!ok) break;
        }
        if (!ok) continue;
        out = std::move(cs);
        rest_ref = std::move(refs);
        colour_batch = std::move(cb);
        return true;
    }
    return false;
}

bool grid_triangles(const pxb_cloth_desc* d) {
    const uint32_t cols = d->columns, rows = d->rows;
    if (d->n_triangle_indices != (cols - 1) * (rows - 1) * 6) return false;
    size_t t = 0;
    for (uint32_t y = 0; y + 1 < rows; ++y) {
        for (uint32_t x = 0; x + 1 < cols; ++x) {
            const uint32_t i00 = y * cols + x, i10 = i00 + 1, i01 = i00 + cols, i11 = i01 + 1;
            const uint32_t want[6] = {i00, i10, i11, i00, i11, i01};
            for (int k = 0; k < 6; ++k)
                if (d->triangles[t++] != want[k]) return false;
        }
    }
    return true;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Whether solve_cloth runs its self-collision stage for this cloth (cloth_solver.h:170).
bool self_on(const ClothEntry& e) {
    return e.params.self_collision && e.params.self_distance > PXB_EPSILON;
}

// Compliance of colour `c` of entry `e` (per-batch override, else the params value).
float colour_compliance(const ClothEntry& e, int c) {
    const bool bend = e.colour_is_bend[c] != 0;
    const int b = e.colour_batch[c];
    if (bend) return e.bend_batch_comp.empty() ? e.params.bend_compliance : e.bend_batch_comp[b];
    return e.stretch_batch_comp.empty() ? e.params.stretch_compliance : e.stretch_batch_comp[b];
}


// CTAs of the cloth kernel one SM holds at once: 228 KB of shared memory (1 KB of it reserved
// per CTA), 2048 threads, 64 K registers, 32 CTAs.
int ctas_per_sm(int smem_bytes, int threads, int regs) {
    const int warps = (threads + 31) / 32;
    const int by_smem = 233472 / (smem_bytes + kClothStaticSmem + 1024);
    const int by_threads = 64 / std::max(warps, 1);
    const int by_regs = 65536 / std::max(warps * 32 * ((regs + 7) & ~7), 1);
    return std::max(1, std::min(std::min(by_smem, by_threads), std::min(by_regs, 32)));
}

// Restricts the recognised colours to the rows of each of `n_ranks` CTAs and builds the device
// segments (power-of-two rows). `refs` lists, in the colours' enumeration order, the reference
// constraint of every item. Fills e.ranks / e.segs / e.n_rest_total and the padded slot map.
bool build_ranks(ClothEntry& e, const std::vector<ColourSpec>& cs, const std::vector<int32_t>& refs,
                 int n_ranks, std::vector<int32_t>& padded_ref, int& max_colour_items) {
    const int S = e.S;
    const int R = (e.rows + n_ranks - 1) / n_ranks;
    e.ranks.assign(n_ranks, ClothEntry::Rank{});
    e.segs.clear();
    padded_ref.clear();
    std::vector<std::vector<size_t>> seg_ref_off(cs.size());
    size_t off = 0;
    for (size_t c = 0; c < cs.size(); ++c)
        for (const HostSeg& h : cs[c].segs) {
            seg_ref_off[c].push_back(off);
            off += static_cast<size_t>(h.count);
        }
    int rest_total = 0;
    max_colour_items = 0;
    for (int r = 0; r < n_ranks; ++r) {
        ClothEntry::Rank& rk = e.ranks[r];
        rk.row0 = r * R;
        rk.n_rows = std::min(e.rows, (r + 1) * R) - rk.row0;
        if (n_ranks > 1 && rk.n_rows < 2) return false;  // a bend reaches two rows ahead
        rk.seg_begin = static_cast<int>(e.segs.size());
        rk.colour_seg.assign(e.n_colours + 1, 0);
        rk.rest_off = rest_total;
        int rest = 0;
        const int Y0 = rk.row0, Y1 = rk.row0 + rk.n_rows;
        for (int c = 0; c < e.n_colours; ++c) {
            rk.colour_seg[c] = static_cast<int>(e.segs.size()) - rk.seg_begin;
            int items = 0;
            for (size_t hi = 0; hi < cs[c].segs.size(); ++hi) {
                const HostSeg& h = cs[c].segs[hi];
                const int nrows = h.count / h.per_row;
                const int y0 = h.a_base / S, step = h.row_stride / S;
                const int r_lo = Y0 <= y0 ? 0 : (Y0 - y0 + step - 1) / step;
                const int r_hi = Y1 <= y0 ? 0 : std::min(nrows, (Y1 - y0 + step - 1) / step);
                if (r_hi <= r_lo) continue;
                PxbSeg g{};
                g.count = (r_hi - r_lo) * h.per_row;
                g.magic = h.per_row > 1 ? static_cast<uint32_t>(((1ull << 32) + h.per_row - 1) / h.per_row) : 0u;
                g.per_row = h.per_row;
                // the device's row of item i is umulhi(i, magic): check it for every item
                for (int i = 0; i < g.count; ++i) {
                    const int row = g.magic ? static_cast<int>((static_cast<uint64_t>(i) * g.magic) >> 32) : i;
                    if (row != i / h.per_row) return false;
                }
                g.a_base = h.a_base + r_lo * h.row_stride - Y0 * S;
                g.row_stride = h.row_stride;
                g.d = h.d;
                g.rest_base = rest;
                g.lam_base = -1;
                for (int i = 0; i < g.count; ++i)
                    padded_ref.push_back(refs[seg_ref_off[c][hi] + static_cast<size_t>(r_lo) * h.per_row + i]);
                rest += g.count;
                items += g.count;
                e.segs.push_back(g);
            }
            max_colour_items = std::max(max_colour_items, items);
        }
        rk.colour_seg[e.n_colours] = static_cast<int>(e.segs.size()) - rk.seg_begin;
        if (rk.colour_seg[e.n_colours] > PXB_MAX_SEGS) return false;
        rk.n_rest_pad = (rest + 3) & ~3;
        for (int i = rest; i < rk.n_rest_pad; ++i) padded_ref.push_back(-1);
        rest_total += rk.n_rest_pad;
    }
    e.n_rest_total = rest_total;
    return true;
}

// Every live item of every rank: `a` in this rank's rows, `b` in them or the next rank's, and
// the pair is the reference constraint its rest slot says.
bool verify_ranks(const ClothEntry& e, const pxb_cloth_desc* d) {
    const int n_ranks = static_cast<int>(e.ranks.size());
    std::vector<uint8_t> seen(static_cast<size_t>(d->n_stretch) + d->n_bend, 0);
    for (int r = 0; r < n_ranks; ++r) {
        const ClothEntry::Rank& rk = e.ranks[r];
        const int n_local = rk.n_rows * e.S;
        const int n_next = r + 1 < n_ranks ? e.ranks[r + 1].n_rows * e.S : 0;
        const int base = rk.row0 * e.S;
        for (int sg = rk.seg_begin; sg < rk.seg_begin + rk.colour_seg[e.n_colours]; ++sg) {
            const PxbSeg& g = e.segs[sg];
            for (int i = 0; i < g.count; ++i) {
                const int32_t ref = e.rest_ref[rk.rest_off + g.rest_base + i];
                const int row = i / g.per_row, k = i - row * g.per_row;
                const int la = g.a_base + row * g.row_stride + k, lb = la + g.d;
                if (la < 0 || la >= n_local || lb < 0 || lb >= n_local + n_next || ref < 0) return false;
                const pxb_constraint& kc = ref < static_cast<int32_t>(d->n_stretch) ? d->stretch[ref]
                                                                                    : d->bend[ref - d->n_stretch];
                if (particle_of_slot(base + la, e.cols, e.rows, e.Q, e.S) != static_cast<int>(kc.a) ||
                    particle_of_slot(base + lb, e.cols, e.rows, e.Q, e.S) != static_cast<int>(kc.b))
                    return false;
                if (seen[ref]++) return false;  // solved twice
            }
        }
    }
    for (uint8_t v : seen)
        if (!v) return false;  // never solved
    return true;
}

// Compliance of batch `b` of the stretch (bend = false) or bend list: the per-batch override,
// else the params value.
float batch_compliance(const ClothEntry& e, bool bend, int b) {
    if (bend) return e.bend_batch_comp.empty() ? e.params.bend_compliance : e.bend_batch_comp[b];
    return e.stretch_batch_comp.empty() ? e.params.stretch_compliance : e.stretch_batch_comp[b];
}

// General topology: any constraint lists, solved as solve_cloth walks them (cloth_solver.h:
// 256-271: every stretch batch, then every bend batch, each in list order; a constraint in no
// batch is never solved). The walk is cut into runs of consecutive items that share no
// particle: inside a run the serial order cannot change a result, so the device projects a
// run's items in parallel and the outcome is the serial walk's. A run may continue into the
// next batch of the same list when both batches have the same compliance. The particles form
// one row of n (slot of particle i = (i % 4) * Q + i / 4), so every per-particle path of the
// grid layout applies unchanged.
pxb_status build_list(const pxb_cloth_desc* d, ClothEntry& e, std::string& why) {
    static_assert(kListMaxSlots % 4 == 0, "slots are whole groups of four");
    const uint32_t n = d->n_particles;
    e.list = true;
    e.cols = static_cast<int>(n);
    e.rows = 1;
    e.Q = (e.cols + 3) / 4;
    e.S = 4 * e.Q;
    e.n_layout = e.S;
    e.n_particles = n;
    if (e.n_layout > kListMaxSlots) {
        why = "a general-topology cloth holds at most 16777212 particles";
        return PXB_ERR_TOO_LARGE;
    }
    e.runs.clear();
    e.run_batch.clear();
    e.item_ends.clear();
    e.rest_ref.clear();
    std::vector<uint32_t> stamp(n, 0);  // run id that last took the particle
    std::vector<uint8_t> seen(static_cast<size_t>(d->n_stretch) + d->n_bend, 0);
    uint32_t run_id = 0;
    int max_run = 0;
    char buf[256];
    for (int bend = 0; bend < 2; ++bend) {
        const uint32_t nb = bend ? d->n_bend_batches : d->n_stretch_batches;
        const pxb_batch* bb = bend ? d->bend_batches : d->stretch_batches;
        const pxb_constraint* list = bend ? d->bend : d->stretch;
        const uint32_t n_list = bend ? d->n_bend : d->n_stretch;
        const float* comp = bend ? d->bend_batch_compliance : d->stretch_batch_compliance;
        bool open = false;
        for (uint32_t b = 0; b < nb; ++b) {
            if (bb[b].begin > bb[b].end || bb[b].end > n_list) {
                snprintf(buf, sizeof(buf), "%s batch %u indexes past its list", bend ? "bend" : "stretch", b);
                why = buf;
                return PXB_ERR_UNSUPPORTED;
            }
            if (b > 0 && comp && std::memcmp(&comp[b], &comp[b - 1], 4) != 0) open = false;
            for (uint32_t k = bb[b].begin; k < bb[b].end; ++k) {
                const pxb_constraint& c = list[k];
                const int32_t ref = bend ? static_cast<int32_t>(d->n_stretch + k) : static_cast<int32_t>(k);
                if (seen[ref]++) {
                    snprintf(buf, sizeof(buf), "%s constraint %u is in more than one batch", bend ? "bend" : "stretch", k);
                    why = buf;
                    return PXB_ERR_UNSUPPORTED;
                }
                if (!open || stamp[c.a] == run_id || stamp[c.b] == run_id) {
                    ++run_id;
                    e.runs.push_back(PxbRun{0, static_cast<int32_t>(e.item_ends.size()), -1, 0.0f});
                    e.run_batch.push_back(make_int2(bend, static_cast<int>(b)));
                    open = true;
                }
                stamp[c.a] = stamp[c.b] = run_id;
                const uint32_t la = static_cast<uint32_t>(slot_of_particle(static_cast<int>(c.a), e.cols, e.Q, e.S));
                const uint32_t lb = static_cast<uint32_t>(slot_of_particle(static_cast<int>(c.b), e.cols, e.Q, e.S));
                e.item_ends.push_back(la | static_cast<uint64_t>(lb) << 32);
                e.rest_ref.push_back(ref);
                max_run = std::max(max_run, ++e.runs.back().count);
            }
        }
    }
    // Inside a run the items may be listed in any order (they share no particle). A warp's float4
    // access to shared memory is served 8 lanes at a time, without bank conflict when those 8
    // slots differ mod 8: order each run so that every aligned group of 8 items has distinct `a`
    // residues and distinct `b` residues where the run allows it. Items are bucketed by (a mod 8,
    // b mod 8); each group is a maximum matching of a residues to b residues over the non-empty
    // buckets (augmenting paths, fullest buckets first), topped up from the fullest buckets.
    for (const PxbRun& run : e.runs) {
        std::vector<std::vector<int>> bucket(64);
        for (int i = run.count - 1; i >= 0; --i) {
            const uint64_t w = e.item_ends[run.item_base + i];
            bucket[(w & 7u) * 8 + ((w >> 32) & 7u)].push_back(i);  // popped from the back: list order
        }
        auto fuller = [&](int x, int y) { return bucket[x].size() > bucket[y].size(); };
        int match_b[8];
        std::function<bool(int, uint32_t&)> augment = [&](int ra, uint32_t& seen) -> bool {
            int cand[8], nc = 0;
            for (int rb = 0; rb < 8; ++rb)
                if (!bucket[ra * 8 + rb].empty()) cand[nc++] = ra * 8 + rb;
            std::stable_sort(cand, cand + nc, fuller);
            for (int q = 0; q < nc; ++q) {
                const int rb = cand[q] & 7;
                if (seen >> rb & 1u) continue;
                seen |= 1u << rb;
                if (match_b[rb] < 0 || augment(match_b[rb], seen)) {
                    match_b[rb] = ra;
                    return true;
                }
            }
            return false;
        };
        std::vector<int> order;
        order.reserve(run.count);
        int left = run.count;
        while (left > 0) {
            std::fill(match_b, match_b + 8, -1);
            int ras[8], options[8];
            for (int ra = 0; ra < 8; ++ra) {
                ras[ra] = ra;
                options[ra] = 0;
                for (int rb = 0; rb < 8; ++rb) options[ra] += bucket[ra * 8 + rb].empty() ? 0 : 1;
            }
            std::stable_sort(ras, ras + 8, [&](int x, int y) { return options[x] < options[y]; });
            for (int q = 0; q < 8; ++q) {
                uint32_t seen = 0;
                augment(ras[q], seen);
            }
            int taken = 0;
            for (int rb = 0; rb < 8; ++rb)
                if (match_b[rb] >= 0) {
                    std::vector<int>& bk = bucket[match_b[rb] * 8 + rb];
                    order.push_back(bk.back());
                    bk.pop_back();
                    ++taken;
                }
            int by_size[64];
            for (int k = 0; k < 64; ++k) by_size[k] = k;
            std::stable_sort(by_size, by_size + 64, fuller);
            for (int q = 0; q < 64 && taken < 8; ++q)
                while (taken < 8 && !bucket[by_size[q]].empty()) {
                    order.push_back(bucket[by_size[q]].back());
                    bucket[by_size[q]].pop_back();
                    ++taken;
                }
            left -= taken;
        }
        std::vector<uint64_t> ends(run.count);
        std::vector<int32_t> refs(run.count);
        for (int i = 0; i < run.count; ++i) {
            ends[i] = e.item_ends[run.item_base + order[i]];
            refs[i] = e.rest_ref[run.item_base + order[i]];
        }
        std::copy(ends.begin(), ends.end(), e.item_ends.begin() + run.item_base);
        std::copy(refs.begin(), refs.end(), e.rest_ref.begin() + run.item_base);
    }
    const int items = static_cast<int>(e.item_ends.size());
    e.list_items_pad = (items + 3) & ~3;
    e.item_ends.resize(e.list_items_pad, 0u);
    e.rest_ref.resize(e.list_items_pad, -1);
    // endpoints after the rest lengths: one word per item (a | b << 16), or two (a, b) for a cloth
    // of more than 65535 slots
    e.n_rest_total = (list_wide(e) ? 3 : 2) * e.list_items_pad;
    e.n_colours = 0;
    e.segs.clear();
    e.colour_is_bend.clear();
    e.colour_batch.clear();
    e.cross_mask = 0;
    e.ranks.assign(1, ClothEntry::Rank{});
    ClothEntry::Rank& rk = e.ranks[0];
    rk.n_rows = 1;
    rk.colour_seg.assign(1, 0);
    rk.n_rest_pad = e.n_rest_total;
    // the triangle index: per slot, its triangles' corner slots in ascending triangle order
    // (a triangle naming a particle twice is listed twice, as the reference adds its share twice)
    const uint32_t nt = d->n_triangle_indices / 3;  // cloth_solver.h:204 reads whole triples
    e.tri_off.assign(e.n_layout + 1, 0);
    for (uint32_t t = 0; t < 3 * nt; ++t)
        ++e.tri_off[slot_of_particle(static_cast<int>(d->triangles[t]), e.cols, e.Q, e.S) + 1];
    for (int l = 0; l < e.n_layout; ++l) e.tri_off[l + 1] += e.tri_off[l];
    e.tri_ent.assign(3 * nt, make_int4(0, 0, 0, 0));
    {
        std::vector<int32_t> fill(e.tri_off.begin(), e.tri_off.end() - 1);
        for (uint32_t t = 0; t < nt; ++t) {
            int s[3];
            for (int q = 0; q < 3; ++q) s[q] = slot_of_particle(static_cast<int>(d->triangles[3 * t + q]), e.cols, e.Q, e.S);
            for (int q = 0; q < 3; ++q) e.tri_ent[fill[s[q]]++] = make_int4(s[0], s[1], s[2], static_cast<int>(t));
        }
    }
    e.threads = std::max(64, (max_run + 31) & ~31);  // one item per thread; fitted to the SM in plan_cloth
    return PXB_OK;
}
}  // namespace

// Whether umulhi(j, ceil(2^32 / cols)) == j / cols for every j < n (the device's row of index j).
static bool rows_by_multiply_high(uint32_t cols, uint32_t n) {
    if (cols == 0) return true;
    const uint64_t magic = ((1ull << 32) + cols - 1) / cols;
    for (uint64_t j = 0; j < n; ++j)
        if (((j * magic) >> 32) != j / cols) return false;
    return true;
}

// Self-collision tables of a one-CTA cloth (the spatial hash's bucket ends, sorted indices and
// scan scratch): in the rest-length region when they fit there (restaged after the stage), else
// after the `smem` bytes the step already uses.
static void place_self_tables(ClothEntry& e, int smem, int pos_bytes, int rest_bytes) {
    uint32_t buckets = 16;  // detail::hash_bucket_count (cloth_solver.h:111-115)
    while (buckets < e.n_particles * 2u && buckets < (1u << 22)) buckets <<= 1;
    const int bytes = (4 * static_cast<int>(PXB_SELF_WORDS(buckets, e.n_particles)) + 15) & ~15;
    e.dev.self_buckets = static_cast<int32_t>(buckets);
    if (bytes <= rest_bytes) {
        e.dev.self_hash_off = pos_bytes;
        e.dev.self_restage = 1;
        e.self_smem = smem;
    } else {
        e.dev.self_hash_off = smem;
        e.self_smem = smem + bytes;
    }
    e.self_ok = rows_by_multiply_high(static_cast<uint32_t>(e.cols), e.n_particles) &&
                rows_by_multiply_high(static_cast<uint32_t>(e.ref_columns), e.n_particles) &&
                e.self_smem <= kMaxDynamicSmem;
}

// Re-derives everything that depends on params: lambda slots, union regions, shared memory.
static void layout_ranks(ClothEntry& e) {
    const bool aero = (e.params.air_drag > 0.0f || e.params.air_lift > 0.0f) && e.n_triangle_indices > 0;
    if (e.list) {
        // one CTA: positions | rest lengths + packed endpoints | lambdas or parked velocities
        int lam = 0;
        for (size_t r = 0; r < e.runs.size(); ++r) {
            const float comp = batch_compliance(e, e.run_batch[r].x != 0, e.run_batch[r].y);
            e.runs[r].compliance = comp;
            const bool has_lam = comp != 0.0f || std::signbit(comp);  // exactly +0: no lambdas
            e.runs[r].lam_base = has_lam ? lam : -1;
            if (has_lam) lam += e.runs[r].count;
        }
        ClothEntry::Rank& rk = e.ranks[0];
        rk.n_lam = lam;
        rk.lam_off = 0;
        const int u_floats = std::max(lam, aero ? 3 * e.n_layout : 0);
        rk.smem = e.list_gmem ? 0 : 16 * e.n_layout + 4 * rk.n_rest_pad + 4 * ((u_floats + 3) & ~3);
        PxbRank& dr = e.dev.rank[0];
        std::memset(&dr, 0, sizeof(dr));
        dr.n_rows = 1;
        dr.n_rest_pad = rk.n_rest_pad;
        dr.n_lam = lam;
        dr.smem_bytes = rk.smem;
        e.n_lam = lam;
        e.dev.smem_bytes = rk.smem;
        e.warm_smem = rk.smem;
        e.self_ok = false;
        e.self_smem = 0;
        e.dev.self_buckets = 0;
        e.dev.self_hash_off = 0;
        e.dev.self_restage = 0;
        if (!e.list_gmem) place_self_tables(e, rk.smem, 16 * e.n_layout, 4 * rk.n_rest_pad);
        return;
    }
    int lam_total = 0, smem_max = 0, warm_max = 0;
    for (size_t r = 0; r < e.ranks.size(); ++r) {
        ClothEntry::Rank& rk = e.ranks[r];
        int lam = 0;
        for (int c = 0; c < e.n_colours; ++c) {
            // a colour without lambdas must have a compliance of exactly +0 (the kernel then
            // takes -c - alpha * lambda as -c); -0 keeps its lambdas like any other value
            const bool has_lam = colour_compliance(e, c) != 0.0f || std::signbit(colour_compliance(e, c));
            for (int sg = rk.seg_begin + rk.colour_seg[c]; sg < rk.seg_begin + rk.colour_seg[c + 1]; ++sg) {
                e.segs[sg].lam_base = has_lam ? lam : -1;
                if (has_lam) lam += e.segs[sg].count;
            }
        }
        rk.n_lam = lam;
        rk.lam_off = lam_total;
        lam_total += lam;
        const int n_local = rk.n_rows * e.S;
        const int u_floats = std::max(lam, (aero && e.aero_grid) ? 3 * n_local : 0);
        if (e.lean && e.soa) {
            // positions as arrays plus the inverse-mass index and table; the warm start's network
            // borrows all of shared memory while the positions wait in HBM
            rk.smem = (pxb::soa_smem_bytes(n_local) + 15) & ~15;
            warm_max = std::max(warm_max, std::max(rk.smem, std::min(kMaxDynamicSmem, kWarmTileOff + kWarmGroups * kWarmTileBytes)));
        } else if (e.lean) {
            // positions only; the warm start's network tiles go right after them, as many of its
            // warpgroups' tiles as fit (at least one)
            rk.smem = 16 * n_local;
            const int tiles = std::min(kMaxDynamicSmem, 16 * n_local + kWarmTileOff + kWarmGroups * kWarmTileBytes);
            warm_max = std::max(warm_max, std::max(16 * n_local + kWarmUMin, tiles));
        } else {
            rk.smem = 16 * n_local + 4 * rk.n_rest_pad + 4 * ((u_floats + 3) & ~3);
            warm_max = std::max(warm_max, 16 * n_local + 4 * rk.n_rest_pad + std::max(4 * ((u_floats + 3) & ~3), kWarmUMin));
        }
        smem_max = std::max(smem_max, rk.smem);
        PxbRank& dr = e.dev.rank[r];
        dr.row0 = rk.row0;
        dr.n_rows = rk.n_rows;
        dr.seg_begin = rk.seg_begin;
        for (int c = 0; c <= e.n_colours; ++c) dr.colour_seg[c] = rk.colour_seg[c];
        dr.rest_off = rk.rest_off;
        dr.n_rest_pad = rk.n_rest_pad;
        dr.lam_off = rk.lam_off;
        dr.n_lam = rk.n_lam;
        dr.smem_bytes = rk.smem;
    }
    e.n_lam = lam_total;
    e.dev.smem_bytes = smem_max;
    e.warm_smem = warm_max;
    // Self-collision tables (one-CTA cloths): in the rest-length region when they fit there (the
    // rest lengths are staged again after the stage), else after the lambda region.
    e.self_ok = false;
    e.self_smem = 0;
    e.dev.self_buckets = 0;
    e.dev.self_hash_off = 0;
    e.dev.self_restage = 0;
    if (e.ranks.size() == 1 && !e.soa) {  // a cloth held as arrays has no room for the tables
        const ClothEntry::Rank& rk = e.ranks[0];
        place_self_tables(e, smem_max, 16 * rk.n_rows * e.S, e.lean ? 0 : 4 * rk.n_rest_pad);
    }
}

void pxb_context::refresh_layout(ClothEntry& e) {
    layout_ranks(e);
    registry_dirty = true;
    ++registry_epoch;
}

pxb_status pxb_context::upload_segments(ClothEntry& e) {
    if (e.list)
        return e.runs.empty() ? PXB_OK
                              : cuda(cudaMemcpyAsync(const_cast<PxbRun*>(e.dev.runs), e.runs.data(),
                                                     sizeof(PxbRun) * e.runs.size(), cudaMemcpyHostToDevice, stream),
                                     "upload runs");
    return cuda(cudaMemcpyAsync(const_cast<PxbSeg*>(e.dev.segs), e.segs.data(),
                                sizeof(PxbSeg) * e.segs.size(), cudaMemcpyHostToDevice, stream),
                "upload segments");
}

pxb_status pxb_context::upload_particles(ClothEntry& e, const pxb_particle* particles) {
    const int n = static_cast<int>(e.n_particles);
    std::vector<float4> pos(e.n_layout, make_float4(0, 0, 0, 0)), vel(e.n_layout, make_float4(0, 0, 0, 0)),
        prv(e.n_layout, make_float4(0, 0, 0, 0));
    for (int i = 0; i < n; ++i) {
        const int l = slot_of_particle(i, e.cols, e.Q, e.S);
        const pxb_particle& p = particles[i];
        pos[l] = make_float4(p.position[0], p.position[1], p.position[2], p.inv_mass);
        vel[l] = make_float4(p.velocity[0], p.velocity[1], p.velocity[2], 1.0f);
        prv[l] = make_float4(p.prev_position[0], p.prev_position[1], p.prev_position[2], 0.0f);
    }
    // Tether anchors must be pinned for the per-particle tether stage to equal the reference's
    // list-order pass (cloth_solver.h:274-275 relies on the same fact).
    for (const pxb_tether& t : e.tethers) {
        if (particles[t.anchor].inv_mass != 0.0f && particles[t.particle].inv_mass != 0.0f)
            return fail(PXB_ERR_UNSUPPORTED, "tether %u anchors to an unpinned particle %u", t.particle,
                        t.anchor);
    }
    if (e.soa) {
        // the table of distinct inverse masses (ascending bit patterns) the kernel indexes; with
        // more than the table holds, the kernel reads them in place from the positions in HBM
        std::vector<uint32_t> bits;
        bits.reserve(static_cast<size_t>(n) + 1);
        for (int l = 0; l < e.n_layout; ++l) {
            uint32_t b;
            std::memcpy(&b, &pos[l].w, 4);
            bits.push_back(b);
        }
        std::sort(bits.begin(), bits.end());
        bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
        const int n_wtab = bits.size() <= static_cast<size_t>(PXB_MAX_WTAB) ? static_cast<int>(bits.size()) : 0;
        if (n_wtab) {
            pxb_status s = cuda(cudaMemcpyAsync(const_cast<float*>(e.dev.wtab), bits.data(), 4 * bits.size(),
                                                cudaMemcpyHostToDevice, stream),
                                "upload inverse-mass table");
            if (s) return s;
        }
        if (n_wtab != e.dev.n_wtab) {
            e.dev.n_wtab = n_wtab;
            registry_dirty = true;
            ++registry_epoch;
        }
    }
    const size_t bytes = 16 * static_cast<size_t>(e.n_layout);
    pxb_status s = cuda(cudaMemcpyAsync(e.dev.pos, pos.data(), bytes, cudaMemcpyHostToDevice, stream), "upload pos");
    if (s) return s;
    s = cuda(cudaMemcpyAsync(e.dev.vel, vel.data(), bytes, cudaMemcpyHostToDevice, stream), "upload vel");
    if (s) return s;
    s = cuda(cudaMemcpyAsync(e.dev.prv, prv.data(), bytes, cudaMemcpyHostToDevice, stream), "upload prv");
    if (s) return s;
    return cuda(cudaStreamSynchronize(stream), "upload particles");
}

pxb_status pxb_context::upload_anchor_records(ClothEntry& e) {
    if (e.anchor_recs.empty()) return PXB_OK;
    pxb_status s = cuda(cudaMemcpyAsync(e.dev.anchors, e.anchor_recs.data(),
                                        sizeof(PxbAnchorRec) * e.anchor_recs.size(),
                                        cudaMemcpyHostToDevice, stream),
                        "upload anchors");
    if (s) return s;
    return cuda(cudaStreamSynchronize(stream), "upload anchors");
}

// Everything add_cloth decides before touching the device: validation, grid recognition, the
// cluster size, per-rank colour segments (verified item by item against the constraint lists)
// and the shared-memory layout. Needs no context, so the layout can be planned on any host.
// soa_layouts: the float-array lean layout may be chosen (pxb_context_set_lean_arrays).
// Barriers of a one-CTA grid cloth's colour loop: the reference projects colour after colour, so
// each colour waits for the one before. Where two consecutive colours touch disjoint particles
// (the bend colours of phases 0 and 1, or 2 and 3, along a row or a column), projecting them
// together gives the same result as one after the other: they form one phase, with no barrier
// between them. A phase grows while its next colour is disjoint from every colour in it. Bit c of
// the mask: a barrier after colour c. Clusters and the whole-GPU path keep every barrier.
static uint32_t colour_sync_mask(const ClothEntry& e) {
    uint32_t mask = 0xffffffffu;
    if (e.ranks.size() != 1 || e.grid || e.list || e.n_colours < 2) return mask;
    const ClothEntry::Rank& rk = e.ranks[0];
    const int n_slots = rk.n_rows * e.S;
    std::vector<uint8_t> phase(static_cast<size_t>(n_slots), 0);  // slot -> phase id + 1 (mod 255)
    int pid = 1;
    auto touch = [&](int c, bool mark, bool& clash) {
        for (int sg = rk.seg_begin + rk.colour_seg[c]; sg < rk.seg_begin + rk.colour_seg[c + 1]; ++sg) {
            const PxbSeg& g = e.segs[sg];
            for (int i = 0; i < g.count; ++i) {
                const int row = i / g.per_row;
                const int la = g.a_base + row * g.row_stride + (i - row * g.per_row), lb = la + g.d;
                for (int l : {la, lb}) {
                    if (l < 0 || l >= n_slots) { clash = true; continue; }
                    if (mark) phase[l] = static_cast<uint8_t>(pid);
                    else if (phase[l] == pid) clash = true;
                }
            }
        }
    };
    bool dummy = false;
    touch(0, true, dummy);
    for (int c = 1; c < e.n_colours; ++c) {
        bool clash = false;
        touch(c, false, clash);
        if (clash) {
            pid = pid % 255 + 1;  // a new phase: stale marks of an old id are ignored below
            if (pid == 1) std::fill(phase.begin(), phase.end(), 0);
        } else {
            mask &= ~(1u << (c - 1));  // colour c joins colour c - 1's phase
        }
        touch(c, true, dummy);
    }
    return mask;
}

// lean_mid: a sheet held whole whose shared memory lets an SM hold only one of its CTAs takes the
// lean layout instead where that lets an SM hold two or more (pxb_context_set_lean_mid).
static pxb_status plan_cloth(const pxb_cloth_desc* d, ClothEntry& e, std::string& err, bool soa_layouts = true,
                             bool lean_mid = true) {
    char buf[512];
    auto fail = [&](pxb_status st, const char* fmt, auto... args) {
        snprintf(buf, sizeof(buf), fmt, args...);
        err = buf;
        return st;
    };
    if (!d) return fail(PXB_ERR_INVALID_ARGUMENT, "null argument");
    if (d->n_particles == 0 || !d->particles)
        return fail(PXB_ERR_INVALID_ARGUMENT, "an empty cloth is refused (PhysicsWorld::add_cloth does the same)");
    const uint32_t n = d->n_particles;
    auto chk_list = [&](const pxb_constraint* l, uint32_t cnt, const char* name) -> bool {
        if (cnt && !l) return false;
        for (uint32_t k = 0; k < cnt; ++k)
            if (l[k].a >= n || l[k].b >= n) {
                fail(PXB_ERR_INVALID_ARGUMENT, "%s[%u] indexes past the particles", name, k);
                return false;
            }
        return true;
    };
    if (!chk_list(d->stretch, d->n_stretch, "stretch") || !chk_list(d->bend, d->n_bend, "bend"))
        return PXB_ERR_INVALID_ARGUMENT;
    if ((d->n_stretch_batches && !d->stretch_batches) || (d->n_bend_batches && !d->bend_batches) ||
        (d->n_tethers && !d->tethers) || (d->n_anchors && !d->anchors) ||
        (d->n_triangle_indices && !d->triangles))
        return fail(PXB_ERR_INVALID_ARGUMENT, "null array with a nonzero count");
    for (uint32_t k = 0; k < d->n_tethers; ++k)
        if (d->tethers[k].particle >= n || d->tethers[k].anchor >= n)
            return fail(PXB_ERR_INVALID_ARGUMENT, "tether %u indexes past the particles", k);
    for (uint32_t k = 0; k < d->n_triangle_indices; ++k)
        if (d->triangles[k] >= n) return fail(PXB_ERR_INVALID_ARGUMENT, "triangle index past the particles");
    // --- what every layout keeps ---
    e.n_particles = n;
    e.n_stretch = d->n_stretch;
    e.n_bend = d->n_bend;
    e.n_stretch_batches = d->n_stretch_batches;
    e.n_bend_batches = d->n_bend_batches;
    if (d->stretch_batch_compliance)
        e.stretch_batch_comp.assign(d->stretch_batch_compliance, d->stretch_batch_compliance + d->n_stretch_batches);
    if (d->bend_batch_compliance)
        e.bend_batch_comp.assign(d->bend_batch_compliance, d->bend_batch_compliance + d->n_bend_batches);
    e.params = d->params;
    e.n_triangle_indices = d->n_triangle_indices;
    // i % columns and i / columns for i < n are the same for every columns >= n
    e.ref_columns = static_cast<int>(std::min<uint32_t>(d->columns, n));
    e.time = d->time;
    e.tethers.assign(d->tethers, d->tethers + d->n_tethers);
    {
        std::vector<int> per(n, 0);
        for (const pxb_tether& t : e.tethers)
            if (++per[t.particle] > 1)
                return fail(PXB_ERR_UNSUPPORTED, "particle %u has more than one tether", t.particle);
    }

    // --- grid recognition: make_grid_cloth's lists and triangles, else the general layout ---
    std::vector<ColourSpec> cs;
    std::vector<int32_t> rest_ref, colour_batch;
    bool is_grid = d->n_stretch_batches <= PXB_MAX_COLOURS && d->n_bend_batches <= PXB_MAX_COLOURS &&
                   d->columns >= 2 && d->rows >= 2 && static_cast<uint64_t>(d->columns) * d->rows == n;
    if (is_grid) {
        e.cols = static_cast<int>(d->columns);
        e.rows = static_cast<int>(d->rows);
        e.Q = (e.cols + 3) / 4;
        e.S = 4 * e.Q;
        e.n_layout = e.rows * e.S;
        is_grid = recognise_grid(d, e.Q, e.S, cs, rest_ref, colour_batch) &&
                  (d->n_triangle_indices == 0 || grid_triangles(d));
    }
    if (!is_grid) {
        std::string why;
        if (pxb_status st = build_list(d, e, why)) return fail(st, "%s", why.c_str());
        e.aero_grid = 0;
        layout_ranks(e);
        if (e.dev.smem_bytes > kMaxDynamicSmem) {
            // beyond one CTA's shared memory: the same walk with the state left in HBM (L2-resident
            // while its CTA runs), one thread per item of the longest run
            e.list_gmem = true;
            layout_ranks(e);
            e.threads = std::min(e.threads, kClothMaxThreads);
            return PXB_OK;
        }
        // the CTAs shared memory lets an SM hold share the 1024 threads the 64-register kernel
        // variant fits in the register file; within that, one thread per item of the longest run
        const int per_sm = std::max(1, 233472 / (e.dev.smem_bytes + kClothStaticSmem + 1024));
        e.threads = std::min(e.threads, std::max(64, (kClothMaxThreads / per_sm) & ~31));
        return PXB_OK;
    }
    e.aero_grid = d->n_triangle_indices > 0 ? 1 : 0;

    // --- colours -> per-rank device segments; the smallest cluster whose ranks fit ---
    e.n_colours = static_cast<int>(cs.size());
    e.colour_is_bend.assign(e.n_colours, 0);
    e.colour_batch = colour_batch;
    e.cross_mask = 0;
    for (int c = 0; c < e.n_colours; ++c) {
        e.colour_is_bend[c] = cs[c].bend ? 1 : 0;
        for (const HostSeg& h : cs[c].segs)
            if (h.a_base / e.S != (h.a_base + h.d) / e.S) e.cross_mask |= 1u << c;
    }
    int max_colour = 0;
    bool placed = false;
    // One CTA with everything in shared memory; else lean (positions only in shared memory, rest
    // lengths and lambdas read in place in HBM) on one CTA as float4, as long as the warm start's
    // tiles still fit beside the positions; else lean on one CTA with the positions as float
    // arrays (12 bytes and an inverse-mass index per slot); else lean on two CTAs; else a
    // cluster of 2, 4 or 8 CTAs.
    const struct { int cl; bool lean, soa; } tries[] = {{1, false, false}, {1, true, false}, {1, true, true},
                                                        {2, true, false}, {2, false, false}, {4, false, false},
                                                        {8, false, false}};
    // CTAs per SM by shared memory, with the self-collision tables when the cloth comes with
    // self-collision on (they may take more room beside a lean sheet's positions)
    const bool self_at_add = self_on(e);
    auto smem_ctas = [&](int bytes) {
        const int b = self_at_add && e.self_ok ? std::max(bytes, e.self_smem) : bytes;
        return 233472 / (b + kClothStaticSmem + 1024);
    };
    bool whole_fits = false;  // held whole, one CTA per SM: kept unless the lean layout does better
    for (const auto& t : tries) {
        if (placed) break;
        if (t.soa && !soa_layouts) continue;
        if (whole_fits && !(t.cl == 1 && t.lean && !t.soa)) break;
        std::vector<int32_t> padded;
        if (!build_ranks(e, cs, rest_ref, t.cl, padded, max_colour)) continue;
        e.lean = t.lean;
        e.soa = t.soa;
        e.rest_ref.swap(padded);
        layout_ranks(e);
        if (e.dev.smem_bytes <= kMaxDynamicSmem && (!t.lean || e.warm_smem <= kMaxDynamicSmem)) placed = true;
        if (placed && whole_fits && smem_ctas(e.dev.smem_bytes) < 2) placed = false;
        if (placed && lean_mid && t.cl == 1 && !t.lean && smem_ctas(e.dev.smem_bytes) < 2) {
            whole_fits = true;
            placed = false;
        }
    }
    if (!placed && whole_fits) {  // back to the sheet held whole
        std::vector<int32_t> padded;
        build_ranks(e, cs, rest_ref, 1, padded, max_colour);
        e.lean = e.soa = false;
        e.rest_ref.swap(padded);
        layout_ranks(e);
        placed = true;
    }
    if (!placed) e.lean = e.soa = false;
    if (!placed) {
        // Beyond a cluster: the whole-GPU path (every SM on this cloth, state in global memory).
        std::vector<int32_t> padded;
        if (!build_ranks(e, cs, rest_ref, 1, padded, max_colour))
            return fail(PXB_ERR_TOO_LARGE, "a %ux%u cloth has more colour segments than supported", d->columns,
                        d->rows);
        e.rest_ref.swap(padded);
        layout_ranks(e);
        e.grid = true;
    }
    if (!verify_ranks(e, d)) return fail(PXB_ERR_UNSUPPORTED, "colour segments do not reproduce the constraint lists");
    e.threads = std::min(kClothMaxThreads, std::max(64, ((max_colour + 1) / 2 + 31) & ~31));
    return PXB_OK;
}

pxb_status pxb_context::add_cloth(const pxb_cloth_desc* d, uint64_t* id_out) {
    if (!d || !id_out) return fail(PXB_ERR_INVALID_ARGUMENT, "null argument");
    ClothEntry e;
    std::string msg;
    if (pxb_status st = plan_cloth(d, e, msg, soa_layouts, lean_mid)) return fail(st, "%s", msg.c_str());
    const uint32_t n = d->n_particles;

    // --- anchors: one device record per anchor; a particle follows its LAST anchor ---
    e.anchors.assign(d->anchors, d->anchors + d->n_anchors);
    e.anchor_recs.resize(e.anchors.size());
    for (size_t a = 0; a < e.anchors.size(); ++a) {
        PxbAnchorRec r{};
        std::memcpy(r.prev, e.anchors[a].prev_world_position, 12);
        std::memcpy(r.world, e.anchors[a].world_position, 12);
        e.anchor_recs[a] = r;
    }
    std::vector<int32_t> anchor_of(e.n_layout, -1);
    for (size_t a = 0; a < e.anchors.size(); ++a)
        if (e.anchors[a].particle < n)
            anchor_of[slot_of_particle(static_cast<int>(e.anchors[a].particle), e.cols, e.Q, e.S)] =
                static_cast<int32_t>(a);
    std::vector<int2> tether(e.n_layout, make_int2(-1, 0));
    for (const pxb_tether& t : e.tethers) {
        int ml;
        std::memcpy(&ml, &t.max_length, 4);
        tether[slot_of_particle(static_cast<int>(t.particle), e.cols, e.Q, e.S)] =
            make_int2(slot_of_particle(static_cast<int>(t.anchor), e.cols, e.Q, e.S), ml);
    }
    // rest lengths by rest slot; a general-topology cloth follows them with its packed endpoints
    std::vector<float> rest_h(e.n_rest_total, 0.0f);
    for (size_t s = 0; s < e.rest_ref.size(); ++s) {
        const int32_t r = e.rest_ref[s];
        if (r < 0) continue;  // row padding
        rest_h[s] = r < static_cast<int32_t>(e.n_stretch) ? d->stretch[r].rest_length
                                                          : d->bend[r - e.n_stretch].rest_length;
    }
    if (e.list) {
        uint32_t* w = reinterpret_cast<uint32_t*>(rest_h.data() + e.list_items_pad);
        for (size_t i = 0; i < e.item_ends.size(); ++i) {
            const uint64_t v = e.item_ends[i];
            const uint32_t la = static_cast<uint32_t>(v), lb = static_cast<uint32_t>(v >> 32);
            if (list_wide(e)) {
                w[2 * i] = la;
                w[2 * i + 1] = lb;
            } else {
                w[i] = la | lb << 16;
            }
        }
    }
    e.topology.resize(d->n_stretch + d->n_bend);
    for (uint32_t k = 0; k < d->n_stretch; ++k) e.topology[k] = {d->stretch[k].a, d->stretch[k].b, d->stretch[k].rest_length};
    for (uint32_t k = 0; k < d->n_bend; ++k) e.topology[d->n_stretch + k] = {d->bend[k].a, d->bend[k].b, d->bend[k].rest_length};

    // --- device memory: one allocation, 256-byte aligned sub-buffers ---
    const size_t L = static_cast<size_t>(e.n_layout);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align256(std::max<size_t>(bytes, 16));
        return o;
    };
    const size_t o_pos = take(16 * L), o_vel = take(16 * L), o_prv = take(16 * L);
    const size_t o_rest = take(4 * static_cast<size_t>(e.n_rest_total));
    const size_t o_lam = take(4 * static_cast<size_t>(e.n_rest_total));
    const size_t o_anc = take(4 * L), o_teth = take(8 * L);
    const size_t o_recs = take(sizeof(PxbAnchorRec) * e.anchor_recs.size());
    const size_t o_segs = take(sizeof(PxbSeg) * e.segs.size());
    const size_t o_edge = take(4 * 6 * L), o_disp = take(16 * L);
    const size_t o_runs = take(sizeof(PxbRun) * e.runs.size()), o_troff = take(4 * e.tri_off.size()),
                 o_tent = take(sizeof(int4) * e.tri_ent.size());
    // topology 2: lambdas (at most one per item) or parked velocities, whichever params ask for
    const size_t o_scr = take(e.list_gmem ? 4 * std::max<size_t>(e.list_items_pad, 3 * L) : 0);
    const size_t o_wtab = take(e.soa ? 4 * PXB_MAX_WTAB : 0);
    cudaError_t ce = cudaMalloc(&e.dmem, off);
    if (ce != cudaSuccess) return cuda(ce, "cudaMalloc(cloth)");
    e.dbytes = off;
    char* base = static_cast<char*>(e.dmem);
    const PxbClothDev keep_ranks = e.dev;  // refresh_layout filled the rank fields
    std::memset(&e.dev, 0, sizeof(e.dev));
    std::memcpy(e.dev.rank, keep_ranks.rank, sizeof(e.dev.rank));
    e.dev.smem_bytes = keep_ranks.smem_bytes;
    e.dev.self_buckets = keep_ranks.self_buckets;
    e.dev.self_hash_off = keep_ranks.self_hash_off;
    e.dev.self_restage = keep_ranks.self_restage;
    e.dev.ref_columns = e.ref_columns;
    e.dev.lean = e.lean ? (e.soa ? 2 : 1) : 0;
    e.dev.wtab = e.soa ? reinterpret_cast<const float*>(base + o_wtab) : nullptr;
    e.dev.n_wtab = 0;  // upload_particles fills the table
    e.dev.pos = reinterpret_cast<float4*>(base + o_pos);
    e.dev.vel = reinterpret_cast<float4*>(base + o_vel);
    e.dev.prv = reinterpret_cast<float4*>(base + o_prv);
    e.dev.rest = reinterpret_cast<const float*>(base + o_rest);
    e.dev.lam_out = reinterpret_cast<float*>(base + o_lam);
    e.dev.anchor_of = reinterpret_cast<const int32_t*>(base + o_anc);
    e.dev.tether = reinterpret_cast<const int2*>(base + o_teth);
    e.dev.anchors = reinterpret_cast<float*>(base + o_recs);
    e.dev.segs = reinterpret_cast<const PxbSeg*>(base + o_segs);
    e.dev.n_ranks = static_cast<int32_t>(e.ranks.size());
    e.dev.rows_per_rank = e.ranks[0].n_rows;
    e.dev.n_colours = e.n_colours;
    e.dev.cross_mask = e.cross_mask;
    e.dev.sync_mask = colour_sync_mask(e);
    e.dev.n_layout = e.n_layout;
    e.dev.n_real = static_cast<int32_t>(n);
    e.dev.columns = e.cols;
    e.dev.rows = e.rows;
    e.dev.Q = e.Q;
    e.dev.S = e.S;
    e.dev.n_anchors = static_cast<int32_t>(e.anchor_recs.size());
    e.dev.threads = e.threads;
    e.dev.aero_grid = e.aero_grid;
    for (int c = 0; c < e.n_colours; ++c)
        if (!e.colour_is_bend[c]) e.dev.stretch_mask |= 1u << c;
    e.dev.edge_rest = reinterpret_cast<const float*>(base + o_edge);
    e.dev.disp = reinterpret_cast<float4*>(base + o_disp);
    if (e.list) {
        e.dev.topology = e.list_gmem ? 2 : 1;
        e.dev.list_scratch = e.list_gmem ? reinterpret_cast<float*>(base + o_scr) : nullptr;
        e.dev.runs = reinterpret_cast<const PxbRun*>(base + o_runs);
        e.dev.tri_off = reinterpret_cast<const int32_t*>(base + o_troff);
        e.dev.tri_ent = reinterpret_cast<const int4*>(base + o_tent);
        e.dev.n_runs = static_cast<int32_t>(e.runs.size());
        e.dev.list_items_pad = e.list_items_pad;
    }
    // rest length from each slot to its six triangulation neighbours (+x, -x, +y, -y, +x+y,
    // -x-y), from the stretch list; 0 where no stretch constraint joins the pair
    std::vector<float> edge_rest(6 * L, 0.0f);
    {
        std::unordered_map<uint64_t, float> by_pair;
        by_pair.reserve(2 * d->n_stretch);
        auto key = [](uint32_t a, uint32_t b) {
            return a < b ? (static_cast<uint64_t>(a) << 32 | b) : (static_cast<uint64_t>(b) << 32 | a);
        };
        for (uint32_t k = 0; k < d->n_stretch; ++k) by_pair[key(d->stretch[k].a, d->stretch[k].b)] = d->stretch[k].rest_length;
        const int dxs[6] = {1, -1, 0, 0, 1, -1}, dys[6] = {0, 0, 1, -1, 1, -1};
        for (int y = 0; y < e.rows; ++y)
            for (int x = 0; x < e.cols; ++x) {
                const int l = slot_of_particle(y * e.cols + x, e.cols, e.Q, e.S);
                for (int k = 0; k < 6; ++k) {
                    const int nx = x + dxs[k], ny = y + dys[k];
                    if (nx < 0 || ny < 0 || nx >= e.cols || ny >= e.rows) continue;
                    auto it = by_pair.find(key(static_cast<uint32_t>(y * e.cols + x), static_cast<uint32_t>(ny * e.cols + nx)));
                    if (it != by_pair.end()) edge_rest[static_cast<size_t>(k) * L + l] = it->second;
                }
            }
    }
    pxb_status st = PXB_OK;
    auto up = [&](void* dst, const void* src, size_t bytes, const char* what) {
        if (st || bytes == 0) return;
        st = cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), what);
    };
    up(base + o_rest, rest_h.data(), 4 * rest_h.size(), "upload rest");
    up(base + o_anc, anchor_of.data(), 4 * L, "upload anchor_of");
    up(base + o_teth, tether.data(), 8 * L, "upload tethers");
    up(base + o_edge, edge_rest.data(), 4 * 6 * L, "upload edge rest lengths");
    up(base + o_troff, e.tri_off.data(), 4 * e.tri_off.size(), "upload triangle index");
    up(base + o_tent, e.tri_ent.data(), sizeof(int4) * e.tri_ent.size(), "upload triangle entries");
    if (!st) st = cuda(cudaMemsetAsync(base + o_disp, 0, 16 * L, stream), "zero displacement scratch");
    if (!st) st = upload_segments(e);
    if (!st) st = cuda(cudaMemsetAsync(base + o_lam, 0, 4 * static_cast<size_t>(e.n_rest_total), stream), "zero lambdas");
    if (!st) st = upload_anchor_records(e);
    if (!st) st = upload_particles(e, d->particles);
    if (st) {
        cudaFree(e.dmem);
        return st;
    }

    // --- slot ---
    uint32_t index = 0;
    while (index < cloths.size() && cloths[index].alive) ++index;
    if (index == cloths.size()) cloths.emplace_back();
    e.generation = cloths[index].generation + 1;
    e.alive = true;
    cloths[index] = std::move(e);
    registry_dirty = true;
    ++registry_epoch;
    *id_out = (static_cast<uint64_t>(cloths[index].generation) << 32) | index;
    return PXB_OK;
}

pxb_status pxb_context::sync_registry() {
    if (!registry_dirty) return PXB_OK;
    std::vector<PxbClothDev> h(std::max<size_t>(cloths.size(), 1));
    std::memset(h.data(), 0, sizeof(PxbClothDev) * h.size());
    for (size_t i = 0; i < cloths.size(); ++i)
        if (cloths[i].alive) h[i] = cloths[i].dev;
    pxb_status s = grow(d_registry, sizeof(PxbClothDev) * h.size(), "registry");
    if (s) return s;
    // The registry may be read by an in-flight launch; order the update on the stream.
    s = cuda(cudaMemcpyAsync(d_registry.p, h.data(), sizeof(PxbClothDev) * h.size(),
                             cudaMemcpyHostToDevice, stream),
             "upload registry");
    if (s) return s;
    s = cuda(cudaStreamSynchronize(stream), "upload registry");
    if (s) return s;
    registry_dirty = false;
    return PXB_OK;
}

// Collider snapshot -> device record with the world-space quantities the reference derives
// per call (collision::world_sphere / world_obb / world_capsule, shape.h:160-188).
void pxb_make_dev_collider(const pxb_collider& c, PxbDevCollider& o) {
    using namespace pxb::hm;
    std::memset(&o, 0, sizeof(o));
    o.type = c.type;
    o.enabled = c.enabled;
    const V3 sweep = ld(c.sweep);
    const bool swept = dot(sweep, sweep) > 1e-6f * 1e-6f;
    o.two_pose = swept && (c.type == PXB_SHAPE_BOX || c.type == PXB_SHAPE_CAPSULE) ? 1 : 0;
    o.swept_sphere = swept && c.type == PXB_SHAPE_SPHERE ? 1 : 0;
    o.radius = c.type == PXB_SHAPE_SPHERE ? c.radius : c.capsule_radius;
    std::memcpy(o.he, c.half_extents, 12);
    std::memcpy(o.sweep, c.sweep, 12);
    std::memcpy(o.bmin, c.bounds_min, 12);
    std::memcpy(o.bmax, c.bounds_max, 12);
    const V3 lc = ld(c.local_center);
    const Q4 lr = ldq(c.local_rotation);
    for (int pose = 0; pose < (o.two_pose ? 2 : 1); ++pose) {
        const V3 pp = pose == 0 ? ld(c.position) : add(ld(c.position), sweep);
        const Q4 rot = pose == 0 ? ldq(c.orientation) : ldq(c.end_orientation);
        PxbPose& ps = o.pose[pose];
        const V3 center = add(pp, qrot(rot, lc));
        st(ps.center, center);
        const Q4 orient = qmul(rot, lr);
        V3 ax, ay, az;
        axes(orient, ax, ay, az);
        st(ps.ax, ax);
        st(ps.ay, ay);
        st(ps.az, az);
        if (c.type == PXB_SHAPE_CAPSULE) {
            V3 axis_local{0.0f, 0.0f, 0.0f};
            if (c.capsule_axis == 0) axis_local.x = 1.0f;
            else if (c.capsule_axis == 1) axis_local.y = 1.0f;
            else axis_local.z = 1.0f;
            const V3 axis_world = qrot(orient, axis_local);
            const V3 ca = sub(center, mul(axis_world, c.capsule_half_height));
            const V3 cb = add(center, mul(axis_world, c.capsule_half_height));
            st(ps.ca, ca);
            st(ps.cb, cb);
            st(ps.t1, orthonormal_t1(safe_normalize(sub(cb, ca))));
        } else if (c.type == PXB_SHAPE_SPHERE) {
            st(ps.cb, add(center, sweep));
        }
    }
}

static pxb_status check_colliders(pxb_context* ctx, const pxb_collider* c, uint32_t n) {
    for (uint32_t k = 0; k < n; ++k) {
        if (!c[k].enabled) continue;
        if (c[k].type < 0 || c[k].type > PXB_SHAPE_CONVEX_HULL)
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider %u has an unknown shape type", k);
        if (c[k].type == PXB_SHAPE_CAPSULE && (c[k].capsule_axis < 0 || c[k].capsule_axis > 2))
            return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "collider %u has capsule_axis outside 0..2", k);
    }
    return PXB_OK;
}

void pxb_context::drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    graph_key.clear();
    graph_kernels = 0;
}

pxb_status pxb_context::step_cloths(const pxb_cloth_step_desc* sd, const WarmCfg* warm, bool use_graph) {
    if (!sd || (sd->n_cloths && !sd->cloths)) return fail(PXB_ERR_INVALID_ARGUMENT, "null step");
    const uint32_t n = sd->n_cloths;
    if (n == 0) return PXB_OK;
    if (!(sd->h > 0.0f)) return PXB_OK;  // solve_cloth is a no-op for h <= 0 (cloth_solver.h:163)
    std::vector<ClothEntry*> ents(n);
    uint32_t n_col = 0, n_src = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ents[k] = lookup(sd->cloths[k]);
        if (!ents[k]) return fail(PXB_ERR_INVALID_HANDLE, "cloth id %llu is not live", (unsigned long long)sd->cloths[k]);
        if (self_on(*ents[k]) && (!ents[k]->self_ok || ents[k]->grid))
            return fail(PXB_ERR_UNSUPPORTED,
                        "cloth %llu: self-collision runs on cloths one CTA holds in shared memory with its hash "
                        "tables (grid sides up to ~84, general topology up to ~2800 particles)",
                        (unsigned long long)sd->cloths[k]);
        if (sd->collider_offsets) {
            if (sd->collider_offsets[k + 1] < sd->collider_offsets[k])
                return fail(PXB_ERR_INVALID_ARGUMENT, "collider offsets decrease");
        }
        if (sd->source_offsets && sd->source_offsets[k + 1] < sd->source_offsets[k])
            return fail(PXB_ERR_INVALID_ARGUMENT, "source offsets decrease");
    }
    if (sd->collider_offsets) n_col = sd->collider_offsets[n];
    if (sd->source_offsets) n_src = sd->source_offsets[n];
    if (n_col && !sd->colliders) return fail(PXB_ERR_INVALID_ARGUMENT, "null colliders");
    if (n_src && !sd->sources) return fail(PXB_ERR_INVALID_ARGUMENT, "null sources");
    if (pxb_status s = check_colliders(this, sd->colliders, n_col)) return s;
    ColliderStage cstage;
    if (pxb_status s = cstage.plan(this, sd->colliders, n_col)) return s;
    if (pxb_status s = sync_registry()) return s;

    if (warm) {
        for (uint32_t k = 0; k < n; ++k)
            if (ents[k]->grid || ents[k]->list)
                return fail(PXB_ERR_UNSUPPORTED, "cloth %llu runs on the %s path, which has no warm start",
                            (unsigned long long)sd->cloths[k], ents[k]->grid ? "whole-GPU" : "general-topology");
        for (uint32_t k = 0; k < n; ++k)
            if (ents[k]->warm_smem > kMaxDynamicSmem)
                return fail(PXB_ERR_TOO_LARGE, "cloth %llu: the warm-start kernel needs %d bytes of shared memory",
                            (unsigned long long)sd->cloths[k], ents[k]->warm_smem);
        if (warm->warm_iters > 0 && !has_mlp) return fail(PXB_ERR_INVALID_ARGUMENT, "no network installed");
        if (pxb_status s = grow(d_wresults, sizeof(PxbWarmResult) * n, "warm results")) return s;
    }

    // --- staging layout: steps | colliders | sources | order | warm controls | posed hulls ---
    const size_t b_steps = sizeof(PxbClothStep) * n;
    const size_t b_cols = sizeof(PxbDevCollider) * std::max<uint32_t>(n_col, 1);
    const size_t b_src = sizeof(pxb_gravity_source) * std::max<uint32_t>(n_src, 1);
    const size_t b_order = sizeof(int32_t) * n;
    const size_t b_warm = warm ? sizeof(PxbWarmStep) * n : 0;
    const size_t b_queue = sizeof(int32_t) * n;  // one work-queue counter per launch group (at most n)
    const size_t o_cols = align256(b_steps), o_src = o_cols + align256(b_cols),
                 o_order = o_src + align256(b_src), o_queue = o_order + align256(b_order),
                 o_warm = o_queue + align256(b_queue), o_geo = o_warm + align256(b_warm),
                 total = o_geo + align256(cstage.bytes());
    if (pxb_status s = grow_pinned(total)) return s;
    if (pxb_status s = grow(d_stage, total, "step staging")) return s;
    if (pxb_status s = grow(d_results, sizeof(PxbFrameResult) * n, "results")) return s;
    if (pxb_status s = cuda(cudaEventSynchronize(staged), "wait for the previous upload")) return s;
    char* hb = static_cast<char*>(pinned);
    auto* hs_steps = reinterpret_cast<PxbClothStep*>(hb);
    auto* hs_cols = reinterpret_cast<PxbDevCollider*>(hb + o_cols);
    auto* hs_src = reinterpret_cast<pxb_gravity_source*>(hb + o_src);
    auto* hs_order = reinterpret_cast<int32_t*>(hb + o_order);
    auto* hs_warm = reinterpret_cast<PxbWarmStep*>(hb + o_warm);
    std::memset(hb + o_queue, 0, b_queue);  // every group's queue starts at its first cloth
    cstage.fill(this, sd->colliders, n_col, hs_cols, reinterpret_cast<float4*>(hb + o_geo),
                reinterpret_cast<const float4*>(static_cast<char*>(d_stage.p) + o_geo));
    if (n_src) std::memcpy(hs_src, sd->sources, sizeof(pxb_gravity_source) * n_src);
    // Launch slots grouped by cluster size and by how many of the cloth's CTAs one SM holds
    // (shared memory, threads, registers): one launch per group, so a small cloth is not
    // launched with a large one's shared memory and thread count. Larger cloths first within a
    // group, so the block scheduler's tail holds the small ones.
    auto launch_smem = [&](const ClothEntry& e) {
        const int base = warm ? e.warm_smem : e.dev.smem_bytes;
        return self_on(e) ? std::max(base, e.self_smem) : base;
    };
    // cloths with a mesh or hull collider, with self-collision or of general topology launch the
    // kernel with those stages compiled in (1); general-topology cloths with their state in HBM
    // launch its HBM instantiation (2)
    std::vector<uint8_t> has_geo(n, 0);
    for (uint32_t k = 0; k < n; ++k)
        has_geo[k] = ents[k]->list_gmem
                         ? 2
                         : (self_on(*ents[k]) || ents[k]->list ||
                            (sd->collider_offsets &&
                             cstage.any_geometry(sd->collider_offsets[k],
                                                 sd->collider_offsets[k + 1] - sd->collider_offsets[k])));
    for (uint32_t k = 0; k < n; ++k)
        if (ents[k]->lean)  // lean instantiations: float4 (3, 4), float arrays (5, 6)
            has_geo[k] = static_cast<uint8_t>((ents[k]->soa ? 5 : 3) + has_geo[k]);
    // Block-size variant of each cloth: its layout class's (autotuned), else the context's. A
    // warm-start step runs the context's.
    auto smem_ctas = [&](const ClothEntry& e) {
        return std::max(1, 233472 / (launch_smem(e) + kClothStaticSmem + 1024));
    };
    std::vector<int> tclass(n), var(n);
    for (uint32_t k = 0; k < n; ++k) {
        tclass[k] = 3 * has_geo[k] + std::min(smem_ctas(*ents[k]), 3) - 1;
        var[k] = (!warm && class_variant[tclass[k]] > 0) ? class_variant[tclass[k]] - 1 : cloth_variant;
    }
    if (!warm) {
        for (double& w : class_work) w = 0.0;
        for (uint32_t k = 0; k < n; ++k)
            if (!ents[k]->grid) class_work[tclass[k]] += static_cast<double>(ents[k]->n_layout);
    }
    auto launch_threads = [&](const ClothEntry& e, int v) {
        const int cap = cloth_variant_threads(v);
        // the warm-start kernel runs whole warpgroups (the network's tiles are 128 rows)
        if (warm) return std::min(cap, std::max(128, (e.threads + 127) & ~127));
        int t = std::min(e.threads, cap);
        if (thread_fit && e.ranks.size() == 1 && !e.grid && !e.list) {
            // the CTAs shared memory lets an SM hold split the threads the variant's registers allow
            const int regs = cloth_variant_registers(v);
            const int share = (65536 / (((regs + 7) & ~7) * smem_ctas(e))) & ~31;
            t = std::min(t, std::max(64, share));
        }
        return t;
    };
    std::vector<int> fit(n);
    for (uint32_t k = 0; k < n; ++k)
        fit[k] = ctas_per_sm(launch_smem(*ents[k]), launch_threads(*ents[k], var[k]), cloth_variant_registers(var[k]));
    std::vector<uint32_t> perm(n);
    for (uint32_t k = 0; k < n; ++k) perm[k] = k;
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) {
        if (ents[x]->grid != ents[y]->grid) return ents[y]->grid;  // whole-GPU cloths last
        const size_t rx = ents[x]->ranks.size(), ry = ents[y]->ranks.size();
        if (rx != ry) return rx < ry;
        if (fit[x] != fit[y]) return fit[x] < fit[y];
        if (has_geo[x] != has_geo[y]) return has_geo[x] < has_geo[y];
        if (var[x] != var[y]) return var[x] < var[y];
        return ents[x]->n_layout > ents[y]->n_layout;
    });
    const pxb::hm::V3 g = pxb::hm::ld(sd->gravity);
    for (uint32_t slot = 0; slot < n; ++slot) {
        const uint32_t k = perm[slot];
        ClothEntry& e = *ents[k];
        const pxb_cloth_params& P = e.params;
        PxbClothStep& s = hs_steps[slot];
        std::memset(&s, 0, sizeof(s));
        // solve_cloth prologue (cloth_solver.h:165-194), evaluated exactly as the reference does
        const uint32_t steps = std::max<uint32_t>(1, P.substeps ? P.substeps : sd->substeps);
        const uint32_t iters = std::max<uint32_t>(1, P.iterations ? P.iterations : sd->iterations);
        const float hs = sd->h / static_cast<float>(steps);
        s.hs = hs;
        s.inv_hs = 1.0f / hs;
        s.steps = static_cast<int32_t>(steps);
        s.iters = static_cast<int32_t>(iters);
        for (int c = 0; c < e.n_colours; ++c) s.alpha[c] = colour_compliance(e, c) / (hs * hs);
        pxb::hm::V3 wind = pxb::hm::ld(P.wind);
        if (P.wind_turbulence > 0.0f) {
            const float t = e.time;
            const pxb::hm::V3 gust{std::sin(t * 1.7f) * std::cos(t * 0.9f),
                                   std::sin(t * 1.1f + 1.3f) * std::cos(t * 1.9f),
                                   std::sin(t * 0.7f + 2.7f) * std::cos(t * 1.3f)};
            wind = pxb::hm::add(wind, pxb::hm::V3{P.wind_turbulence * gust.x, P.wind_turbulence * gust.y,
                                                  P.wind_turbulence * gust.z});
        }
        pxb::hm::st(s.wind, wind);
        const pxb::hm::V3 base = pxb::hm::add(pxb::hm::mul(g, P.gravity_scale), pxb::hm::ld(P.external_acceleration));
        pxb::hm::st(s.base_accel, base);
        pxb::hm::st(s.gravity, g);
        s.gravity_scale = P.gravity_scale;
        std::memcpy(s.external_acceleration, P.external_acceleration, 12);
        s.aero = ((P.air_drag > 0.0f || P.air_lift > 0.0f) && e.n_triangle_indices > 0) ? 1 : 0;
        s.air_drag = P.air_drag;
        s.air_lift = P.air_lift;
        s.max_velocity = P.max_velocity;
        s.max_velocity2 = P.max_velocity * P.max_velocity;
        s.damping_factor = 1.0f / (1.0f + P.damping * hs);
        s.thickness = P.thickness;
        s.friction = P.friction;
        s.col_begin = sd->collider_offsets ? static_cast<int32_t>(sd->collider_offsets[k]) : 0;
        s.col_count = sd->collider_offsets ? static_cast<int32_t>(sd->collider_offsets[k + 1] - sd->collider_offsets[k]) : 0;
        s.src_begin = sd->source_offsets ? static_cast<int32_t>(sd->source_offsets[k]) : 0;
        s.src_count = sd->source_offsets ? static_cast<int32_t>(sd->source_offsets[k + 1] - sd->source_offsets[k]) : 0;
        s.write_lambdas = 1;
        s.grid_wait_polls = grid_wait_polls;
        s.grid_extra_arrivals = grid_extra_arrivals;
        s.self_collision = self_on(e) ? 1 : 0;
        s.self_distance = self_on(e) ? P.self_distance : 0.0f;
        hs_order[slot] = static_cast<int32_t>(ents[k] - cloths.data());
        if (warm) {
            PxbWarmStep& w = hs_warm[slot];
            std::memset(&w, 0, sizeof(w));
            w.tau = warm->taus ? warm->taus[k] : warm->tau;
            w.warm_iters = warm->warm_iters;
            w.record = warm->record;
            w.record_substep = warm->record_substep;
            w.rec_x = warm->rec_x;
            w.rec_y = warm->rec_y;
            w.rec_row0 = warm->rec_row0 ? warm->rec_row0[k] : 0;
            w.continue_iters = warm->continue_iters;
        }
        // Cloth::time advances by hs per substep (cloth_solver.h:453), mirrored on the host.
        for (uint32_t q = 0; q < steps; ++q) e.time += hs;
        // Anchors reach their targets: next step lerps from here (cloth_solver.h:457).
        for (PxbAnchorRec& r : e.anchor_recs) std::memcpy(r.prev, r.world, 12);
        for (pxb_anchor& a : e.anchors) std::memcpy(a.prev_world_position, a.world_position, 12);
    }
    char* db = static_cast<char*>(d_stage.p);
    uint32_t n_plain = n;
    while (n_plain > 0 && ents[perm[n_plain - 1]]->grid) --n_plain;
    if (n_plain < n)
        if (pxb_status s = grow(d_grid, sizeof(PxbGridSync) * (n - n_plain), "grid barriers")) return s;
    // Everything from the upload to the join is one enqueue, which a graph step captures once and
    // replays (the upload node copies the pinned staging filled above at each replay).
    int enqueued = 0;
    bool capturing = false;
    auto enqueue = [&]() -> pxb_status {
    if (pxb_status s = cuda(cudaMemcpyAsync(db, hb, total, cudaMemcpyHostToDevice, stream), "upload step")) return s;
    // The pinned staging is free again once this upload ran. A captured graph cannot carry that
    // event (an event recorded inside a capture cannot be waited on from the host); the graph
    // path records it after the whole replay instead.
    if (!capturing)
        if (pxb_status s = cuda(cudaEventRecord(staged, stream), "record upload")) return s;
    // Launch groups: (cluster size, CTAs per SM). With several, each goes to a side stream so
    // they share the SMs instead of running one after another (a group of small cloths alone
    // leaves most of the device idle).
    // Whole-GPU cloths first, one cooperative launch each on the context stream: the side
    // streams below fork after them, so nothing else holds SMs while they run.
    if (n_plain < n) {
        const size_t gbytes = sizeof(PxbGridSync) * (n - n_plain);
        if (pxb_status s = cuda(cudaMemsetAsync(d_grid.p, 0, gbytes, stream), "zero grid barriers")) return s;
        for (uint32_t slot = n_plain; slot < n; ++slot) {
            cudaError_t le = launch_cloth_grid(static_cast<const PxbClothDev*>(d_registry.p),
                                               reinterpret_cast<const PxbClothStep*>(db),
                                               reinterpret_cast<const PxbDevCollider*>(db + o_cols),
                                               reinterpret_cast<const pxb_gravity_source*>(db + o_src),
                                               reinterpret_cast<const int32_t*>(db + o_order),
                                               static_cast<PxbFrameResult*>(d_results.p), d_err,
                                               static_cast<PxbGridSync*>(d_grid.p) + (slot - n_plain),
                                               static_cast<int>(slot), n_sms, stream, has_geo[perm[slot]] != 0);
            if (le != cudaSuccess) return cuda(le, "launch whole-GPU cloth");
            ++enqueued;
        }
    }
    struct Group { uint32_t g0, g1; int cluster, threads, smem; double work; int ext; int fit; int variant; };
    std::vector<Group> groups;
    for (uint32_t g0 = 0; g0 < n_plain;) {
        const int cluster = static_cast<int>(ents[perm[g0]]->ranks.size());
        const int group_fit = fit[perm[g0]];
        const int ext = has_geo[perm[g0]];
        const int gv = var[perm[g0]];
        Group G{g0, g0, cluster, 64, 0, 0.0, ext, group_fit, gv};
        while (G.g1 < n_plain && static_cast<int>(ents[perm[G.g1]]->ranks.size()) == cluster &&
               fit[perm[G.g1]] == group_fit && has_geo[perm[G.g1]] == ext && var[perm[G.g1]] == gv) {
            const ClothEntry& e = *ents[perm[G.g1]];
            G.threads = std::max(G.threads, launch_threads(e, gv));
            G.smem = std::max(G.smem, launch_smem(e));
            G.work += static_cast<double>(e.n_layout);
            ++G.g1;
        }
        groups.push_back(G);
        g0 = G.g1;
    }
    std::stable_sort(groups.begin(), groups.end(), [](const Group& a, const Group& b) { return a.work > b.work; });
    const bool fan_out = groups.size() > 1;
    // the persistent form (launch_mode 1): a group's CTAs stay resident and pop its cloths
    const bool persistent = launch_mode == 1;
    if (fan_out) {
        if (pxb_status s = cuda(cudaEventRecord(fork, stream), "fork")) return s;
        for (int k = 0; k < std::min<int>(kSideStreams, static_cast<int>(groups.size())); ++k)
            if (pxb_status s = cuda(cudaStreamWaitEvent(side[k], fork, 0), "fork wait")) return s;
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& G = groups[gi];
        cudaStream_t st = fan_out ? side[gi % kSideStreams] : stream;
        cudaError_t le = launch_cloth_step(G.variant, G.cluster, static_cast<const PxbClothDev*>(d_registry.p),
                                           reinterpret_cast<const PxbClothStep*>(db) + G.g0,
                                           reinterpret_cast<const PxbDevCollider*>(db + o_cols),
                                           reinterpret_cast<const pxb_gravity_source*>(db + o_src),
                                           reinterpret_cast<const int32_t*>(db + o_order) + G.g0,
                                           static_cast<PxbFrameResult*>(d_results.p) + G.g0, d_err,
                                           static_cast<int>(G.g1 - G.g0), G.threads, G.smem, st,
                                           warm ? reinterpret_cast<const PxbWarmStep*>(db + o_warm) + G.g0 : nullptr,
                                           warm && warm->warm_iters > 0 ? static_cast<const unsigned char*>(d_mlp.p) : nullptr,
                                           warm ? static_cast<PxbWarmResult*>(d_wresults.p) + G.g0 : nullptr, G.ext,
                                           persistent ? reinterpret_cast<int*>(db + o_queue) + gi : nullptr,
                                           persistent ? std::max(1, n_sms * std::max(G.fit, 1) / G.cluster) : 0);
        if (le != cudaSuccess) return cuda(le, "launch cloth_step");
        ++enqueued;
    }
    if (fan_out) {
        for (int k = 0; k < std::min<int>(kSideStreams, static_cast<int>(groups.size())); ++k) {
            if (pxb_status s = cuda(cudaEventRecord(join[k], side[k]), "join")) return s;
            if (pxb_status s = cuda(cudaStreamWaitEvent(stream, join[k], 0), "join wait")) return s;
        }
    }
    return PXB_OK;
    };
    if (!use_graph || warm) {
        if (pxb_status s = enqueue()) return s;
        launches += static_cast<uint64_t>(enqueued);
    } else {
        // The replayed graph is valid while the launch sequence and every buffer it names are the
        // same: same cloths in the same order, same collider / source counts and variant, no
        // buffer regrown. A new key runs eagerly once, then is captured on its second use.
        std::vector<uint64_t> key(sd->cloths, sd->cloths + n);
        for (uint64_t v : {uint64_t(n_col), uint64_t(n_src), uint64_t(cloth_variant), uint64_t(total),
                           uint64_t(reinterpret_cast<uintptr_t>(d_stage.p)), uint64_t(reinterpret_cast<uintptr_t>(d_results.p)),
                           uint64_t(reinterpret_cast<uintptr_t>(d_registry.p)), uint64_t(reinterpret_cast<uintptr_t>(pinned)),
                           uint64_t(reinterpret_cast<uintptr_t>(d_grid.p)), registry_epoch})
            key.push_back(v);
        for (uint32_t k = 0; k < n; k += 21) {  // which kernel instantiation each cloth launches
            uint64_t bits = 0;
            for (uint32_t j = k; j < std::min(n, k + 21); ++j) bits |= uint64_t(has_geo[j]) << (3 * (j - k));
            key.push_back(bits);
        }
        for (uint32_t k = 0; k < n; k += 32) {  // and with which block-size variant
            uint64_t bits = 0;
            for (uint32_t j = k; j < std::min(n, k + 32); ++j) bits |= uint64_t(var[j]) << (2 * (j - k));
            key.push_back(bits);
        }
        if (graph_exec && key == graph_key) {
            if (pxb_status s = cuda(cudaGraphLaunch(graph_exec, stream), "launch step graph")) return s;
            if (pxb_status s = cuda(cudaEventRecord(staged, stream), "record step graph")) return s;
            launches += static_cast<uint64_t>(graph_kernels);
        } else if (key == graph_pending) {
            drop_graph();
            if (pxb_status s = cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
                return s;
            capturing = true;
            const pxb_status es = enqueue();
            capturing = false;
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (es) {
                if (g) cudaGraphDestroy(g);
                return es;
            }
            if (ce != cudaSuccess) return cuda(ce, "end capture");
            graph = g;
            if (pxb_status s = cuda(cudaGraphInstantiate(&graph_exec, graph, 0), "instantiate step graph")) return s;
            graph_key = key;
            graph_kernels = enqueued;
            if (pxb_status s = cuda(cudaGraphLaunch(graph_exec, stream), "launch step graph")) return s;
            if (pxb_status s = cuda(cudaEventRecord(staged, stream), "record step graph")) return s;
            launches += static_cast<uint64_t>(enqueued);
        } else {
            if (pxb_status s = enqueue()) return s;
            launches += static_cast<uint64_t>(enqueued);
            graph_pending = key;
        }
    }
    last_step.resize(n);
    for (uint32_t slot = 0; slot < n; ++slot) {
        last_step[slot] = sd->cloths[perm[slot]];
        ents[perm[slot]]->last_slot = static_cast<int32_t>(slot);
    }
    last_step_warm = warm != nullptr;
    warm_fresh = false;
    results_fresh = false;
    return PXB_OK;
}

pxb_status pxb_context::check_device_error() {
    uint32_t h = 0;
    pxb_status s = cuda(cudaMemcpyAsync(&h, d_err, 4, cudaMemcpyDeviceToHost, stream), "read error word");
    if (s) return s;
    s = cuda(cudaStreamSynchronize(stream), "synchronize");
    if (s) return s;
    if (h) {
        cudaMemsetAsync(d_err, 0, 4, stream);
        return fail(PXB_ERR_DEVICE_STATUS, "device error word 0x%x (1 bad index, 2 staging wait expired, 4 queue wait expired, 8 tensor-core wait expired)", h);
    }
    return PXB_OK;
}

pxb_status pxb_context::fetch_warm_results() {
    if (warm_fresh) return PXB_OK;
    if (!last_step_warm) return PXB_OK;
    const size_t n = last_step.size();
    std::vector<PxbWarmResult> h(n);
    if (n) {
        pxb_status s = cuda(cudaMemcpyAsync(h.data(), d_wresults.p, sizeof(PxbWarmResult) * n,
                                            cudaMemcpyDeviceToHost, stream), "read warm results");
        if (s) return s;
    }
    if (pxb_status s = check_device_error()) return s;
    for (size_t k = 0; k < n; ++k) {
        ClothEntry* e = lookup(last_step[k]);
        if (!e) continue;
        e->warm_result = h[k];
        e->has_warm_result = true;
    }
    warm_fresh = true;
    return PXB_OK;
}

pxb_status pxb_context::fetch_results() {
    if (results_fresh) return PXB_OK;
    const size_t n = last_step.size();
    std::vector<PxbFrameResult> h(n);
    if (n) {
        pxb_status s = cuda(cudaMemcpyAsync(h.data(), d_results.p, sizeof(PxbFrameResult) * n,
                                            cudaMemcpyDeviceToHost, stream),
                            "read results");
        if (s) return s;
    }
    if (pxb_status s = check_device_error()) return s;
    for (size_t k = 0; k < n; ++k) {
        ClothEntry* e = lookup(last_step[k]);
        if (!e) continue;
        e->result = h[k];
        e->result.time = e->time;
        e->has_result = true;
    }
    results_fresh = true;
    return PXB_OK;
}

// ------------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------------

extern "C" {

pxb_status pxb_context_create(int device, pxb_context** out) {
    if (!out) return PXB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* ctx = new (std::nothrow) pxb_context();
    if (!ctx) return PXB_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->staged, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming);
    for (int k = 0; k < pxb_context::kSideStreams && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->n_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_err, 4);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, 4);
    if (e != cudaSuccess) {
        delete ctx;
        return e == cudaErrorMemoryAllocation ? PXB_ERR_OUT_OF_MEMORY : PXB_ERR_CUDA;
    }
    *out = ctx;
    return PXB_OK;
}

pxb_status pxb_context_destroy(pxb_context* ctx) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    delete ctx;
    return PXB_OK;
}

const char* pxb_last_error(const pxb_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

pxb_status pxb_context_stream(pxb_context* ctx, void** stream_out) {
    if (!ctx || !stream_out) return PXB_ERR_INVALID_ARGUMENT;
    *stream_out = ctx->stream;
    return PXB_OK;
}

pxb_status pxb_context_synchronize(pxb_context* ctx) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    return ctx->check_device_error();
}

uint64_t pxb_context_launch_count(const pxb_context* ctx) { return ctx ? ctx->launches : 0; }

pxb_status pxb_cloth_add(pxb_context* ctx, const pxb_cloth_desc* desc, uint64_t* id_out) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    return ctx->add_cloth(desc, id_out);
}

pxb_status pxb_cloth_plan_layout(const pxb_cloth_desc* desc, pxb_cloth_plan* out, char* err, uint32_t err_cap) {
    if (err && err_cap) err[0] = 0;
    if (!out) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry e;
    std::string msg;
    const pxb_status st = plan_cloth(desc, e, msg);
    if (st) {
        if (err && err_cap) snprintf(err, err_cap, "%s", msg.c_str());
        return st;
    }
    out->n_ranks = e.grid ? 0 : static_cast<int32_t>(e.ranks.size());
    out->rows_per_rank = e.ranks[0].n_rows;
    out->threads = e.threads;
    out->smem_bytes = e.grid ? 0 : e.dev.smem_bytes;
    out->n_colours = e.n_colours;
    out->n_segments = static_cast<int32_t>(e.segs.size());
    out->layout_slots = e.n_layout;
    out->constraint_slots = e.n_rest_total;
    out->self_collision = e.self_ok && !e.grid ? 1 : 0;
    out->self_smem_bytes = e.self_ok && !e.grid ? e.self_smem : 0;
    out->topology = e.list_gmem ? 2 : (e.list ? 1 : 0);
    out->lean = e.lean ? (e.soa ? 2 : 1) : 0;
    if (e.list) out->n_colours = static_cast<int32_t>(e.runs.size());
    {
        const uint32_t m = colour_sync_mask(e);
        out->phases = e.list ? out->n_colours
                             : __builtin_popcount(m & (e.n_colours >= 32 ? 0xffffffffu : ((1u << e.n_colours) - 1u)));
    }
    return PXB_OK;
}

pxb_status pxb_cloth_remove(pxb_context* ctx, uint64_t id) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    cudaStreamSynchronize(ctx->stream);
    cudaFree(e->dmem);
    const uint32_t gen = e->generation;
    *e = ClothEntry();
    e->generation = gen;
    e->alive = false;
    ctx->registry_dirty = true;
    ++ctx->registry_epoch;
    ctx->results_fresh = false;
    ctx->last_step.clear();
    return PXB_OK;
}

pxb_status pxb_cloth_set_params(pxb_context* ctx, uint64_t id, const pxb_cloth_params* params) {
    if (!ctx || !params) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    const pxb_cloth_params old = e->params;
    e->params = *params;
    ctx->refresh_layout(*e);
    if (!e->grid && e->dev.smem_bytes > kMaxDynamicSmem) {
        e->params = old;
        ctx->refresh_layout(*e);
        return ctx->fail(PXB_ERR_TOO_LARGE, "these params need more shared memory than the path holds");
    }
    if (pxb_status s = ctx->upload_segments(*e)) return s;
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "set params");
}

pxb_status pxb_cloth_write_particles(pxb_context* ctx, uint64_t id, const pxb_particle* particles, uint32_t n) {
    if (!ctx || !particles) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    if (n != e->n_particles) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "particle count mismatch");
    return ctx->upload_particles(*e, particles);
}

pxb_status pxb_cloth_read_particles(pxb_context* ctx, uint64_t id, pxb_particle* out, uint32_t n) {
    if (!ctx || !out) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    if (n != e->n_particles) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "particle count mismatch");
    const size_t L = static_cast<size_t>(e->n_layout);
    std::vector<float4> pos(L), vel(L), prv(L);
    pxb_status s = ctx->cuda(cudaMemcpyAsync(pos.data(), e->dev.pos, 16 * L, cudaMemcpyDeviceToHost, ctx->stream), "read pos");
    if (!s) s = ctx->cuda(cudaMemcpyAsync(vel.data(), e->dev.vel, 16 * L, cudaMemcpyDeviceToHost, ctx->stream), "read vel");
    if (!s) s = ctx->cuda(cudaMemcpyAsync(prv.data(), e->dev.prv, 16 * L, cudaMemcpyDeviceToHost, ctx->stream), "read prv");
    if (!s) s = ctx->check_device_error();
    if (s) return s;
    for (uint32_t i = 0; i < n; ++i) {
        const int l = slot_of_particle(static_cast<int>(i), e->cols, e->Q, e->S);
        pxb_particle& p = out[i];
        p.position[0] = pos[l].x; p.position[1] = pos[l].y; p.position[2] = pos[l].z;
        p.inv_mass = pos[l].w;
        p.velocity[0] = vel[l].x; p.velocity[1] = vel[l].y; p.velocity[2] = vel[l].z;
        p.prev_position[0] = prv[l].x; p.prev_position[1] = prv[l].y; p.prev_position[2] = prv[l].z;
    }
    return PXB_OK;
}

pxb_status pxb_cloth_read_lambdas(pxb_context* ctx, uint64_t id, float* stretch_out, uint32_t n_stretch,
                                  float* bend_out, uint32_t n_bend) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    if ((stretch_out && n_stretch != e->n_stretch) || (bend_out && n_bend != e->n_bend))
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "lambda count mismatch");
    std::vector<float> lam(std::max(e->n_lam, 1));
    pxb_status s = PXB_OK;
    if (e->n_lam)
        s = ctx->cuda(cudaMemcpyAsync(lam.data(), e->dev.lam_out, 4 * static_cast<size_t>(e->n_lam),
                                      cudaMemcpyDeviceToHost, ctx->stream), "read lambdas");
    if (!s) s = ctx->check_device_error();
    if (s) return s;
    if (stretch_out) std::fill(stretch_out, stretch_out + n_stretch, 0.0f);
    if (bend_out) std::fill(bend_out, bend_out + n_bend, 0.0f);
    if (e->list) {
        for (const PxbRun& run : e->runs) {
            if (run.lam_base < 0) continue;
            for (int i = 0; i < run.count; ++i) {
                const int32_t r = e->rest_ref[run.item_base + i];
                const float v = lam[run.lam_base + i];
                if (r < static_cast<int32_t>(e->n_stretch)) { if (stretch_out) stretch_out[r] = v; }
                else if (bend_out) bend_out[r - e->n_stretch] = v;
            }
        }
        return PXB_OK;
    }
    for (const ClothEntry::Rank& rk : e->ranks) {
        for (int sg = rk.seg_begin; sg < rk.seg_begin + rk.colour_seg[e->n_colours]; ++sg) {
            const PxbSeg& g = e->segs[sg];
            if (g.lam_base < 0) continue;
            for (int i = 0; i < g.count; ++i) {
                const int32_t r = e->rest_ref[rk.rest_off + g.rest_base + i];
                if (r < 0) continue;
                const float v = lam[rk.lam_off + g.lam_base + i];
                if (r < static_cast<int32_t>(e->n_stretch)) { if (stretch_out) stretch_out[r] = v; }
                else if (bend_out) bend_out[r - e->n_stretch] = v;
            }
        }
    }
    return PXB_OK;
}

pxb_status pxb_cloth_set_anchor_targets(pxb_context* ctx, uint64_t id, const float* world_xyz, uint32_t n) {
    if (!ctx || (n && !world_xyz)) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    if (n != e->anchors.size()) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "anchor count mismatch");
    for (uint32_t a = 0; a < n; ++a) {
        std::memcpy(e->anchor_recs[a].world, world_xyz + 3 * a, 12);
        std::memcpy(e->anchors[a].world_position, world_xyz + 3 * a, 12);
    }
    return ctx->upload_anchor_records(*e);
}

pxb_status pxb_cloth_read_anchors(pxb_context* ctx, uint64_t id, pxb_anchor* out, uint32_t n) {
    if (!ctx || (n && !out)) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    if (n != e->anchors.size()) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "anchor count mismatch");
    if (n) std::memcpy(out, e->anchors.data(), sizeof(pxb_anchor) * n);
    return PXB_OK;
}

pxb_status pxb_cloth_read_time(pxb_context* ctx, uint64_t id, float* time_out) {
    if (!ctx || !time_out) return PXB_ERR_INVALID_ARGUMENT;
    ClothEntry* e = ctx->lookup(id);
    if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
    *time_out = e->time;
    return PXB_OK;
}

pxb_status pxb_cloths_step(pxb_context* ctx, const pxb_cloth_step_desc* step) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    return ctx->step_cloths(step);
}

pxb_status pxb_cloths_step_graph(pxb_context* ctx, const pxb_cloth_step_desc* step) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    return ctx->step_cloths(step, nullptr, true);
}

pxb_status pxb_cloths_read_results(pxb_context* ctx, const uint64_t* cloths, uint32_t n,
                                   pxb_cloth_frame_result* out) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    if (pxb_status s = ctx->fetch_results()) return s;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        if (!e->has_result) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "cloth has not been stepped");
        static_assert(sizeof(pxb_cloth_frame_result) == sizeof(PxbFrameResult), "result layout");
        std::memcpy(&out[k], &e->result, sizeof(PxbFrameResult));
    }
    return PXB_OK;
}

pxb_status pxb_cloths_read_positions(pxb_context* ctx, const uint64_t* cloths, uint32_t n, float* out,
                                     size_t capacity) {
    if (!ctx || (n && (!cloths || !out))) return PXB_ERR_INVALID_ARGUMENT;
    std::vector<int32_t> order(n);
    std::vector<int64_t> offs(n);
    int64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ClothEntry* e = ctx->lookup(cloths[k]);
        if (!e) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        order[k] = static_cast<int32_t>(e - ctx->cloths.data());
        offs[k] = total;
        total += 3 * static_cast<int64_t>(e->n_particles);
    }
    if (static_cast<size_t>(total) > capacity) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "output too small");
    if (n == 0) return PXB_OK;
    if (pxb_status s = ctx->sync_registry()) return s;
    // the cloth order, then (256-byte aligned) the output offsets: sized before anything is copied
    if (pxb_status s = ctx->grow(ctx->d_gather_meta, align256(4 * static_cast<size_t>(n)) + 8 * static_cast<size_t>(n),
                                 "gather meta"))
        return s;
    if (pxb_status s = ctx->grow(ctx->d_gather, 4 * static_cast<size_t>(total), "gather")) return s;
    char* meta = static_cast<char*>(ctx->d_gather_meta.p);
    pxb_status s = ctx->cuda(cudaMemcpyAsync(meta, order.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), "gather order");
    if (!s) s = ctx->cuda(cudaMemcpyAsync(meta + align256(4 * n), offs.data(), 8 * n, cudaMemcpyHostToDevice, ctx->stream), "gather offsets");
    if (s) return s;
    cudaError_t le = launch_gather_positions(static_cast<const PxbClothDev*>(ctx->d_registry.p),
                                             reinterpret_cast<const int32_t*>(meta),
                                             reinterpret_cast<const int64_t*>(meta + align256(4 * n)),
                                             static_cast<int>(n), static_cast<float*>(ctx->d_gather.p),
                                             ctx->stream);
    if (le != cudaSuccess) return ctx->cuda(le, "launch gather");
    s = ctx->cuda(cudaMemcpyAsync(out, ctx->d_gather.p, 4 * static_cast<size_t>(total), cudaMemcpyDeviceToHost,
                                  ctx->stream), "read positions");
    if (s) return s;
    return ctx->check_device_error();
}

pxb_status pxb_project_particles(pxb_context* ctx, const pxb_collider* collider, float thickness,
                                 const float* points_xyz, const float* motion_start_xyz, uint32_t n,
                                 float* points_out, float* normals_out, float* depths_out, int32_t* hit_out) {
    if (!ctx || !collider || (n && (!points_xyz || !points_out || !normals_out || !depths_out || !hit_out)))
        return PXB_ERR_INVALID_ARGUMENT;
    if (pxb_status s = check_colliders(ctx, collider, 1)) return s;
    ColliderStage cstage;
    if (pxb_status s = cstage.plan(ctx, collider, 1)) return s;
    const size_t nb = static_cast<size_t>(n);
    const size_t o_geo = align256(sizeof(PxbDevCollider)), o_pts = o_geo + align256(cstage.bytes()),
                 o_st = o_pts + align256(12 * nb), o_out = o_st + align256(motion_start_xyz ? 12 * nb : 0),
                 o_nrm = o_out + align256(12 * nb), o_dep = o_nrm + align256(12 * nb),
                 o_hit = o_dep + align256(4 * nb), total = o_hit + align256(4 * nb);
    if (pxb_status s = ctx->grow(ctx->d_scratch, total, "projection scratch")) return s;
    char* b = static_cast<char*>(ctx->d_scratch.p);
    std::vector<char> host(o_pts);
    cstage.fill(ctx, collider, 1, reinterpret_cast<PxbDevCollider*>(host.data()),
                reinterpret_cast<float4*>(host.data() + o_geo), reinterpret_cast<const float4*>(b + o_geo));
    pxb_status s = ctx->cuda(cudaMemcpyAsync(b, host.data(), o_pts, cudaMemcpyHostToDevice, ctx->stream), "upload collider");
    if (!s && n) s = ctx->cuda(cudaMemcpyAsync(b + o_pts, points_xyz, 12 * nb, cudaMemcpyHostToDevice, ctx->stream), "upload points");
    if (!s && n && motion_start_xyz)
        s = ctx->cuda(cudaMemcpyAsync(b + o_st, motion_start_xyz, 12 * nb, cudaMemcpyHostToDevice, ctx->stream), "upload starts");
    if (s) return s;
    // the host staging above must outlive the copies
    if (pxb_status s2 = ctx->cuda(cudaStreamSynchronize(ctx->stream), "upload collider")) return s2;
    cudaError_t le = launch_project_points(reinterpret_cast<const PxbDevCollider*>(b), thickness,
                                           reinterpret_cast<const float*>(b + o_pts),
                                           motion_start_xyz ? reinterpret_cast<const float*>(b + o_st) : nullptr,
                                           static_cast<int>(n),
                                           reinterpret_cast<float*>(b + o_out), reinterpret_cast<float*>(b + o_nrm),
                                           reinterpret_cast<float*>(b + o_dep), reinterpret_cast<int32_t*>(b + o_hit),
                                           ctx->stream);
    if (le != cudaSuccess) return ctx->cuda(le, "launch projection");
    ++ctx->launches;
    if (n) {
        s = ctx->cuda(cudaMemcpyAsync(points_out, b + o_out, 12 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, ctx->stream), "read points");
        if (!s) s = ctx->cuda(cudaMemcpyAsync(normals_out, b + o_nrm, 12 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, ctx->stream), "read normals");
        if (!s) s = ctx->cuda(cudaMemcpyAsync(depths_out, b + o_dep, 4 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, ctx->stream), "read depths");
        if (!s) s = ctx->cuda(cudaMemcpyAsync(hit_out, b + o_hit, 4 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, ctx->stream), "read hits");
        if (s) return s;
    }
    return ctx->check_device_error();
}

pxb_status pxb_solve_cloth_host(pxb_context* ctx, const pxb_cloth_desc* desc, pxb_particle* particles,
                                pxb_constraint* stretch, pxb_constraint* bend, pxb_anchor* anchors,
                                const pxb_collider* colliders, uint32_t n_colliders, const float gravity[3],
                                uint32_t substeps, uint32_t iterations, float h, float* time_inout,
                                float* bounds_out) {
    if (!ctx || !desc || !gravity) return PXB_ERR_INVALID_ARGUMENT;
    if (desc->n_particles == 0 || !(h > 0.0f)) return PXB_OK;  // solve_cloth no-ops (cloth_solver.h:163)
    // Reuse the registration made for these arrays when the topology is unchanged.
    HostSolveCache* hit = nullptr;
    for (HostSolveCache& c : ctx->host_cache) {
        if (c.particles != desc->particles || !ctx->lookup(c.id)) continue;
        ClothEntry* e = ctx->lookup(c.id);
        bool same = e->n_particles == desc->n_particles && e->n_stretch == desc->n_stretch &&
                    e->n_bend == desc->n_bend && e->anchors.size() == desc->n_anchors &&
                    e->tethers.size() == desc->n_tethers;
        for (uint32_t k = 0; same && k < desc->n_stretch; ++k)
            same = e->topology[k].a == desc->stretch[k].a && e->topology[k].b == desc->stretch[k].b &&
                   e->topology[k].rest == desc->stretch[k].rest_length;
        for (uint32_t k = 0; same && k < desc->n_bend; ++k)
            same = e->topology[desc->n_stretch + k].a == desc->bend[k].a &&
                   e->topology[desc->n_stretch + k].b == desc->bend[k].b &&
                   e->topology[desc->n_stretch + k].rest == desc->bend[k].rest_length;
        for (uint32_t k = 0; same && k < desc->n_tethers; ++k)
            same = std::memcmp(&e->tethers[k], &desc->tethers[k], sizeof(pxb_tether)) == 0;
        if (same) { hit = &c; break; }
        pxb_cloth_remove(ctx, c.id);
        c.particles = nullptr;
    }
    uint64_t id = 0;
    pxb_status s = PXB_OK;
    if (!hit) {
        if ((s = ctx->add_cloth(desc, &id))) return s;
        ctx->host_cache.push_back(HostSolveCache{desc->particles, id});
    } else {
        id = hit->id;
        ClothEntry* e = ctx->lookup(id);
        e->params = desc->params;
        ctx->refresh_layout(*e);
        if (!e->grid && e->dev.smem_bytes > kMaxDynamicSmem) return ctx->fail(PXB_ERR_TOO_LARGE, "params need too much shared memory");
        if ((s = ctx->upload_segments(*e))) return s;
        if ((s = ctx->upload_particles(*e, desc->particles))) return s;
        for (uint32_t a = 0; a < desc->n_anchors; ++a) {
            e->anchors[a] = desc->anchors[a];
            std::memcpy(e->anchor_recs[a].prev, desc->anchors[a].prev_world_position, 12);
            std::memcpy(e->anchor_recs[a].world, desc->anchors[a].world_position, 12);
        }
        if ((s = ctx->upload_anchor_records(*e))) return s;
        e->time = desc->time;
    }
    ClothEntry* e = ctx->lookup(id);
    if (time_inout) e->time = *time_inout;
    std::vector<uint32_t> offs = {0, n_colliders};
    pxb_cloth_step_desc sd{};
    sd.cloths = &id;
    sd.n_cloths = 1;
    sd.colliders = colliders;
    sd.collider_offsets = offs.data();
    std::memcpy(sd.gravity, gravity, 12);
    sd.substeps = substeps;
    sd.iterations = iterations;
    sd.h = h;
    if ((s = ctx->step_cloths(&sd))) return s;
    if ((s = pxb_cloth_read_particles(ctx, id, particles, desc->n_particles))) return s;
    if (stretch || bend) {
        std::vector<float> ls(desc->n_stretch), lb(desc->n_bend);
        if ((s = pxb_cloth_read_lambdas(ctx, id, ls.data(), desc->n_stretch, lb.data(), desc->n_bend))) return s;
        if (stretch) for (uint32_t k = 0; k < desc->n_stretch; ++k) stretch[k].lambda = ls[k];
        if (bend) for (uint32_t k = 0; k < desc->n_bend; ++k) bend[k].lambda = lb[k];
    }
    if (anchors) for (uint32_t a = 0; a < desc->n_anchors; ++a) std::memcpy(anchors[a].prev_world_position, anchors[a].world_position, 12);
    if (time_inout) *time_inout = e->time;
    if (bounds_out) {
        pxb_cloth_frame_result r;
        if ((s = pxb_cloths_read_results(ctx, &id, 1, &r))) return s;
        std::memcpy(bounds_out, r.bounds_min, 12);
        std::memcpy(bounds_out + 3, r.bounds_max, 12);
    }
    return PXB_OK;
}


pxb_status pxb_context_set_wait_test(pxb_context* ctx, uint32_t grid_wait_polls, uint32_t unreachable) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (grid_wait_polls == 0) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "a wait needs at least one poll");
    ctx->grid_wait_polls = grid_wait_polls;
    ctx->grid_extra_arrivals = unreachable ? 1u : 0u;
    return PXB_OK;
}

pxb_status pxb_context_set_launch_mode(pxb_context* ctx, int32_t mode) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (mode != 0 && mode != 1) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "launch mode must be 0 or 1");
    ctx->launch_mode = mode;
    return PXB_OK;
}

pxb_status pxb_context_get_tuning(pxb_context* ctx, int32_t* variant, int32_t* launch_mode, int32_t* thread_fit,
                                  int32_t* class_variants, double* class_slots) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (variant) *variant = ctx->cloth_variant;
    if (launch_mode) *launch_mode = ctx->launch_mode;
    if (thread_fit) *thread_fit = ctx->thread_fit;
    for (int c = 0; c < PXB_TUNE_CLASSES; ++c) {
        if (class_variants) class_variants[c] = ctx->class_variant[c] > 0 ? ctx->class_variant[c] - 1 : ctx->cloth_variant;
        if (class_slots) class_slots[c] = ctx->class_work[c];
    }
    return PXB_OK;
}

pxb_status pxb_context_set_thread_fit(pxb_context* ctx, int32_t mode) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (mode != 0 && mode != 1) return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "thread fit must be 0 or 1");
    ctx->thread_fit = mode;
    return PXB_OK;
}

pxb_status pxb_context_set_lean_mid(pxb_context* ctx, int32_t enable) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    ctx->lean_mid = enable != 0;
    return PXB_OK;
}

pxb_status pxb_context_set_lean_arrays(pxb_context* ctx, int32_t enable) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    ctx->soa_layouts = enable != 0;
    return PXB_OK;
}

pxb_status pxb_context_set_cloth_variant(pxb_context* ctx, int32_t variant) {
    if (!ctx) return PXB_ERR_INVALID_ARGUMENT;
    if (variant < 0 || variant >= kClothVariants)
        return ctx->fail(PXB_ERR_INVALID_ARGUMENT, "variant must be in [0, %d)", kClothVariants);
    ctx->cloth_variant = variant;
    std::memset(ctx->class_variant, 0, sizeof(ctx->class_variant));  // every class at this variant
    return PXB_OK;
}

pxb_status pxb_cloths_autotune(pxb_context* ctx, const pxb_cloth_step_desc* step, uint32_t trials,
                               int32_t* variant_out, float* ms_out) {
    if (!ctx || !step) return PXB_ERR_INVALID_ARGUMENT;
    if (trials == 0) trials = 1;
    const uint32_t n = step->n_cloths;
    std::vector<ClothEntry*> ents(n);
    size_t bytes = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ents[k] = ctx->lookup(step->cloths[k]);
        if (!ents[k]) return ctx->fail(PXB_ERR_INVALID_HANDLE, "cloth id is not live");
        bytes += 48 * static_cast<size_t>(ents[k]->n_layout) + 4 * static_cast<size_t>(ents[k]->n_lam) +
                 sizeof(PxbAnchorRec) * ents[k]->anchor_recs.size() + 3 * 256;
    }
    if (pxb_status s = ctx->grow(ctx->d_tune, bytes, "autotune state")) return s;
    // Save the device state and the host mirrors a step touches.
    struct Saved { float time; std::vector<PxbAnchorRec> recs; std::vector<pxb_anchor> anchors; PxbFrameResult result; bool has; };
    std::vector<Saved> saved(n);
    auto copy_state = [&](bool save) -> pxb_status {
        char* t = static_cast<char*>(ctx->d_tune.p);
        for (uint32_t k = 0; k < n; ++k) {
            ClothEntry& e = *ents[k];
            const size_t L = 16 * static_cast<size_t>(e.n_layout);
            void* parts[4] = {e.dev.pos, e.dev.vel, e.dev.prv, e.dev.lam_out};
            const size_t sz[4] = {L, L, L, 4 * static_cast<size_t>(e.n_lam)};
            for (int q = 0; q < 4; ++q) {
                if (sz[q]) {
                    cudaError_t ce = cudaMemcpyAsync(save ? static_cast<void*>(t) : parts[q],
                                                     save ? parts[q] : static_cast<void*>(t), sz[q],
                                                     cudaMemcpyDeviceToDevice, ctx->stream);
                    if (ce != cudaSuccess) return ctx->cuda(ce, "autotune save/restore");
                }
                t += align256(sz[q]);
            }
            if (save) saved[k] = Saved{e.time, e.anchor_recs, e.anchors, e.result, e.has_result};
            else {
                e.time = saved[k].time;
                e.anchor_recs = saved[k].recs;
                e.anchors = saved[k].anchors;
                e.result = saved[k].result;
                e.has_result = saved[k].has;
                if (pxb_status s = ctx->upload_anchor_records(e)) return s;
            }
        }
        return PXB_OK;
    };
    if (pxb_status s = copy_state(true)) return s;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const int before = ctx->cloth_variant, before_mode = ctx->launch_mode;
    int before_class[PXB_TUNE_CLASSES];
    std::memcpy(before_class, ctx->class_variant, sizeof(before_class));
    std::memset(ctx->class_variant, 0, sizeof(ctx->class_variant));
    int best = before + kClothVariants * before_mode;
    float best_ms = 0.0f;
    pxb_status st = PXB_OK;
    // one warm-up step (attribute set-up), then `trials` timed steps
    auto time_steps = [&](float& ms) -> pxb_status {
        if (pxb_status s = ctx->step_cloths(step)) return s;
        cudaEventRecord(t0, ctx->stream);
        for (uint32_t r = 0; r < trials; ++r)
            if (pxb_status s = ctx->step_cloths(step)) return s;
        cudaEventRecord(t1, ctx->stream);
        if (cudaEventSynchronize(t1) != cudaSuccess) return ctx->fail(PXB_ERR_CUDA, "autotune timing");
        ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        ms /= static_cast<float>(trials);
        return PXB_OK;
    };
    for (int v = 0; v < 2 * kClothVariants && !st; ++v) {
        ctx->cloth_variant = v % kClothVariants;
        ctx->launch_mode = v / kClothVariants;
        float ms = 0.0f;
        st = time_steps(ms);
        if (st) break;
        if (ms_out) ms_out[v] = ms;
        if (v == 0 || ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    // Per layout class, largest share first: each other variant for its cloths alone, timed in
    // turn with the current choice (current, other, current, other, so that a drift of the clock
    // over the comparison falls on both) and kept when faster by more than 1 %.
    if (!st) {
        ctx->cloth_variant = best % kClothVariants;
        ctx->launch_mode = best / kClothVariants;
        float cur = 0.0f;
        st = time_steps(cur);  // also records each class's share under the chosen pair
        std::vector<int> classes;
        for (int c = 0; c < PXB_TUNE_CLASSES; ++c)
            if (ctx->class_work[c] > 0.0) classes.push_back(c);
        std::stable_sort(classes.begin(), classes.end(),
                         [&](int a, int b) { return ctx->class_work[a] > ctx->class_work[b]; });
        for (size_t ci = 0; ci < classes.size() && classes.size() > 1 && !st; ++ci) {
            const int c = classes[ci];
            int keep = 0;
            for (int v = 0; v < kClothVariants && !st; ++v) {
                if (v == ctx->cloth_variant || v + 1 == keep) continue;
                float base = 0.0f, alt = 0.0f;
                for (int rep = 0; rep < 2 && !st; ++rep) {
                    float ms = 0.0f;
                    ctx->class_variant[c] = keep;
                    st = time_steps(ms);
                    base += ms;
                    if (st) break;
                    ctx->class_variant[c] = v + 1;
                    st = time_steps(ms);
                    alt += ms;
                }
                if (!st && alt < base * 0.99f) keep = v + 1;
            }
            ctx->class_variant[c] = keep;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    pxb_status rs = copy_state(false);
    if (!rs) rs = ctx->check_device_error();
    ctx->results_fresh = false;
    ctx->last_step.clear();
    ctx->cloth_variant = st ? before : best % kClothVariants;
    ctx->launch_mode = st ? before_mode : best / kClothVariants;
    if (st) std::memcpy(ctx->class_variant, before_class, sizeof(before_class));
    if (st) return st;
    if (rs) return rs;
    if (variant_out) *variant_out = best;
    return PXB_OK;
}

}  // extern "C"
