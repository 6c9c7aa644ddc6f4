// cloth_step.cuh -- the XPBD cloth substep kernel on sm_100a: one CTA per cloth, the cloth resident
// in shared memory for the whole step.
//
// Replaces cloth::solve_cloth (physxcoopa/cloth/cloth_solver.h:158-460). One
// launch advances a batch of cloths by one call each (the loop of PhysicsWorld::step_cloths_,
// world.h:1759-1847). Per CTA:
//
//   prologue   cp.async.bulk (TMA, no multicast) stages positions and rest lengths from HBM into
//              shared memory behind an mbarrier. A thread owns layout slots tid, tid + T, ...;
//              their velocities and substep-start positions stay in the cloth's own HBM arrays
//              (L2-resident while the CTA runs; only the owner touches a slot), which leaves the
//              whole register budget to the projection loop.
//   substeps   1 aero (per-particle gather of its incident triangles, ascending triangle order)
//              2+3 integrate + anchor lerp (owner thread)
//              4 iterations x colours of project_distance over affine colour segments,
//                one __syncthreads per colour (colours are particle-disjoint); a cloth of
//                general topology walks its runs instead (PxbRun, kExt instantiations only)
//              5+7+8 tethers, collider projection, velocity + friction + clamp (owner thread)
//   epilogue   positions back to HBM with cp.async.bulk, lambdas stored, bounds and max speed
//              reduced with warp shuffles.
//
// Arithmetic is IEEE single precision with no contraction (built with -fmad=false) and the
// reference's operation order, so a step reproduces the CPU oracle to the bit (up to the sign of
// an exactly-zero coordinate; see the lambda note in the colour loop).
//
// This header holds the kernel template; its instantiations are launched from one translation
// unit per launch family (cloth_step_plain.cu, _warm, _geo, _lean, _gmem), so the library's
// heaviest code compiles in parallel. cloth_kernel.cu dispatches between them.
#ifndef PXB_CLOTH_STEP_CUH
#define PXB_CLOTH_STEP_CUH

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"
#include "pxb_kernels.h"
#include "pxb_mlp.cuh"
#include "pxb_device_math.cuh"
#include "pxb_self_collision.cuh"

namespace cg = cooperative_groups;

namespace pxb {
namespace {

constexpr uint32_t kWaitLimit = 1u << 26;  // bounded mbarrier polls before giving up

// ------------------------------------------------------------------------------------------
// TMA bulk copies and mbarriers (inline PTX)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t saddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on phase `parity`; returns false (and the caller raises an error word) if the
// transaction never completes.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    return false;
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(saddr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit_and_wait() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------------------------------------------
// Aerodynamics: one triangle's per-corner share (cloth_solver.h:204-225)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ void tri_share(f3 p0, f3 p1, f3 p2, f3 v0, f3 v1, f3 v2, f3 wind,
                                          float drag, float lift, f3& acc) {
    const f3 e1 = sub(p1, p0);
    const f3 e2 = sub(p2, p0);
    const f3 cr = cross(e1, e2);
    const float twice_area = len(cr);
    if (twice_area < PXB_EPSILON) return;
    const f3 face_n = divs(cr, twice_area);
    const f3 v = sub(mul(add(add(v0, v1), v2), 1.0f / 3.0f), wind);
    const float vn = dot(v, face_n);
    const f3 vt = sub(v, smul(vn, face_n));
    const float scale = -0.5f * twice_area * fabsf(vn);
    const f3 inner = add(smul(drag * vn, face_n), smul(lift, vt));
    const f3 force = smul(scale, inner);
    acc = add(acc, mul(force, 1.0f / 3.0f));
}

__device__ __forceinline__ int lay(int x, int y, int Q, int S) { return y * S + (x & 3) * Q + (x >> 2); }

// ------------------------------------------------------------------------------------------
// Block reductions (warp shuffles, fixed order -> deterministic)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ------------------------------------------------------------------------------------------
// One colour segment: project_distance (cloth_solver.h:119-138) for every item
// ------------------------------------------------------------------------------------------

// Items of one colour share no particle, so with registers to spare (512-thread blocks) a
// thread takes two per pass and loads both before storing either: two independent dependency
// chains (square root, divisions) in flight per thread. The reference's early returns (both
// endpoints pinned; coincident endpoints) become a predicate on the stores, with its comparisons
// kept as written (a NaN weight is not skipped). An item's row is a multiply-high by the
// segment's magic reciprocal (exact for every item index used), so segments carry no padding;
// a second item past the segment reads item 0's slots and stores nothing.
// h0 = {count, magic, per_row, a_base}, h1 = {row_stride, d, rest_base, lam_base}.
struct PairItem {
    float4* pa;
    float4* pb;
    float4 a, b;
    float rest, lam;
    bool live;
};

__device__ __forceinline__ int seg_row(int i, uint32_t magic) {
    return magic ? static_cast<int>(__umulhi(static_cast<uint32_t>(i), magic)) : i;
}

template <int CL, bool kLam>
__device__ __forceinline__ void load_item(PairItem& it, float4* pos, float4* pos_next, const float* rest,
                                          const float* lamv, int n_local, int i, int count, uint32_t magic,
                                          int per_row, int a_base, int row_stride, int d) {
    it.live = i < count;
    const int ii = it.live ? i : 0;
    const int row = seg_row(ii, magic);
    const int la = a_base + row * row_stride + (ii - row * per_row);
    const int lb = la + d;
    it.pa = &pos[la];
    it.pb = (CL == 1 || lb < n_local) ? &pos[lb] : &pos_next[lb - n_local];
    it.a = *it.pa;
    it.b = *it.pb;
    it.rest = rest[ii];
    it.lam = kLam ? lamv[ii] : 0.0f;
}

template <bool kLam>
__device__ __forceinline__ void project_item(PairItem& it, float* lamv, int i, float alpha) {
    float4 a = it.a, b = it.b;
    float dlambda;
    const bool ok = distance_core<kLam>(a, b, it.rest, it.lam, alpha, dlambda) && it.live;
    if (ok) {
        *it.pa = a;
        *it.pb = b;
        if (kLam) lamv[i] = it.lam + dlambda;
    }
}

template <int CL, bool kLam, int kItems>
__device__ __forceinline__ void project_segment(float4* __restrict__ pos, float4* __restrict__ pos_next,
                                                const float* __restrict__ rest, float* __restrict__ lamv,
                                                int n_local, int4 h0, int4 h1, float alpha, int& i0, int T) {
    const int tid = i0;
    const int count = h0.x, per_row = h0.z, a_base = h0.w;
    const uint32_t magic = static_cast<uint32_t>(h0.y);
    const int row_stride = h1.x, d = h1.y;
    if constexpr (kItems == 2) {
        for (int i = tid; i < count; i += 2 * T) {
            PairItem x, y;
            load_item<CL, kLam>(x, pos, pos_next, rest, lamv, n_local, i, count, magic, per_row, a_base,
                                row_stride, d);
            load_item<CL, kLam>(y, pos, pos_next, rest, lamv, n_local, i + T, count, magic, per_row,
                                a_base, row_stride, d);
            project_item<kLam>(x, lamv, i, alpha);
            project_item<kLam>(y, lamv, i + T, alpha);
        }
    } else {
        int i = i0;
        for (; i < count; i += T) {
            PairItem x;
            load_item<CL, kLam>(x, pos, pos_next, rest, lamv, n_local, i, count, magic, per_row, a_base,
                                row_stride, d);
            project_item<kLam>(x, lamv, i, alpha);
        }
        i0 = i - count;  // the thread's first item in the next segment of the phase
    }
}

// One run of a general-topology cloth (PxbRun): item i joins the slots packed in ends[i]
// (a | b << 16), reads rest[i] and, when the batch is compliant, lamv[i]. The items of a run
// share no particle, so they are projected like the items of a colour segment.
template <bool kLam>
__device__ __forceinline__ void load_run_item(PairItem& it, float4* pos, const float* rest, const uint32_t* ends,
                                              const float* lamv, int i, int count, bool wide = false) {
    it.live = i < count;
    const int ii = it.live ? i : 0;
    if (wide) {  // two words per item: (a, b)
        const uint2 w = reinterpret_cast<const uint2*>(ends)[ii];
        it.pa = &pos[w.x];
        it.pb = &pos[w.y];
    } else {
        const uint32_t w = ends[ii];
        it.pa = &pos[w & 0xffffu];
        it.pb = &pos[w >> 16];
    }
    it.a = *it.pa;
    it.b = *it.pb;
    it.rest = rest[ii];
    it.lam = kLam ? lamv[ii] : 0.0f;
}

// wide: ends holds (a, b) word pairs (a cloth of more than kListNarrowSlots slots, in HBM); the
// runs' item offsets index items either way.
template <bool kLam, int kItems, bool kWide = false>
__device__ __forceinline__ void project_run(float4* __restrict__ pos, const float* __restrict__ rest,
                                            const uint32_t* __restrict__ ends, float* __restrict__ lamv, int count,
                                            float alpha, int tid, int T) {
    if constexpr (kItems == 2) {
        for (int i = tid; i < count; i += 2 * T) {
            PairItem x, y;
            load_run_item<kLam>(x, pos, rest, ends, lamv, i, count, kWide);
            load_run_item<kLam>(y, pos, rest, ends, lamv, i + T, count, kWide);
            project_item<kLam>(x, lamv, i, alpha);
            project_item<kLam>(y, lamv, i + T, alpha);
        }
    } else {
        for (int i = tid; i < count; i += T) {
            PairItem x;
            load_run_item<kLam>(x, pos, rest, ends, lamv, i, count, kWide);
            project_item<kLam>(x, lamv, i, alpha);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Positions of a lean one-CTA cloth as float arrays (PxbClothDev::lean == 2)
// ------------------------------------------------------------------------------------------

// x, y of slot l at xy[l] (one 8-byte access), z at z[l]; its inverse mass is wt[wi[l]] (the
// cloth's table of distinct values, in shared memory), or, with w_hbm, pos[l].w read in place in
// HBM.
// Indexing yields a reference that reads and writes a float4 (x, y, z, inverse mass), so the
// stages outside the projection read like those of the float4 layout; a write keeps the inverse
// mass, which no stage changes.
struct SoaPos {
    float2* xy;
    float* z;
    const uint8_t* wi;
    const float* wt;
    const float4* g;
    int n;
    bool w_hbm;
    __device__ __forceinline__ float w(int l) const { return w_hbm ? __ldg(&g[l].w) : wt[wi[l]]; }
    __device__ __forceinline__ float4 get(int l) const {
        const float2 p = xy[l];
        return make_float4(p.x, p.y, z[l], w(l));
    }
    __device__ __forceinline__ void set(int l, float4 v) const {
        xy[l] = make_float2(v.x, v.y);
        z[l] = v.z;
    }
    struct Ref;
    __device__ __forceinline__ Ref operator[](int l) const;
};

struct SoaPos::Ref {
    SoaPos s;
    int l;
    __device__ __forceinline__ operator float4() const { return s.get(l); }
    __device__ __forceinline__ Ref& operator=(float4 v) {
        s.set(l, v);
        return *this;
    }
    __device__ __forceinline__ Ref& operator=(const Ref& o) {
        s.set(l, o.s.get(o.l));
        return *this;
    }
};

__device__ __forceinline__ SoaPos::Ref SoaPos::operator[](int l) const { return Ref{*this, l}; }

// Positions from HBM (layout order, float4) into the arrays; each slot's inverse mass becomes
// its index in the table (binary search over the bit patterns, ascending). A value missing from
// the table records PXB_DEVERR_BAD_INDEX and takes index 0. Plain loads: the warm start stages
// from positions this kernel wrote. Called by every thread; the caller synchronises afterwards.
__device__ __forceinline__ void soa_stage(const SoaPos& P, float* wt_smem, const float4* src,
                                          const float* __restrict__ wtab, int n_wtab, uint32_t* err, int tid,
                                          int T) {
    for (int i = tid; i < n_wtab; i += T) wt_smem[i] = __ldg(&wtab[i]);
    __syncthreads();
    uint8_t* wi = const_cast<uint8_t*>(P.wi);
    for (int l = tid; l < P.n; l += T) {
        const float4 v = src[l];
        P.xy[l] = make_float2(v.x, v.y);
        P.z[l] = v.z;
        if (!P.w_hbm) {
            const uint32_t key = __float_as_uint(v.w);
            int lo = 0, hi = n_wtab - 1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__float_as_uint(wt_smem[mid]) < key) lo = mid + 1;
                else hi = mid;
            }
            if (n_wtab == 0 || __float_as_uint(wt_smem[lo]) != key) {
                atomicOr(err, PXB_DEVERR_BAD_INDEX);
                lo = 0;
            }
            wi[l] = static_cast<uint8_t>(lo);
        }
    }
}

// One colour segment of a lean one-CTA cloth held as arrays: the same items, addresses and
// arithmetic as project_segment; the inverse masses from the table (kWH false) or from HBM.
template <bool kWH, bool kLam, int kItems>
__device__ __forceinline__ void project_segment_soa(const SoaPos& P, const float* __restrict__ rest,
                                                    float* __restrict__ lamv, int4 h0, int4 h1, float alpha, int& i0,
                                                    int T) {
    const int tid = i0;
    const int count = h0.x, per_row = h0.z, a_base = h0.w;
    const uint32_t magic = static_cast<uint32_t>(h0.y);
    const int row_stride = h1.x, d = h1.y;
    float2* __restrict__ XY = P.xy;
    float* __restrict__ Z = P.z;
    auto wof = [&](int l) -> float { return kWH ? __ldg(&P.g[l].w) : P.wt[P.wi[l]]; };
    auto one = [&](int i, int& la, int& lb, float4& a, float4& b, float& r, float& lam, bool& live) {
        live = i < count;
        const int ii = live ? i : 0;
        const int row = seg_row(ii, magic);
        la = a_base + row * row_stride + (ii - row * per_row);
        lb = la + d;
        const float2 pa = XY[la], pb = XY[lb];
        a = make_float4(pa.x, pa.y, Z[la], wof(la));
        b = make_float4(pb.x, pb.y, Z[lb], wof(lb));
        r = rest[ii];
        lam = kLam ? lamv[ii] : 0.0f;
    };
    auto put = [&](int i, int la, int lb, float4 a, float4 b, float r, float lam, bool live) {
        float dlambda;
        if (distance_core<kLam>(a, b, r, lam, alpha, dlambda) && live) {
            XY[la] = make_float2(a.x, a.y);
            Z[la] = a.z;
            XY[lb] = make_float2(b.x, b.y);
            Z[lb] = b.z;
            if (kLam) lamv[i] = lam + dlambda;
        }
    };
    if constexpr (kItems == 2) {
        for (int i = tid; i < count; i += 2 * T) {
            int la0, lb0, la1, lb1;
            float4 a0, b0, a1, b1;
            float r0, r1, m0, m1;
            bool v0, v1;
            one(i, la0, lb0, a0, b0, r0, m0, v0);
            one(i + T, la1, lb1, a1, b1, r1, m1, v1);
            put(i, la0, lb0, a0, b0, r0, m0, v0);
            put(i + T, la1, lb1, a1, b1, r1, m1, v1);
        }
    } else {
        int i = i0;
        for (; i < count; i += T) {
            int la, lb;
            float4 a, b;
            float r, m;
            bool v;
            one(i, la, lb, a, b, r, m, v);
            put(i, la, lb, a, b, r, m, v);
        }
        i0 = i - count;
    }
}

// ------------------------------------------------------------------------------------------
// The constraint iterations of a general-topology cloth (one CTA), out of line
// ------------------------------------------------------------------------------------------

// `iters` walks of the runs in order, a CTA barrier after each run; alpha of a run evaluated as
// the reference does, compliance / (hs * hs). Out of line for the same reason as the grid loop
// below. kWideOk compiles the two-word endpoint form in (the instantiation whose state is in HBM,
// the only one a cloth of more than kListNarrowSlots slots runs in); `wide` selects it.
template <int kItems, bool kWideOk>
__device__ __noinline__ void list_iterations(int iters, int n_runs, const int4* __restrict__ runs, float hs2,
                                             float4* __restrict__ pos, const float* __restrict__ rest,
                                             const uint32_t* __restrict__ ends, float* __restrict__ U, bool wide,
                                             int tid, int T) {
    for (int it = 0; it < iters; ++it) {
        for (int r = 0; r < n_runs; ++r) {
            const int4 run = __ldg(&runs[r]);
            const float alpha = __int_as_float(run.w) / hs2;
            bool done = false;
            if constexpr (kWideOk) {
                if (wide) {
                    if (run.z >= 0)
                        project_run<true, kItems, true>(pos, rest + run.y, ends + 2 * run.y, U + run.z, run.x, alpha, tid, T);
                    else
                        project_run<false, kItems, true>(pos, rest + run.y, ends + 2 * run.y, U, run.x, alpha, tid, T);
                    done = true;
                }
            }
            if (!done) {
                if (run.z >= 0)
                    project_run<true, kItems>(pos, rest + run.y, ends + run.y, U + run.z, run.x, alpha, tid, T);
                else
                    project_run<false, kItems>(pos, rest + run.y, ends + run.y, U, run.x, alpha, tid, T);
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------------------------
// The constraint iterations of a one-CTA grid cloth, out of line
// ------------------------------------------------------------------------------------------

// `iters` sweeps of every colour, a CTA barrier after each phase. Called, not inlined, from the step
// kernel: the projection loop is then register-allocated on its own instead of sharing the
// kernel's register budget (64 per thread at 1024 threads) with every value the kernel keeps
// live across the iterations; the call's register saves happen once per substep.
// The thread's items continue from segment to segment (items t, t + T, ... of the colour's
// segments end to end), so every thread of a colour gets the floor or the ceiling of its share,
// however the items split into segments.
// Bit c of sync_mask clear: colours c and c + 1 touch disjoint particles and run as one phase
// (no barrier between them; the thread's items continue from one into the other).
template <int kItems>
__device__ __noinline__ void grid_iterations(int iters, int n_colours, const int4* __restrict__ seg4,
                                             const int* __restrict__ colour_seg, const float* __restrict__ alpha_of,
                                             float4* __restrict__ pos, const float* __restrict__ RG,
                                             float* __restrict__ U, int n_local, int tid, int T, uint32_t sync_mask) {
    int i0 = tid;
    for (int it = 0; it < iters; ++it) {
        for (int c = 0; c < n_colours; ++c) {
            const float alpha = alpha_of[c];
            const int se = colour_seg[c + 1];
            for (int sg = colour_seg[c]; sg < se; ++sg) {
                const int4 h0 = seg4[2 * sg], h1 = seg4[2 * sg + 1];
                if (h1.w >= 0)
                    project_segment<1, true, kItems>(pos, nullptr, RG + h1.z, U + h1.w, n_local, h0, h1, alpha, i0, T);
                else
                    project_segment<1, false, kItems>(pos, nullptr, RG + h1.z, U, n_local, h0, h1, alpha, i0, T);
            }
            if ((sync_mask >> c) & 1u) {
                __syncthreads();
                i0 = tid;
            }
        }
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// The kernel
// ------------------------------------------------------------------------------------------

// Slot addressing of a cloth split over a cluster: a CTA (rank) holds rows [row0, row0 +
// n_rows); its neighbours' rows are reached through distributed shared memory.
struct RankView {
    float4* pos;        // this rank's positions (shared memory)
    float* U;           // this rank's union region (lambdas / velocity scratch)
    int base;           // global layout slot of local slot 0
    int n_local;        // slots held
};

template <int CL>
__device__ __forceinline__ RankView rank_view(const PxbClothDev& C, unsigned char* smem, int r) {
    const PxbRank& R = C.rank[r];
    RankView v;
    v.n_local = R.n_rows * C.S;
    v.base = R.row0 * C.S;
    unsigned char* b = smem;
    if constexpr (CL > 1) {
        b = static_cast<unsigned char*>(cg::this_cluster().map_shared_rank(static_cast<void*>(smem), r));
    }
    v.pos = reinterpret_cast<float4*>(b);
    v.U = reinterpret_cast<float*>(b + 16 * static_cast<size_t>(v.n_local)) + R.n_rest_pad;
    return v;
}

template <int CL>
__device__ __forceinline__ void cluster_or_block_sync() {
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();
}

template <int kMaxThreads, int CL, bool kWarm, bool kExt, bool kGmem = false, int kLean = 0>
__global__ void __launch_bounds__(kMaxThreads, 1)
cloth_step_kernel(const PxbClothDev* __restrict__ cloths, const PxbClothStep* __restrict__ stepp,
                  const PxbDevCollider* __restrict__ colliders,
                  const pxb_gravity_source* __restrict__ sources,
                  const int32_t* __restrict__ order, PxbFrameResult* __restrict__ results,
                  uint32_t* __restrict__ err, const PxbWarmStep* __restrict__ wsteps,
                  const unsigned char* __restrict__ mlp_blob, PxbWarmResult* __restrict__ wres,
                  int* __restrict__ queue, int n_items) {
    extern __shared__ __align__(16) unsigned char smem[];
    // warm-start state: per-rank residuals, the network warpgroups' MMA barriers, TMEM base
    __shared__ float s_resid[PXB_MAX_RANKS];
    __shared__ __align__(8) uint64_t s_wbar[kWarmGroups];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(16) PxbSeg s_seg[PXB_MAX_SEGS];
    // Per-cloth scalars live in shared memory and are read at their point of use: held in
    // registers for the whole kernel they would crowd out the projection loop (64 registers
    // at 1024 threads).
    __shared__ __align__(16) PxbClothDev sC;
    __shared__ PxbClothStep sP;
    __shared__ float s_red[32][7];
    __shared__ float s_rank_red[PXB_MAX_RANKS][7];
    __shared__ float s_base[3];
    __shared__ float s_run[3];

    __shared__ int s_slot;

    const int tid = threadIdx.x;
    const int T = blockDim.x;
    int rank = 0;
    if constexpr (CL > 1) rank = static_cast<int>(cg::this_cluster().block_rank());
    if (tid == 0) {
        mbar_init(&bar, 1);
        if constexpr (kWarm)
            for (int g = 0; g < kWarmGroups; ++g) tc::mbar_init(&s_wbar[g], 1);
        fence_proxy_async();
    }
    // barrier parities live as long as the CTA: a persistent CTA stages cloth after cloth
    uint32_t wphase = 0;       // parity of this thread's network-warpgroup MMA barrier
    uint32_t stage_phase = 1;  // parity of the staging barrier's last completed phase

    // One cloth per CTA (cluster), or, with a work queue, cloth after cloth: the queue holds
    // the launch group's cloths in decreasing size (the runtime's order), rank 0 pops the next
    // with one atomic and hands it to the cluster; every pop returns, so the loop is bounded
    // by n_items.
    for (int item = 0;; ++item) {
    int slot;
    if (queue == nullptr) {
        if (item > 0) break;
        slot = blockIdx.x / CL;
    } else {
        if (rank == 0 && tid == 0) {
            const int v = atomicAdd(queue, 1);
            if constexpr (CL > 1) {
                for (int q = 0; q < CL; ++q) *cg::this_cluster().map_shared_rank(&s_slot, q) = v;
            } else {
                s_slot = v;
            }
        }
        cluster_or_block_sync<CL>();
        slot = s_slot;
        if (slot >= n_items) break;
    }
    {
        const int ci = __ldg(&order[slot]);
        const int* srcC = reinterpret_cast<const int*>(&cloths[ci]);
        int* dstC = reinterpret_cast<int*>(&sC);
        for (int i = tid; i < static_cast<int>(sizeof(PxbClothDev) / 4); i += T) dstC[i] = srcC[i];
        const int* srcP = reinterpret_cast<const int*>(&stepp[slot]);
        int* dstP = reinterpret_cast<int*>(&sP);
        for (int i = tid; i < static_cast<int>(sizeof(PxbClothStep) / 4); i += T) dstP[i] = srcP[i];
    }
    __syncthreads();

    // a general-topology cloth whose state stays in HBM runs only in the kGmem instantiation,
    // and that instantiation runs nothing else
    constexpr bool kG = kGmem && kExt && CL == 1 && !kWarm;
    // a lean cloth (only positions in shared memory; rest lengths and lambdas read in place in
    // HBM, velocities for the aerodynamic gather too) runs only in the kLean instantiations
    constexpr bool kL = kLean != 0 && CL <= 2 && !kG;
    // a lean one-CTA cloth whose positions are float arrays runs only in the kLean == 2
    // instantiations
    constexpr bool kS = kLean == 2 && CL == 1 && !kG;
    constexpr int kWantLean = kS ? 2 : (kL ? 1 : 0);
    if ((sC.topology == 2) != kG || sC.lean != kWantLean) {  // every rank of a cluster agrees
        if (tid == 0) atomicOr(err, PXB_DEVERR_BAD_INDEX);
        return;
    }
    const int n_ranks = CL > 1 ? sC.n_ranks : 1;
    const RankView me = rank_view<1>(sC, smem, rank);  // local view, plain shared addresses
    auto pos = [&]() {
        if constexpr (kS) {
            const int n = me.n_local;
            return SoaPos{reinterpret_cast<float2*>(smem), reinterpret_cast<float*>(smem + 8 * static_cast<size_t>(n)),
                          smem + 12 * static_cast<size_t>(n),
                          reinterpret_cast<const float*>(smem + 12 * static_cast<size_t>(n) + ((n + 15) & ~15)),
                          sC.pos + me.base, n, sC.n_wtab == 0};
        } else {
            return kG ? sC.pos : me.pos;
        }
    }();
    float* U = kG ? sC.list_scratch : (kL ? sC.lam_out + sC.rank[rank].lam_off : me.U);
    const int n_local = me.n_local;
    const int base = me.base;
    float* rest = kG ? const_cast<float*>(sC.rest) : reinterpret_cast<float*>(smem + 16 * static_cast<size_t>(n_local));
    // where the colour loop reads rest lengths: shared memory, or in place in HBM (lean)
    float* RG = kL ? const_cast<float*>(sC.rest) + sC.rank[rank].rest_off : rest;
    RankView prv_rank{}, nxt_rank{};
    if constexpr (CL > 1) {
        if (rank > 0) prv_rank = rank_view<CL>(sC, smem, rank - 1);
        if (rank + 1 < n_ranks) nxt_rank = rank_view<CL>(sC, smem, rank + 1);
    }

    // --- prologue: stage positions and rest lengths with TMA bulk copies -------------------
    if constexpr (!kS) {  // a cloth held as arrays is staged by its threads below
        if (tid == 0 && !kG) {
            const uint32_t pos_bytes = 16u * static_cast<uint32_t>(n_local);
            const uint32_t rest_bytes = kL ? 0u : 4u * static_cast<uint32_t>(sC.rank[rank].n_rest_pad);
            mbar_arrive_expect_tx(&bar, pos_bytes + rest_bytes);
            bulk_g2s(pos, sC.pos + base, pos_bytes, &bar);
            if (rest_bytes) bulk_g2s(rest, sC.rest + sC.rank[rank].rest_off, rest_bytes, &bar);
        }
    }
    {
        const int sb = sC.rank[rank].seg_begin;
        const int ns = sC.rank[rank].colour_seg[sC.n_colours];
        for (int i = tid; i < ns; i += T) s_seg[i] = sC.segs[sb + i];
    }
    // A staging wait that runs out records the error and carries on: leaving early would strand
    // the other ranks of the cluster at their barriers.
    bool staged = true;
    if constexpr (kS) {
        soa_stage(pos, const_cast<float*>(pos.wt), sC.pos + base, sC.wtab, sC.n_wtab, err, tid, T);
    } else if (!kG) {
        stage_phase ^= 1u;
        staged = mbar_wait_bounded(&bar, stage_phase);
    }
    if (!staged && tid == 0) atomicOr(err, PXB_DEVERR_TMA_TIMEOUT);
    __syncthreads();

    // --- gravity: uniform, or the source field at the cloth's mean position (world.h:1833) --
    if (sP.src_count > 0) {
        // PhysicsWorld::cloth_centre_ (world.h:2072-2076): the mean in particle order, summed
        // sequentially exactly as the reference does (rank after rank, handing the running sum
        // on), so the gravity it selects is the reference's to the bit.
        for (int r = 0; r < n_ranks; ++r) {
            if (r == rank && tid == 0) {
                const int Q = sC.Q, S = sC.S, cols = sC.columns;
                float cx = 0.0f, cy = 0.0f, cz = 0.0f;
                if (r > 0) { cx = s_run[0]; cy = s_run[1]; cz = s_run[2]; }
                const int y0 = sC.rank[r].row0, y1 = y0 + sC.rank[r].n_rows;
                for (int y = y0; y < y1 && y < sC.rows; ++y)
                    for (int x = 0; x < cols; ++x) {
                        const float4 p = pos[lay(x, y, Q, S) - base];
                        cx += p.x; cy += p.y; cz += p.z;
                    }
                if (r + 1 < n_ranks) {
                    float* dst = s_run;
                    if constexpr (CL > 1) dst = cg::this_cluster().map_shared_rank(s_run, r + 1);
                    dst[0] = cx; dst[1] = cy; dst[2] = cz;
                } else {
                    const float fn = static_cast<float>(sC.n_real);
                    const f3 centre = mk(cx / fn, cy / fn, cz / fn);
                    // PhysicsWorld::field_at_ (world.h:2048-2068)
                    float best = 0.0f;
                    f3 pull = mk(sP.gravity[0], sP.gravity[1], sP.gravity[2]);
                    bool found = false;
                    for (int k = 0; k < sP.src_count; ++k) {
                        const pxb_gravity_source* g = &sources[sP.src_begin + k];
                        const f3 d = sub(ld3(g->centre), centre);
                        const float rr = len(d);
                        const float range = __ldg(&g->range), radius = __ldg(&g->radius),
                                    strength = __ldg(&g->strength);
                        if (range > 0.0f && rr > range) continue;
                        if (rr < 1e-6f) continue;
                        const float a = rr <= radius ? strength : strength * (radius / rr) * (radius / rr);
                        if (!found || a > best) {
                            best = a;
                            pull = mul(divs(d, rr), a);
                            found = true;
                        }
                    }
                    const f3 bacc = add(mul(pull, sP.gravity_scale),
                                        mk(sP.external_acceleration[0], sP.external_acceleration[1],
                                           sP.external_acceleration[2]));
                    for (int q = 0; q < n_ranks; ++q) {
                        float* dst = s_base;
                        if constexpr (CL > 1) dst = cg::this_cluster().map_shared_rank(s_base, q);
                        dst[0] = bacc.x; dst[1] = bacc.y; dst[2] = bacc.z;
                    }
                }
            }
            cluster_or_block_sync<CL>();
        }
    } else if (tid == 0) {
        s_base[0] = sP.base_accel[0]; s_base[1] = sP.base_accel[1]; s_base[2] = sP.base_accel[2];
    }
    cluster_or_block_sync<CL>();

    const int4* seg4 = reinterpret_cast<const int4*>(s_seg);
    float4* pos_next = nxt_rank.pos;
    auto iterate = [&](int iters) {
        if constexpr (kExt && CL == 1 && !kWarm && !kS) {
            if (sC.topology != 0) {
                // general topology: run after run, a block barrier after each; alpha evaluated
                // as the reference does, compliance / (hs * hs)
                const uint32_t* ends = reinterpret_cast<const uint32_t*>(rest + sC.list_items_pad);
                constexpr int kItems = kMaxThreads <= 512 ? 2 : 1;
                const bool wide = kG && sC.n_layout > kListNarrowSlots;  // endpoints as (a, b) word pairs
                list_iterations<kItems, kG>(iters, sC.n_runs, reinterpret_cast<const int4*>(sC.runs), sP.hs * sP.hs,
                                            pos, rest, ends, U, wide, tid, T);
                return;
            }
        }
        // Float4 positions on one CTA: the colour loop out of line (float arrays measured slower
        // that way and stay inline).
        if constexpr (CL == 1 && !kG && !kS) {
            constexpr int kItems = kMaxThreads <= 512 ? 2 : 1;
            grid_iterations<kItems>(iters, sC.n_colours, seg4, sC.rank[0].colour_seg, sP.alpha, pos, RG, U, n_local, tid, T,
                                    sC.sync_mask);
            return;
        }
        const int n_colours = sC.n_colours;
        const uint32_t cross = sC.cross_mask;
        // one CTA: a clear bit joins colour c and c + 1 into one phase (disjoint particles)
        const uint32_t sync_mask = CL == 1 ? sC.sync_mask : 0xffffffffu;
        // The thread's items continue from segment to segment (items t, t + T, ... of the
        // phase's segments end to end), so every thread gets the floor or the ceiling of its
        // share, however the items split into segments.
        int i0 = tid;
        for (int it = 0; it < iters; ++it) {
            for (int c = 0; c < n_colours; ++c) {
                const float alpha = sP.alpha[c];
                const int se = sC.rank[rank].colour_seg[c + 1];
                for (int sg = sC.rank[rank].colour_seg[c]; sg < se; ++sg) {
                    const int4 h0 = seg4[2 * sg], h1 = seg4[2 * sg + 1];
                    constexpr int kItems = kMaxThreads <= 512 ? 2 : 1;
                    if constexpr (kS) {
                        if (pos.w_hbm) {
                            if (h1.w >= 0) project_segment_soa<true, true, kItems>(pos, RG + h1.z, U + h1.w, h0, h1, alpha, i0, T);
                            else project_segment_soa<true, false, kItems>(pos, RG + h1.z, U, h0, h1, alpha, i0, T);
                        } else {
                            if (h1.w >= 0) project_segment_soa<false, true, kItems>(pos, RG + h1.z, U + h1.w, h0, h1, alpha, i0, T);
                            else project_segment_soa<false, false, kItems>(pos, RG + h1.z, U, h0, h1, alpha, i0, T);
                        }
                    } else if (h1.w >= 0) {
                        project_segment<CL, true, kItems>(pos, pos_next, RG + h1.z, U + h1.w, n_local, h0, h1, alpha, i0, T);
                    } else {
                        project_segment<CL, false, kItems>(pos, pos_next, RG + h1.z, U, n_local, h0, h1, alpha, i0, T);
                    }
                }
                // Colours that join rows need every rank to see the others' writes; a pair
                // of row-local colours only needs this CTA's. The last colour always syncs
                // the cluster: the tether stage reads anchors anywhere in the cloth.
                const int cn = (c + 1 < n_colours) ? c + 1 : 0;
                const bool last = it + 1 == iters && c + 1 == n_colours;
                if (CL > 1 && (((cross >> c) | (cross >> cn)) & 1u || last)) {
                    cluster_or_block_sync<CL>();
                    i0 = tid;
                } else if ((sync_mask >> c) & 1u) {
                    __syncthreads();
                    i0 = tid;
                }
            }
        }
    };
    // Max relative strain of the stretch-list constraints, max |len / rest - 1|, over the whole
    // cloth (every rank gets the same value).
    auto stretch_residual = [&]() -> float {
        float r = 0.0f;
        const uint32_t smask = sC.stretch_mask;
        for (int c = 0; c < sC.n_colours; ++c) {
            if (!((smask >> c) & 1u)) continue;
            const int se = sC.rank[rank].colour_seg[c + 1];
            for (int sg = sC.rank[rank].colour_seg[c]; sg < se; ++sg) {
                const int4 h0 = seg4[2 * sg], h1 = seg4[2 * sg + 1];
                const int count = h0.x, per_row = h0.z, a_base = h0.w;
                const uint32_t magic = static_cast<uint32_t>(h0.y);
                const int row_stride = h1.x, d = h1.y;
                const float* rr = RG + h1.z;
                for (int i = tid; i < count; i += T) {
                    const int row = seg_row(i, magic);
                    const int la = a_base + row * row_stride + (i - row * per_row), lb = la + d;
                    const float4 pa = pos[la];
                    const float4 pb = (CL == 1 || lb < n_local) ? pos[lb] : pos_next[lb - n_local];
                    const float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
                    const float len = sqrtf(dx * dx + dy * dy + dz * dz);
                    r = fmaxf(r, fabsf(len / rr[i] - 1.0f));
                }
            }
        }
        r = warp_max(r);
        if ((tid & 31) == 0) s_red[tid >> 5][0] = r;
        __syncthreads();
        if (tid == 0) {
            float m = s_red[0][0];
            for (int w = 1; w < ((T + 31) >> 5); ++w) m = fmaxf(m, s_red[w][0]);
            for (int q = 0; q < n_ranks; ++q) {
                float* dst = &s_resid[rank];
                if constexpr (CL > 1) dst = cg::this_cluster().map_shared_rank(&s_resid[rank], q);
                *dst = m;
            }
        }
        cluster_or_block_sync<CL>();
        float m = s_resid[0];
        for (int q = 1; q < n_ranks; ++q) m = fmaxf(m, s_resid[q]);
        cluster_or_block_sync<CL>();  // s_red / s_resid free again
        return m;
    };
    float w_resid = 0.0f;  // max residual over the step's substeps
    int w_fallbacks = 0;
    int w_extra = 0;       // iterations run after the warm ones

    const int steps = sP.steps;
    float4* __restrict__ gvel = sC.vel;
    float4* __restrict__ gprv = sC.prv;
    for (int step = 0; step < steps; ++step) {
        const bool list = kExt && CL == 1 && sC.topology != 0;
        const bool aero = sP.aero != 0 && (sC.aero_grid != 0 || list);
        // --- 1. aerodynamics: gather the shares of the incident triangles -----------------
        // Velocities are parked in U (SoA) for the neighbour reads; each particle's summed
        // share is parked in its own prv slot until integrate consumes it.
        if (aero) {
            if constexpr (!kL) {  // a lean cloth reads the velocities in place
                for (int l = tid; l < n_local; l += T) {
                    const float4 vv = gvel[base + l];
                    U[l] = vv.x;
                    U[n_local + l] = vv.y;
                    U[2 * n_local + l] = vv.z;
                }
            }
            cluster_or_block_sync<CL>();
            const int Q = sC.Q, S = sC.S, cols = sC.columns, rows = sC.rows;
            const f3 wind = mk(sP.wind[0], sP.wind[1], sP.wind[2]);
            const float drag = sP.air_drag, lift = sP.air_lift;
            if (list) {
                // general topology: a slot's triangles from the triangle index, ascending
                for (int l = tid; l < n_local; l += T) {
                    const int e0 = __ldg(&sC.tri_off[l]), e1 = __ldg(&sC.tri_off[l + 1]);
                    f3 a = mk(0.0f, 0.0f, 0.0f);
                    for (int k = e0; k < e1; ++k) {
                        const int4 t = __ldg(&sC.tri_ent[k]);
                        tri_share(xyz(pos[t.x]), xyz(pos[t.y]), xyz(pos[t.z]),
                                  mk(U[t.x], U[n_local + t.x], U[2 * n_local + t.x]),
                                  mk(U[t.y], U[n_local + t.y], U[2 * n_local + t.y]),
                                  mk(U[t.z], U[n_local + t.z], U[2 * n_local + t.z]), wind, drag, lift, a);
                    }
                    gprv[l] = make_float4(a.x, a.y, a.z, 0.0f);
                }
            } else {
            // neighbour rows may belong to the previous / next rank
            auto P3 = [&](int g) -> f3 {
                const int l = g - base;
                if (CL == 1 || (l >= 0 && l < n_local)) return xyz(pos[l]);
                if (l < 0) return xyz(prv_rank.pos[l + prv_rank.n_local]);
                return xyz(nxt_rank.pos[l - n_local]);
            };
            auto V3 = [&](int g) -> f3 {
                if constexpr (kL) return xyz(gvel[g]);
                const int l = g - base;
                if (CL == 1 || (l >= 0 && l < n_local)) return mk(U[l], U[n_local + l], U[2 * n_local + l]);
                if (l < 0) {
                    const int m = l + prv_rank.n_local, n = prv_rank.n_local;
                    return mk(prv_rank.U[m], prv_rank.U[n + m], prv_rank.U[2 * n + m]);
                }
                const int m = l - n_local, n = nxt_rank.n_local;
                return mk(nxt_rank.U[m], nxt_rank.U[n + m], nxt_rank.U[2 * n + m]);
            };
            for (int l = tid; l < n_local; l += T) {
                const int gl = base + l;
                const int y = gl / S;
                const int j = gl - y * S;
                const int cls = j / Q;
                const int x = 4 * (j - cls * Q) + cls;
                if (x >= cols || y >= rows) continue;  // ghost slot
                const bool xm = x >= 1, xp = x + 1 < cols, ym = y >= 1, yp = y + 1 < rows;
                const f3 p00 = xyz(pos[l]);
                const f3 v00 = kL ? xyz(gvel[gl]) : mk(U[l], U[n_local + l], U[2 * n_local + l]);
                f3 a = mk(0.0f, 0.0f, 0.0f);
                if (xm && ym) {  // cell (x-1, y-1): T0 then T1
                    const int lmm = lay(x - 1, y - 1, Q, S), l0m = lay(x, y - 1, Q, S),
                              lm0 = lay(x - 1, y, Q, S);
                    tri_share(P3(lmm), P3(l0m), p00, V3(lmm), V3(l0m), v00, wind, drag, lift, a);
                    tri_share(P3(lmm), p00, P3(lm0), V3(lmm), v00, V3(lm0), wind, drag, lift, a);
                }
                if (xp && ym) {  // cell (x, y-1): T1
                    const int l0m = lay(x, y - 1, Q, S), lp0 = lay(x + 1, y, Q, S);
                    tri_share(P3(l0m), P3(lp0), p00, V3(l0m), V3(lp0), v00, wind, drag, lift, a);
                }
                if (xm && yp) {  // cell (x-1, y): T0
                    const int lm0 = lay(x - 1, y, Q, S), l0p = lay(x, y + 1, Q, S);
                    tri_share(P3(lm0), p00, P3(l0p), V3(lm0), v00, V3(l0p), wind, drag, lift, a);
                }
                if (xp && yp) {  // cell (x, y): T0 then T1
                    const int lp0 = lay(x + 1, y, Q, S), lpp = lay(x + 1, y + 1, Q, S),
                              l0p = lay(x, y + 1, Q, S);
                    tri_share(p00, P3(lp0), P3(lpp), v00, V3(lp0), V3(lpp), wind, drag, lift, a);
                    tri_share(p00, P3(lpp), P3(l0p), v00, V3(lpp), V3(l0p), wind, drag, lift, a);
                }
                gprv[gl] = make_float4(a.x, a.y, a.z, 0.0f);
            }
            }
            cluster_or_block_sync<CL>();
        }

        // --- 4a. lambda reset (cloth_solver.h:253-254); the warm-start path resets after
        // the network, whose tiles borrow the lambda region ----------------------------------
        if constexpr (!kWarm)
            for (int i = tid; i < sC.rank[rank].n_lam; i += T) U[i] = 0.0f;

        // --- 2 + 3. integrate, then the anchor lerp (cloth_solver.h:230-250) --------------
        {
            const float alpha_t = static_cast<float>(step + 1) / static_cast<float>(steps);
            const float hs = sP.hs, damping_factor = sP.damping_factor;
            const f3 base_accel = mk(s_base[0], s_base[1], s_base[2]);
            const PxbAnchorRec* anchors = reinterpret_cast<const PxbAnchorRec*>(sC.anchors);
            for (int l = tid; l < n_local; l += T) {
                const int gl = base + l;
                float4 p = pos[l];
                const f3 acc = aero ? xyz(gprv[gl]) : mk(0.0f, 0.0f, 0.0f);
                gprv[gl] = make_float4(p.x, p.y, p.z, 0.0f);
                if (p.w != 0.0f) {
                    f3 vv = xyz(gvel[gl]);
                    vv = add(vv, mul(add(base_accel, mul(acc, p.w)), hs));
                    vv = mul(vv, damping_factor);
                    p.x = p.x + vv.x * hs;
                    p.y = p.y + vv.y * hs;
                    p.z = p.z + vv.z * hs;
                }
                const int anc = __ldg(&sC.anchor_of[gl]);
                if (anc >= 0) {
                    const PxbAnchorRec& a = anchors[anc];
                    const float om = 1.0f - alpha_t;
                    p.x = a.prev[0] * om + a.world[0] * alpha_t;
                    p.y = a.prev[1] * om + a.world[1] * alpha_t;
                    p.z = a.prev[2] * om + a.world[2] * alpha_t;
                }
                pos[l] = p;
            }
        }
        cluster_or_block_sync<CL>();

        // --- 4b. constraint iterations: colour by colour (cloth_solver.h:256-271) ----------
        // Per segment the descriptor is read once. An item's `a` endpoint is local; its `b`
        // endpoint is local or in the next rank. A zero-compliance colour keeps no lambda: with
        // alpha == 0 the multiplier never reaches a position (dlambda = (-c - 0*lambda)/w); only
        // the sign of an exactly-zero correction could differ, which moves no coordinate that
        // is not itself +-0.
        if constexpr (!kWarm) {
            iterate(sP.iters);
        } else {
            // --- warm start: network displacement, a few iterations, residual, fallback ---
            const PxbWarmStep& W = wsteps[slot];
            const int warm_iters = W.warm_iters;
            const bool rec = W.record != 0 && step == W.record_substep;
            const bool net = warm_iters > 0 && mlp_blob != nullptr;
            float4* __restrict__ gpos = sC.pos;
            // the prediction goes to HBM: the fallback restarts from it, targets are measured from it
            for (int l = tid; l < n_local; l += T) gpos[base + l] = pos[l];
            // The features are read from HBM and the network borrows all of shared memory
            // (positions, rest lengths and the lambda region, staged again after it; the lambdas
            // are reset after it anyway), so every warpgroup the block has can run tiles, not
            // only those whose tiles fit beside the positions. Every rank's prediction is in HBM
            // before any feature is read or any scratch written.
            if (net || rec) cluster_or_block_sync<CL>();
            if (net || rec) {
                uint32_t dyn;
                asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
                unsigned char* ub = smem;
                const int u_cap = static_cast<int>(dyn);
                int n_wg = (u_cap - kWarmTileOff) / kWarmTileBytes;
                n_wg = n_wg < T / 128 ? n_wg : T / 128;
                n_wg = n_wg < kWarmGroups ? n_wg : kWarmGroups;
                if (n_wg < 1) {
                    if (tid == 0) atomicOr(err, PXB_DEVERR_BAD_INDEX);
                } else {
                    if (net) {
                        for (int i = tid; i < kMlpBlobBytes / 16; i += T)
                            reinterpret_cast<uint4*>(ub)[i] = reinterpret_cast<const uint4*>(mlp_blob)[i];
                        if (tid < 32) tc::tmem_alloc(&s_tmem, n_wg > 2 ? 256u : (n_wg > 1 ? 128u : 64u));
                    }
                    tc::fence_before_sync();
                    __syncthreads();
                    tc::fence_after_sync();
                    const int g = tid >> 7;
                    if (g < n_wg) {
                        const int wt = tid & 127;
                        MlpSmem S;
                        S.w = ub;
                        S.f = reinterpret_cast<const float*>(ub + kMlpWBytes);
                        S.a = ub + kWarmTileOff + g * kWarmTileBytes;
                        S.h = S.a;
                        S.bar = &s_wbar[g];
                        S.tmem = s_tmem + 64u * static_cast<uint32_t>(g);
                        const int Q = sC.Q, S_ = sC.S, cols = sC.columns, rows = sC.rows, nl = sC.n_layout;
                        bool mma_ok = true;
                        for (int t = g; t * 128 < n_local; t += n_wg) {
                            const int l = t * 128 + wt;
                            float x[kMlpIn];
                            for (int k = 0; k < kMlpIn; ++k) x[k] = 0.0f;
                            const int gl = base + l;
                            if (l < n_local) {
                                const int y = gl / S_;
                                const int j = gl - y * S_;
                                const int cls = j / Q;
                                const int xx = 4 * (j - cls * Q) + cls;
                                if (xx < cols && y < rows) {
                                    const float4 p = gpos[gl];
                                    const float4 q0 = gprv[gl], v = gvel[gl];
                                    x[0] = p.x - q0.x; x[1] = p.y - q0.y; x[2] = p.z - q0.z;
                                    x[3] = v.x; x[4] = v.y; x[5] = v.z;
                                    const int dxs[6] = {1, -1, 0, 0, 1, -1}, dys[6] = {0, 0, 1, -1, 1, -1};
#pragma unroll
                                    for (int e = 0; e < 6; ++e) {
                                        const int nx = xx + dxs[e], ny = y + dys[e];
                                        const float r = __ldg(&sC.edge_rest[e * nl + gl]);
                                        if (nx < 0 || ny < 0 || nx >= cols || ny >= rows || !(r > 0.0f)) continue;
                                        const float4 q = gpos[lay(nx, ny, Q, S_)];
                                        const float ex = q.x - p.x, ey = q.y - p.y, ez = q.z - p.z;
                                        const float len = sqrtf(ex * ex + ey * ey + ez * ez);
                                        if (len > PXB_EPSILON) {
                                            const float f = 1.0f - __fdividef(r, len);
                                            x[6 + 3 * e] = ex * f; x[7 + 3 * e] = ey * f; x[8 + 3 * e] = ez * f;
                                        }
                                    }
                                }
                                if (rec) {
                                    float* row = W.rec_x + (W.rec_row0 + gl) * kMlpIn;
                                    for (int k = 0; k < kMlpIn; ++k) row[k] = x[k];
                                }
                            }
                            if (net) {
                                mlp_put_input(S, wt, x);
                                float d3[kMlpOut];
                                if (mma_ok) mma_ok = mlp_tile(S, wt, (tid >> 5) & 3, 1 + g, wphase, d3);
                                if (l < n_local)
                                    sC.disp[gl] = make_float4(mma_ok ? d3[0] : 0.0f, mma_ok ? d3[1] : 0.0f,
                                                              mma_ok ? d3[2] : 0.0f, 0.0f);
                            }
                        }
                        if (!mma_ok && wt == 0) atomicOr(err, PXB_DEVERR_MMA_TIMEOUT);
                    }
                    tc::fence_before_sync();
                    __syncthreads();
                    tc::fence_after_sync();
                    if (net && tid < 32) tc::tmem_dealloc(s_tmem, n_wg > 2 ? 256u : (n_wg > 1 ? 128u : 64u));
                }
                if (net) {
                    // the prediction back from HBM (plain loads: this kernel wrote it)
                    __syncthreads();
                    if constexpr (kS) {
                        soa_stage(pos, const_cast<float*>(pos.wt), gpos + base, sC.wtab, sC.n_wtab, err, tid, T);
                    } else {
                        for (int l = tid; l < n_local; l += T) pos[l] = gpos[base + l];
                    }
                }
                if (net && !kL) {
                    // the rest lengths come back: TMA bulk copy, next phase of the staging barrier
                    fence_proxy_async();
                    __syncthreads();
                    if (tid == 0) {
                        const uint32_t rest_bytes = 4u * static_cast<uint32_t>(sC.rank[rank].n_rest_pad);
                        mbar_arrive_expect_tx(&bar, rest_bytes);
                        if (rest_bytes) bulk_g2s(rest, sC.rest + sC.rank[rank].rest_off, rest_bytes, &bar);
                    }
                    stage_phase ^= 1u;
                    if (!mbar_wait_bounded(&bar, stage_phase) && tid == 0) atomicOr(err, PXB_DEVERR_TMA_TIMEOUT);
                }
                // every rank's positions are back before any rank moves a particle (or reads a
                // neighbour's through distributed shared memory)
                cluster_or_block_sync<CL>();
                if (net) {
                    for (int l = tid; l < n_local; l += T) {
                        const int gl = base + l;
                        float4 p = pos[l];
                        if (p.w != 0.0f && __ldg(&sC.anchor_of[gl]) < 0 && gvel[gl].w != 0.0f) {
                            const float4 d = sC.disp[gl];
                            p.x = p.x + d.x; p.y = p.y + d.y; p.z = p.z + d.z;
                            pos[l] = p;
                        }
                    }
                }
            }
            for (int i = tid; i < sC.rank[rank].n_lam; i += T) U[i] = 0.0f;
            cluster_or_block_sync<CL>();
            iterate(net ? warm_iters : sP.iters);
            float r = stretch_residual();
            if (net && r > W.tau) {
                ++w_fallbacks;
                if (W.continue_iters) {
                    // keep iterating from the warm state, warm_iters at a time, until the
                    // residual is within the threshold or the plain count is reached (the
                    // residual is the same on every rank, so every rank loops alike)
                    int done = warm_iters;
                    while (r > W.tau && done < sP.iters) {
                        const int k = warm_iters < sP.iters - done ? warm_iters : sP.iters - done;
                        iterate(k);
                        done += k;
                        w_extra += k;
                        r = stretch_residual();
                    }
                } else {
                    // restart from the unmoved prediction with the plain iteration count
                    for (int l = tid; l < n_local; l += T) pos[l] = gpos[base + l];
                    for (int i = tid; i < sC.rank[rank].n_lam; i += T) U[i] = 0.0f;
                    cluster_or_block_sync<CL>();
                    iterate(sP.iters);
                    w_extra += sP.iters;
                    r = stretch_residual();
                }
            }
            w_resid = fmaxf(w_resid, r);
            if (rec) {
                for (int l = tid; l < n_local; l += T) {
                    const int gl = base + l;
                    const float4 p = pos[l], q = gpos[gl];
                    const bool free = p.w != 0.0f && __ldg(&sC.anchor_of[gl]) < 0 && gvel[gl].w != 0.0f;
                    float* row = W.rec_y + (W.rec_row0 + gl) * 4;
                    row[0] = p.x - q.x; row[1] = p.y - q.y; row[2] = p.z - q.z; row[3] = free ? 1.0f : 0.0f;
                }
            }
        }

        // --- 5 + 7 + 8. tethers, collisions, velocities (owner thread) ---------------------
        {
            const int col_begin = sP.col_begin, col_count = sP.col_count;
            const float thickness = sP.thickness, inv_hs = sP.inv_hs;
            bool self = false;
            if constexpr (kExt && CL == 1 && !kS) {
                self = sP.self_collision != 0;
                if (self) {
                    // 5. tethers on their own: 6. self-collision reads every particle after them
                    for (int l = tid; l < n_local; l += T) {
                        const float4 p4 = pos[l];
                        if (p4.w == 0.0f) continue;
                        const int2 teth = __ldg(&sC.tether[base + l]);
                        if (teth.x < 0) continue;
                        const f3 anchor = xyz(pos[teth.x]);
                        const f3 d = sub(xyz(p4), anchor);
                        const float l2 = len(d);
                        const float max_len = __int_as_float(teth.y);
                        if (!(l2 <= max_len || l2 < PXB_EPSILON)) {
                            const f3 q = add(anchor, mul(d, max_len / l2));
                            pos[l] = make_float4(q.x, q.y, q.z, p4.w);
                        }
                    }
                    __syncthreads();
                    // 6. self-collision (cloth_solver.h:291-366) over tables in shared memory
                    uint32_t* tab = reinterpret_cast<uint32_t*>(smem + sC.self_hash_off);
                    const uint32_t buckets = static_cast<uint32_t>(sC.self_buckets);
                    const float d_min = sP.self_distance;
                    const float inv_cell = 1.0f / d_min;
                    // the tables must be a power-of-two hash after the positions, inside this
                    // launch's shared memory: otherwise record the error and skip the stage
                    uint32_t dyn;
                    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
                    const bool tables_ok =
                        buckets >= 16u && (buckets & (buckets - 1u)) == 0u && sC.self_hash_off >= 16 * n_local &&
                        (sC.self_hash_off & 15) == 0 &&
                        static_cast<uint64_t>(sC.self_hash_off) +
                                4ull * PXB_SELF_WORDS(static_cast<uint64_t>(buckets), static_cast<uint64_t>(sC.n_real)) <=
                            dyn;
                    if (!tables_ok) {
                        if (tid == 0) atomicOr(err, PXB_DEVERR_BAD_INDEX);
                    } else {
                        self_build_hash(pos, tab, sC.n_real, sC.columns, sC.Q, sC.S, buckets, inv_cell, tid, T);
                        if (tid < 32)
                            self_pair_pass(pos, tab, sC.n_real, sC.columns, sC.ref_columns, sC.Q, sC.S, buckets, d_min,
                                           inv_cell, tid);
                    }
                    __syncthreads();
                    if (sC.self_restage) {
                        // the tables borrowed the rest lengths' bytes: stage them again
                        fence_proxy_async();
                        __syncthreads();
                        if (tid == 0) {
                            const uint32_t rest_bytes = 4u * static_cast<uint32_t>(sC.rank[0].n_rest_pad);
                            mbar_arrive_expect_tx(&bar, rest_bytes);
                            if (rest_bytes) bulk_g2s(rest, sC.rest + sC.rank[0].rest_off, rest_bytes, &bar);
                        }
                        stage_phase ^= 1u;
                        if (!mbar_wait_bounded(&bar, stage_phase) && tid == 0) atomicOr(err, PXB_DEVERR_TMA_TIMEOUT);
                        __syncthreads();
                    }
                }
            }
            for (int l = tid; l < n_local; l += T) {
                const int gl = base + l;
                float4 p4 = pos[l];
                f3 p = xyz(p4);
                bool moved = false;
                f3 nsum = mk(0.0f, 0.0f, 0.0f);
                float dsum = 0.0f;
                if (p4.w != 0.0f) {
                    // 5. tether (cloth_solver.h:276-289); its anchor is a pinned particle
                    const int2 teth = self ? make_int2(-1, 0) : __ldg(&sC.tether[gl]);
                    if (teth.x >= 0) {
                        f3 anchor;
                        if (CL == 1) {
                            anchor = xyz(pos[teth.x]);
                        } else {
                            int o = 0;
                            while (o + 1 < n_ranks && teth.x >= sC.rank[o + 1].row0 * sC.S) ++o;
                            const RankView ov = o == rank ? me : rank_view<CL>(sC, smem, o);
                            anchor = xyz(ov.pos[teth.x - ov.base]);
                        }
                        const f3 d = sub(p, anchor);
                        const float l2 = len(d);
                        const float max_len = __int_as_float(teth.y);
                        if (!(l2 <= max_len || l2 < PXB_EPSILON)) {
                            p = add(anchor, mul(d, max_len / l2));
                            moved = true;
                        }
                    }
                    // 7. colliders in list order (cloth_solver.h:379-410)
                    for (int k = 0; k < col_count; ++k) {
                        const PxbDevCollider* c = &colliders[col_begin + k];
                        if (p.x < __ldg(&c->bmin[0]) - thickness || p.x > __ldg(&c->bmax[0]) + thickness ||
                            p.y < __ldg(&c->bmin[1]) - thickness || p.y > __ldg(&c->bmax[1]) + thickness ||
                            p.z < __ldg(&c->bmin[2]) - thickness || p.z > __ldg(&c->bmax[2]) + thickness) {
                            continue;
                        }
                        f3 n = mk(0.0f, 0.0f, 0.0f);
                        float depth = 0.0f;
                        // a mesh's swept test starts from the substep's start (cloth_solver.h:398-403)
                        const bool mesh = kExt && __ldg(&c->type) == PXB_SHAPE_TRIANGLE_MESH;
                        const f3 start = mesh ? xyz(gprv[gl]) : p;
                        if (!project_particle<kExt>(c, thickness, p, n, depth, start, mesh)) continue;
                        moved = true;
                        nsum = add(nsum, n);
                        dsum += depth;
                    }
                }
                if (moved) {
                    p4.x = p.x; p4.y = p.y; p4.z = p.z;
                    pos[l] = p4;
                }
                // 8. finalize (cloth_solver.h:414-451), every particle
                const float4 pv = gprv[gl];
                f3 vv = mul(sub(p, xyz(pv)), inv_hs);
                if (dsum > 0.0f) {
                    const float nlen = len(nsum);
                    if (nlen > PXB_EPSILON) {
                        const f3 nrm = divs(nsum, nlen);
                        const float vn = dot(vv, nrm);
                        const f3 vt = sub(vv, smul(vn, nrm));
                        if (vn < 0.0f) vv = sub(vv, smul(vn, nrm));
                        const float budget = sP.friction * dsum * inv_hs;
                        const float vt_len = len(vt);
                        if (vt_len > PXB_EPSILON) vv = sub(vv, mul(vt, minr(1.0f, budget / vt_len)));
                    }
                }
                const float v2 = dot(vv, vv);
                if (v2 > sP.max_velocity2) vv = mul(vv, sP.max_velocity / sqrtf(v2));
                const float real = gvel[gl].w;
                gvel[gl] = make_float4(vv.x, vv.y, vv.z, real);
            }
        }
        cluster_or_block_sync<CL>();
    }

    // --- epilogue --------------------------------------------------------------------------
    // One CTA: a bulk copy back to HBM (its own threads wrote every slot, then fenced). A
    // cluster rank's slots were also written by its neighbour through distributed shared
    // memory, so it stores with plain coalesced writes instead of the async proxy.
    if constexpr (kG) {
        // the positions never left HBM
    } else if constexpr (kS) {
        for (int l = tid; l < n_local; l += T) sC.pos[base + l] = pos[l];
    } else if constexpr (CL == 1) {
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            bulk_s2g(sC.pos + base, pos, 16u * static_cast<uint32_t>(n_local));
            bulk_commit_and_wait();
        }
    } else {
        for (int l = tid; l < n_local; l += T) sC.pos[base + l] = pos[l];
    }
    float bmin[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float bmax[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    float vmax2 = 0.0f;
    for (int l = tid; l < n_local; l += T) {
        const float4 vv = gvel[base + l];
        if (vv.w == 0.0f) continue;  // ghost slot
        const float4 p = pos[l];
        bmin[0] = minr(bmin[0], p.x); bmin[1] = minr(bmin[1], p.y); bmin[2] = minr(bmin[2], p.z);
        bmax[0] = maxr(bmax[0], p.x); bmax[1] = maxr(bmax[1], p.y); bmax[2] = maxr(bmax[2], p.z);
        vmax2 = maxr(vmax2, dot(xyz(vv), xyz(vv)));
    }
    if (sP.write_lambdas) {
        float* lo = sC.lam_out + sC.rank[rank].lam_off;
        for (int i = tid; i < sC.rank[rank].n_lam; i += T) lo[i] = U[i];
    }
    if (rank == 0) {
        for (int a = tid; a < sC.n_anchors; a += T) {
            PxbAnchorRec* rec = reinterpret_cast<PxbAnchorRec*>(sC.anchors) + a;
            rec->prev[0] = rec->world[0];
            rec->prev[1] = rec->world[1];
            rec->prev[2] = rec->world[2];
        }
    }
    float r[7] = {bmin[0], bmin[1], bmin[2], bmax[0], bmax[1], bmax[2], vmax2};
    r[0] = warp_min(r[0]); r[1] = warp_min(r[1]); r[2] = warp_min(r[2]);
    r[3] = warp_max(r[3]); r[4] = warp_max(r[4]); r[5] = warp_max(r[5]);
    r[6] = warp_max(r[6]);
    if ((tid & 31) == 0) {
        for (int k = 0; k < 7; ++k) s_red[tid >> 5][k] = r[k];
    }
    __syncthreads();
    if (tid == 0) {
        const int nw = (T + 31) >> 5;
        for (int w = 1; w < nw; ++w) {
            for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], s_red[w][k]);
            for (int k = 3; k < 7; ++k) r[k] = fmaxf(r[k], s_red[w][k]);
        }
        float* dst = s_rank_red[rank];
        if constexpr (CL > 1) dst = cg::this_cluster().map_shared_rank(&s_rank_red[rank][0], 0);
        for (int k = 0; k < 7; ++k) dst[k] = r[k];
    }
    cluster_or_block_sync<CL>();
    if (rank == 0 && tid == 0) {
        for (int q = 1; q < n_ranks; ++q) {
            for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], s_rank_red[q][k]);
            for (int k = 3; k < 7; ++k) r[k] = fmaxf(r[k], s_rank_red[q][k]);
        }
        if constexpr (kWarm) {
            PxbWarmResult* wr = &wres[slot];
            wr->residual = w_resid;
            wr->fallbacks = w_fallbacks;
            wr->substeps = sP.steps;
            wr->extra_iterations = w_extra;
        }
        PxbFrameResult* out = &results[slot];
        for (int k = 0; k < 3; ++k) { out->bounds_min[k] = r[k]; out->bounds_max[k] = r[k + 3]; }
        out->max_speed = sqrtf(r[6]);
        out->time = 0.0f;
    }
    // no rank leaves (or takes the next cloth) while its memory is read; no thread overwrites
    // the cloth's shared state before every thread is done with it
    cluster_or_block_sync<CL>();
    }  // cloth loop
}

template <int kMaxThreads, int CL, bool kWarm, bool kExt, bool kGmem = false, int kLean = 0>
static cudaError_t launch_variant(const PxbClothDev* cloths, const PxbClothStep* steps,
                                  const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                                  const int32_t* order, PxbFrameResult* results, uint32_t* err,
                                  int n_cloths, int threads, int smem_bytes, cudaStream_t stream,
                                  const PxbWarmStep* wsteps, const unsigned char* mlp, PxbWarmResult* wres,
                                  int* queue, int persistent_units) {
    static uint64_t configured = 0;  // one bit per device the attributes have been set on
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured >> dev & 1ull)) {
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, cloth_step_kernel<kMaxThreads, CL, kWarm, kExt, kGmem, kLean>);
        if (e != cudaSuccess) return e;
        if (fa.sharedSizeBytes > static_cast<size_t>(kClothStaticSmem)) return cudaErrorInvalidConfiguration;
        e = cudaFuncSetAttribute(cloth_step_kernel<kMaxThreads, CL, kWarm, kExt, kGmem, kLean>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
        if (e != cudaSuccess) return e;
        configured |= 1ull << dev;
    }
    // one CTA (cluster) per cloth, or persistent_units of them popping cloths from `queue`
    const bool persistent = queue != nullptr && persistent_units > 0 && persistent_units < n_cloths;
    const int units = persistent ? persistent_units : n_cloths;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(units * CL));
    cfg.blockDim = dim3(static_cast<unsigned>(threads));
    cfg.dynamicSmemBytes = static_cast<size_t>(smem_bytes);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, cloth_step_kernel<kMaxThreads, CL, kWarm, kExt, kGmem, kLean>, cloths, steps, colliders,
                              sources, order, results, err, wsteps, mlp, wres, persistent ? queue : nullptr, n_cloths);
}

template <int kMaxThreads, bool kWarm, bool kExt>
static cudaError_t launch_cl(int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                             const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                             const int32_t* order, PxbFrameResult* results, uint32_t* err,
                             int n_cloths, int threads, int smem_bytes, cudaStream_t stream,
                             const PxbWarmStep* wsteps, const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    switch (cluster) {
        case 1: return launch_variant<kMaxThreads, 1, kWarm, kExt>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 2: return launch_variant<kMaxThreads, 2, kWarm, kExt>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 4: return launch_variant<kMaxThreads, 4, kWarm, kExt>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 8: return launch_variant<kMaxThreads, 8, kWarm, kExt>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        default: return cudaErrorInvalidValue;
    }
}

// Launch families (one translation unit each).
cudaError_t launch_cloth_plain(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);
cudaError_t launch_cloth_warm(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);
cudaError_t launch_cloth_geo(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);
cudaError_t launch_cloth_lean(bool ext, int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);
cudaError_t launch_cloth_soa(bool ext, int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                             const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                             const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                             int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                             const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);
cudaError_t launch_cloth_gmem(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units);

}  // namespace pxb

#endif  // PXB_CLOTH_STEP_CUH
