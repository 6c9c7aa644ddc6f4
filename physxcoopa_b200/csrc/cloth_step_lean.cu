// cloth_step_lean.cu -- launches of the lean cloth-step kernels: positions alone in shared
// memory, rest lengths and lambdas read in place in HBM, on one CTA or a 2-CTA cluster.
#include "cloth_step.cuh"

namespace pxb {

// Launches carrying a mesh or hull collider: the same dispatch over the kExt instantiations.
// Lean cloths: one CTA or a 2-CTA cluster, plain / extended, plain / warm-start kernels.
template <int kMaxThreads, bool kWarm, bool kExt>
static cudaError_t launch_lean_cl(int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                                  const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                                  const int32_t* order, PxbFrameResult* results, uint32_t* err,
                                  int n_cloths, int threads, int smem_bytes, cudaStream_t stream,
                                  const PxbWarmStep* wsteps, const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    switch (cluster) {
        case 1: return launch_variant<kMaxThreads, 1, kWarm, kExt, false, true>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 2: return launch_variant<kMaxThreads, 2, kWarm, kExt, false, true>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        default: return cudaErrorInvalidValue;
    }
}

template <bool kExt>
static cudaError_t launch_lean_family(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                               const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                               const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                               int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                               const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (wsteps) {
        if (variant == 0) {
            if (threads > 512) threads = 512;
            return launch_lean_cl<512, true, kExt>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        }
        if (threads > 1024) threads = 1024;
        if (threads < 128) threads = 128;
        return launch_lean_cl<1024, true, kExt>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
    if (threads > cloth_variant_threads(variant)) threads = cloth_variant_threads(variant);
    switch (variant) {
        case 0: return launch_lean_cl<512, false, kExt>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        case 1: return launch_lean_cl<768, false, kExt>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        default: return launch_lean_cl<1024, false, kExt>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
    }
}

cudaError_t launch_cloth_lean(bool ext, int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    return ext ? launch_lean_family<true>(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units)
               : launch_lean_family<false>(variant, cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
}

}  // namespace pxb
