// cloth_step_geo.cu -- launches of the extended cloth-step kernels: mesh and convex-hull
// colliders, self-collision and general-topology cloths in shared memory.
#include "cloth_step.cuh"

namespace pxb {

cudaError_t launch_cloth_geo(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (wsteps) {
        if (variant == 0) {
            if (threads > 512) threads = 512;
            return launch_cl<512, true, true>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        }
        if (threads > 1024) threads = 1024;
        if (threads < 128) threads = 128;
        return launch_cl<1024, true, true>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
    if (threads > cloth_variant_threads(variant)) threads = cloth_variant_threads(variant);
    switch (variant) {
        case 0: return launch_cl<512, false, true>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        case 1: return launch_cl<768, false, true>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        default: return launch_cl<1024, false, true>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
    }
}

}  // namespace pxb
