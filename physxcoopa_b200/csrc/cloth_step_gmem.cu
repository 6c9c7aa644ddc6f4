// cloth_step_gmem.cu -- launches of the general-topology cloth-step kernel whose state stays
// in HBM (one CTA per cloth, no warm start).
#include "cloth_step.cuh"

namespace pxb {

cudaError_t launch_cloth_gmem(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (cluster != 1 || wsteps) return cudaErrorInvalidValue;
    if (threads > cloth_variant_threads(variant)) threads = cloth_variant_threads(variant);
    switch (variant) {
        case 0: return launch_variant<512, 1, false, true, true>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 1: return launch_variant<768, 1, false, true, true>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        default: return launch_variant<1024, 1, false, true, true>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
}

}  // namespace pxb
