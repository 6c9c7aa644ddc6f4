// cloth_step_soa.cu -- launches of the lean cloth-step kernels whose positions are float arrays
// (PxbClothDev::lean 2): one CTA per cloth, rest lengths and lambdas read in place in HBM.
#include "cloth_step.cuh"

namespace pxb {

template <bool kExt>
static cudaError_t launch_soa_family(int variant, const PxbClothDev* cloths, const PxbClothStep* steps,
                                     const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                                     const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                                     int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                                     const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (wsteps) {
        if (variant == 0) {
            if (threads > 512) threads = 512;
            return launch_variant<512, 1, true, kExt, false, 2>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        }
        if (threads > 1024) threads = 1024;
        if (threads < 128) threads = 128;
        return launch_variant<1024, 1, true, kExt, false, 2>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
    if (threads > cloth_variant_threads(variant)) threads = cloth_variant_threads(variant);
    switch (variant) {
        case 0: return launch_variant<512, 1, false, kExt, false, 2>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        case 1: return launch_variant<768, 1, false, kExt, false, 2>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
        default: return launch_variant<1024, 1, false, kExt, false, 2>(cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, nullptr, nullptr, nullptr, queue, persistent_units);
    }
}

cudaError_t launch_cloth_soa(bool ext, int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                             const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                             const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                             int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                             const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (cluster != 1) return cudaErrorInvalidValue;
    return ext ? launch_soa_family<true>(variant, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units)
               : launch_soa_family<false>(variant, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
}

}  // namespace pxb
