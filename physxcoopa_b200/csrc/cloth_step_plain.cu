// cloth_step_plain.cu -- launches of the plain cloth-step kernels (grid cloths, sphere /
// capsule / box colliders, no warm start) on one CTA or a 2/4/8-CTA cluster.
#include "cloth_step.cuh"

namespace pxb {

cudaError_t launch_cloth_plain(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (threads > cloth_variant_threads(variant)) threads = cloth_variant_threads(variant);
    switch (variant) {
        case 0: return launch_cl<512, false, false>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        case 1: return launch_cl<768, false, false>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
        default: return launch_cl<1024, false, false>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
}

int cloth_variant_registers(int variant) {
    static int regs[kClothVariants] = {0, 0, 0};
    const int v = variant < 0 ? 0 : (variant >= kClothVariants ? kClothVariants - 1 : variant);
    if (!regs[v]) {
        cudaFuncAttributes fa;
        cudaError_t e = v == 0 ? cudaFuncGetAttributes(&fa, cloth_step_kernel<512, 1, false, false>)
                               : (v == 1 ? cudaFuncGetAttributes(&fa, cloth_step_kernel<768, 1, false, false>)
                                         : cudaFuncGetAttributes(&fa, cloth_step_kernel<1024, 1, false, false>));
        regs[v] = e == cudaSuccess ? fa.numRegs : 255;
    }
    return regs[v];
}

}  // namespace pxb
