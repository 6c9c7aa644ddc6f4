// cloth_step_warm.cu -- launches of the warm-start cloth-step kernels (the network phase, then
// the iterations, residual and fallback): the 512-thread variant (registers for the network
// epilogue) or the 1024-thread one.
#include "cloth_step.cuh"

namespace pxb {

cudaError_t launch_cloth_warm(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err, int n_cloths,
                              int threads, int smem_bytes, cudaStream_t stream, const PxbWarmStep* wsteps,
                              const unsigned char* mlp, PxbWarmResult* wres, int* queue, int persistent_units) {
    if (variant == 0) {
        if (threads > 512) threads = 512;
        return launch_cl<512, true, false>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
    }
    if (threads > 1024) threads = 1024;
    if (threads < 128) threads = 128;
    return launch_cl<1024, true, false>(cluster, cloths, steps, colliders, sources, order, results, err, n_cloths, threads, smem_bytes, stream, wsteps, mlp, wres, queue, persistent_units);
}

}  // namespace pxb
