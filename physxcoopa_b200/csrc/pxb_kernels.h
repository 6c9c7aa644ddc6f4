// pxb_kernels.h -- launch entry points of the device kernels (host side).
#ifndef PXB_KERNELS_H
#define PXB_KERNELS_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/physxcoopa_b200.h"
#include "pxb_internal.h"

namespace pxb {

// Static shared memory the cloth kernel may declare (checked against the compiled kernel before
// its first launch on a device) and the dynamic shared memory left to a cloth CTA under the
// sm_100 per-block limit of 227 KB.
constexpr int kClothStaticSmem = 4608;
constexpr int kMaxDynamicSmem = 232448 - kClothStaticSmem;
// Dynamic shared memory of a lean one-CTA cloth held as float arrays (PxbClothDev::lean 2):
// x, y, z (12 bytes per slot), one inverse-mass index byte per slot padded to 16, the table.
__host__ __device__ constexpr int soa_smem_bytes(int n_local) {
    return 12 * n_local + ((n_local + 15) & ~15) + 4 * PXB_MAX_WTAB;
}
constexpr int kClothOwned = 4;      // particles per thread in the cloth kernel
constexpr int kClothMaxThreads = 1024;

// Kernel variants differ in their block-size cap (and so their register budget): 0 = 512
// threads (no spills), 1 = 768, 2 = 1024.
constexpr int kClothVariants = 3;
int cloth_variant_threads(int variant);
// Registers per thread of a variant's one-CTA kernel (read from the compiled kernel once).
int cloth_variant_registers(int variant);
// wsteps non-null selects the warm-start kernel (mlp may then be null: plain solve with the
// residual measured, or recording only). ext: 0 the plain kernel, 1 with the mesh / hull,
// self-collision and general-topology stages, 2 general topology with the state in HBM, 3 and 4
// the lean instantiations of 0 and 1 (rest lengths and lambdas in HBM; one CTA or two).
// queue / persistent_units: with a zeroed counter and a unit count below n_cloths, that many
// CTAs (clusters) stay resident and pop the group's cloths from the counter, largest first;
// else one CTA (cluster) per cloth.
cudaError_t launch_cloth_step(int variant, int cluster, const PxbClothDev* cloths, const PxbClothStep* steps,
                              const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                              const int32_t* order, PxbFrameResult* results, uint32_t* err,
                              int n_cloths, int threads, int smem_bytes, cudaStream_t stream,
                              const PxbWarmStep* wsteps = nullptr, const unsigned char* mlp = nullptr,
                              PxbWarmResult* wres = nullptr, int ext = 0, int* queue = nullptr,
                              int persistent_units = 0);

// Warm-start kernel: network warpgroups per CTA and the shared memory they borrow from the
// lambda region (weights blob, then per warpgroup an input and an activation tile).
// During the network phase the rest lengths and the lambda region together are its scratch
// (the rest lengths are staged again afterwards); a warpgroup's input tile and activation tile
// share their bytes (the first layer's MMAs consume the inputs before the activations are
// written). At most 4 warpgroups: 4 x 64 TMEM columns leave room for a second CTA per SM.
constexpr int kWarmGroups = 4;
constexpr int kWarmTileOff = 15232;      // kMlpBlobBytes rounded up to 128
constexpr int kWarmTileBytes = 16384;    // max(kMlpTileA, kMlpTileH)
constexpr int kWarmUMin = kWarmTileOff + kWarmTileBytes;

// Whole-GPU path for one cloth beyond an 8-CTA cluster: a cooperative launch of one CTA per SM.
cudaError_t launch_cloth_grid(const PxbClothDev* cloths, const PxbClothStep* steps, const PxbDevCollider* colliders,
                              const pxb_gravity_source* sources, const int32_t* order, PxbFrameResult* results,
                              uint32_t* err, PxbGridSync* gs, int slot, int n_sms, cudaStream_t stream,
                              bool geo = false);

// Warm-start network (mlp_kernel.cu).
int mlp_infer_smem_bytes();
cudaError_t launch_mlp_infer(const float* X, int n, const unsigned char* blob, float* Y, uint32_t* err,
                             int n_sms, cudaStream_t stream);
void mlp_pack_blob(const pxb_mlp_weights& m, unsigned char* out);
// Training (mlp_train.cu), on the tensor cores: gradients of `rows` rows given as indices (part of
// an optimiser batch of batch_rows rows) as per-CTA partials in `part` (mlp_partial_floats(n_sms)
// floats); returns the number of CTAs launched (the partials to sum), *status the launch error.
// Adam (or a plain reduce into G) then sums the partials in CTA order.
size_t mlp_partial_floats(int n_sms);
int launch_mlp_grad(const float* X, const float* T, const uint32_t* idx, int rows, int batch_rows,
                    const pxb_mlp_weights* W, float* part, uint32_t* err, int n_sms, cudaStream_t stream,
                    cudaError_t* status);
cudaError_t launch_mlp_adam(const float* part, int n_parts, int n_sms, pxb_mlp_weights* W, pxb_mlp_weights* M,
                            pxb_mlp_weights* V, float lr, float b1t, float b2t, float* loss, cudaStream_t stream);
cudaError_t launch_mlp_reduce(const float* part, int n_parts, int n_sms, pxb_mlp_weights* G, float* loss,
                              cudaStream_t stream);

cudaError_t launch_project_points(const PxbDevCollider* collider, float thickness,
                                  const float* pts, const float* starts, int n, float* out,
                                  float* normals, float* depths, int32_t* hits, cudaStream_t stream);

// Gathers positions of the listed cloths from layout order into particle order, 3 floats per
// particle, cloth after cloth starting at out_offsets[k] (floats).
cudaError_t launch_gather_positions(const PxbClothDev* cloths, const int32_t* order,
                                    const int64_t* out_offsets, int n_cloths, float* out,
                                    cudaStream_t stream);

// geo: the step's colliders include a mesh or hull (selects the kernel with those branches; a
// launch of the cloth kernels takes the same flag).
cudaError_t launch_strand_step(const PxbStrandDev& d, const PxbStrandStep& p,
                               const PxbDevCollider* colliders, const pxb_gravity_source* sources,
                               cudaStream_t stream, bool geo = false);

}  // namespace pxb

#endif  // PXB_KERNELS_H
