// gr_batch_classes.cu -- the batched trace grids specialised by scene class: clear
// isotropic stones and the general (birefringent or absorbing) ones, each per
// environment kind, as the single-scene kernels are (gr_single_clear.cu,
// gr_single_general.cu).  A batched launch holds segments of one class only.
#include "gr_batch.cuh"
#include "gr_ctx.h"

// Resident blocks per SM of the class-specialised batched grids.  Measured on B200
// with the c4 stones (batched path-samples/s at film scales 1/32 and 1/8): 9 blocks
// 328 M / 428 M, 16 blocks 311 M / 405 M (another run: 9, 10, 12 blocks 350 / 350 /
// 345 M and 448 / 447 / 443 M) -- unlike the single-scene kernels, these
// grids lose more to their spills (the scene constants come from shared memory) than
// they gain from the extra warps.
#ifndef GR_BATCH_MIN_BLOCKS
#define GR_BATCH_MIN_BLOCKS 9
#endif

namespace grh {

gr_status launch_batch_class(int K, const grd::SceneSlot *slots, const grd::BatchSegment *segs, uint32_t n_segs,
                             grd::Path *park, unsigned int *counts, uint64_t blocks, uint64_t park_blocks, size_t smem,
                             cudaStream_t s) {
    constexpr int IC = grd::K_ISO | grd::K_CLEAR;
    constexpr int MB = GR_BATCH_MIN_BLOCKS;
#define GR_BATCH_CASE(KK)                                                                                       \
    case KK:                                                                                                    \
        grd::launch_batch_grids<false, KK, MB>(slots, segs, n_segs, park, counts, blocks, park_blocks, smem, s); \
        break;
    switch (K) {
        GR_BATCH_CASE(IC | grd::k_env(GR_ENV_UNIFORM))
        GR_BATCH_CASE(IC | grd::k_env(GR_ENV_STUDIO))
        GR_BATCH_CASE(IC | grd::k_env(GR_ENV_LATLONG))
        GR_BATCH_CASE(grd::k_env(GR_ENV_UNIFORM))
        GR_BATCH_CASE(grd::k_env(GR_ENV_STUDIO))
        GR_BATCH_CASE(grd::k_env(GR_ENV_LATLONG))
    default: return fail(GR_EINVAL, "scene class %d has no batched kernels", K);
    }
#undef GR_BATCH_CASE
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

}  // namespace grh
