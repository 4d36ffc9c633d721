// gr_single.cuh -- launches of the single-scene transport kernels for one scene class K
// (plain, or the three staged launches over park buffers the caller has prepared).
// Included by the translation units that instantiate the specialised classes.
#pragma once

#include "gr_ctx.h"
#include "gr_sorted.cuh"
#include "gr_transport.cuh"

namespace grh {

// The three staged launches at MB blocks per SM.
template <int K, int MB>
gr_status launch_staged_mb(const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R, float *xyz,
                           cudaStream_t stream, const StagedLaunch *st) {
    const size_t smem = grd::planes_smem_bytes(S.n_planes);
    const unsigned blocks = (unsigned)((R.n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
    const grd::ParkOut out1{st->park1, (uint32_t)st->cap1, st->counts};
    const grd::ParkOut out2{st->park2, (uint32_t)st->cap2, st->counts + 1};
    const grd::ParkOut none{nullptr, 0, nullptr};
    const unsigned b2 = (unsigned)((st->cap1 + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
    const unsigned b3 = (unsigned)((st->cap2 + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
    grd::k_trace_stage1<false, K, MB><<<blocks, grd::TRACE_THREADS, smem, stream>>>(S, B, R, xyz, out1, st->cap_first);
    grd::k_trace_stage2<false, K, MB><<<b2, grd::TRACE_THREADS, smem, stream>>>(
        S, B, st->park1, (uint32_t)st->cap1, st->counts, st->cap_second, out2, xyz);
    if (st->cap2)
        grd::k_trace_stage2<false, K, MB><<<b3, grd::TRACE_THREADS, smem, stream>>>(
            S, B, st->park2, (uint32_t)st->cap2, st->counts + 1, 0xFFFFFFFFu, none, xyz);
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

// The plain kernel (st == NULL, at the built-in GR_TRACE_MIN_BLOCKS), or the staged
// launches at the blocks per SM the schedule asks for (kScheduleBlocks; 0 =
// kBuiltinScheduleBlocks).
template <int K>
gr_status launch_single_k(const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R, float *xyz,
                          cudaStream_t stream, const StagedLaunch *st) {
    if (!st) {
        const size_t smem = grd::planes_smem_bytes(S.n_planes);
        const unsigned blocks = (unsigned)((R.n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
        grd::k_trace_plain<grd::NoCounters, false, false, K, GR_TRACE_MIN_BLOCKS>
            <<<blocks, grd::TRACE_THREADS, smem, stream>>>(S, B, R, xyz, nullptr);
        GR_CUDA(cudaGetLastError());
        return GR_OK;
    }
    static_assert(kScheduleBlockCount == 4, "one launch per kScheduleBlocks entry");
    switch (st->blocks ? st->blocks : kBuiltinScheduleBlocks) {
        case kScheduleBlocks[0]: return launch_staged_mb<K, kScheduleBlocks[0]>(S, B, R, xyz, stream, st);
        case kScheduleBlocks[1]: return launch_staged_mb<K, kScheduleBlocks[1]>(S, B, R, xyz, stream, st);
        case kScheduleBlocks[2]: return launch_staged_mb<K, kScheduleBlocks[2]>(S, B, R, xyz, stream, st);
        case kScheduleBlocks[3]: return launch_staged_mb<K, kScheduleBlocks[3]>(S, B, R, xyz, stream, st);
        default: return fail(GR_EINVAL, "no staged kernels for %u blocks per SM", st->blocks);
    }
}

// The block-sorted kernel (gr_sorted.cuh) over a launch's tuples: one block per
// resident slot set (blocks per SM from the occupancy calculator, at most one block per
// SORT_THREADS tuples); `work` is a zeroed counter the blocks claim tuples from.
template <int K>
gr_status launch_sorted_k(const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R, float *xyz,
                          cudaStream_t stream, unsigned int *work, int sm_count) {
    const size_t smem = grd::sorted_smem_bytes(S.n_planes);
    if (smem > 48 * 1024) GR_CUDA(cudaFuncSetAttribute(grd::k_trace_sorted<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem));
    int per_sm = 0;
    GR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grd::k_trace_sorted<K>, grd::SORT_THREADS, smem));
    if (per_sm < 1) return fail(GR_EINVAL, "the sorted kernel does not fit an SM with %u planes", S.n_planes);
    uint64_t blocks = (uint64_t)per_sm * (uint64_t)(sm_count > 0 ? sm_count : 1);
    const uint64_t need = (R.n_tuples + grd::SORT_THREADS - 1) / grd::SORT_THREADS;
    if (blocks > need) blocks = need;
    GR_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned int), stream));
    grd::k_trace_sorted<K><<<(unsigned)blocks, grd::SORT_THREADS, smem, stream>>>(S, B, R, xyz, work);
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

}  // namespace grh
