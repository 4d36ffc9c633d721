// gr_batch.cuh -- batched launches: many scenes (each with its own planes, material,
// environment and film) in one grid.  Included by gr_batch.cu only.
#pragma once

#include "gr_stage.cuh"

namespace grd {

// A segment is one scene's run of whole pixels for one sample
// range; every block of the trace kernel (every warp of the fold kernel) belongs to
// exactly one segment, found by binary search over the segments' first block (warp).
// The scene's constants are copied into shared memory, so per-tuple arithmetic is
// that of the single-scene kernel and results are bit-identical to rendering each
// scene alone.
struct SceneSlot {
    SceneConst S;
    SceneBuffers B;
};

struct BatchSegment {
    LaunchRange R;         // pixels / samples of this segment
    float *xyz;            // its per-tuple XYZ (3 f32 per tuple)
    float *film;           // the scene's film (W*H*3 f32), folded into (fold_pixel)
    float *comp;           // continue mode with Kahan: the film's compensation terms
    uint64_t block_begin;  // first trace block of the segment
    uint64_t warp_begin;   // first fold warp of the segment
    uint32_t scene;        // index into the SceneSlot table
    uint32_t kahan;
    uint32_t cont;         // fold_pixel continue mode
    uint32_t park_cap;     // park slots of this segment (paths alive after the stage cap)
    uint32_t stage_cap;    // stage-1 bounce cap: the scene's chosen one (StageCapTune)
    uint64_t park_off;     // first park slot of this segment in the launch's park buffer
    uint64_t park_block_begin;  // first continuation block of the segment
};

// KEY 0: trace blocks, 1: fold warps, 2: continuation blocks.
template <int KEY>
__device__ __forceinline__ uint32_t find_segment(const BatchSegment *__restrict__ segs, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;  // last segment whose begin <= key
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint64_t b = KEY == 1 ? segs[mid].warp_begin : (KEY == 2 ? segs[mid].park_block_begin : segs[mid].block_begin);
        if (b <= key) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void load_slot(SceneSlot &dst_slot, const SceneSlot *__restrict__ src_slot) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(src_slot);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&dst_slot);
    for (uint32_t i = threadIdx.x; i < sizeof(SceneSlot) / 4; i += blockDim.x) dst[i] = src[i];
}

// Stage 1 of a batched launch (the staged scheme of the single-scene kernels): paths
// run up to their segment's stage cap; survivors are parked in their segment's park region
// (`park`, slot counters `counts` per segment of the launch) for k_trace_batch_cont.
// EXTRAS: the variant for launches holding a scene with frosted facets, scattering or
// a biaxial material.  K: the scene class every segment of the launch belongs to
// (gr_trace.cuh K_*; K_ANY: checked at run time), MB: resident blocks per SM.
template <bool EXTRAS, int K = K_ANY, int MB = GR_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(TRACE_THREADS, MB)
    k_trace_batch(const SceneSlot *__restrict__ slots, const BatchSegment *__restrict__ segs, uint32_t n_segs,
                  Path *__restrict__ park, unsigned int *__restrict__ counts) {
    __shared__ SceneSlot s_slot;
    __shared__ uint32_t s_seg;
    extern __shared__ float4 s_planes[];
    if (threadIdx.x == 0) s_seg = find_segment<0>(segs, n_segs, blockIdx.x);
    __syncthreads();
    const BatchSegment &G = segs[s_seg];
    load_slot(s_slot, slots + G.scene);
    __syncthreads();
    const SceneConst &S = s_slot.S;
    const SceneBuffers &B = s_slot.B;
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const LaunchRange R = G.R;
    const uint64_t t = (uint64_t)(blockIdx.x - G.block_begin) * blockDim.x + threadIdx.x;
    const bool active = t < R.n_tuples;
    Path P;
    if (active) {
        uint32_t pixel, sample;
        tuple_coords(R, t, pixel, sample);
        path_init<1, EXTRAS, K>(P, S, B, pixel, sample, (uint32_t)t);
    }
    const ParkOut out{park + G.park_off, G.park_cap, counts + s_seg};
    if (run_or_park<EXTRAS, K>(P, S, PL, active, G.stage_cap, out) || !active) return;
    const V3 c = path_finish<1, false, K>(P, S, B);
    float *xyz = G.xyz;
    xyz[3 * t + 0] = c.x;
    xyz[3 * t + 1] = c.y;
    xyz[3 * t + 2] = c.z;
}

// Stage 2: each block resumes up to 128 parked paths of one segment (its scene in
// shared memory, as in stage 1) and runs them to their end.
template <bool EXTRAS, int K = K_ANY, int MB = GR_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(TRACE_THREADS, MB)
    k_trace_batch_cont(const SceneSlot *__restrict__ slots, const BatchSegment *__restrict__ segs, uint32_t n_segs,
                       const Path *__restrict__ park, const unsigned int *__restrict__ counts) {
    __shared__ SceneSlot s_slot;
    __shared__ uint32_t s_seg;
    extern __shared__ float4 s_planes[];
    if (threadIdx.x == 0) s_seg = find_segment<2>(segs, n_segs, blockIdx.x);
    __syncthreads();
    const BatchSegment &G = segs[s_seg];
    const uint32_t n = min((uint32_t)counts[s_seg], G.park_cap);
    const uint64_t j0 = (uint64_t)(blockIdx.x - G.park_block_begin) * blockDim.x;
    if (j0 >= n) return;  // block-uniform: no thread of this block reaches a barrier
    load_slot(s_slot, slots + G.scene);
    __syncthreads();
    const SceneConst &S = s_slot.S;
    const SceneBuffers &B = s_slot.B;
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint64_t i = j0 + threadIdx.x;
    if (i >= n) return;
    Path P = park[G.park_off + i];
    NoCounters nc;
    const V3 c = trace_path<NoCounters, false, EXTRAS, K>(P, S, B, PL, nc);
    const uint64_t t = p_tuple(P);
    float *xyz = G.xyz;
    xyz[3 * t + 0] = c.x;
    xyz[3 * t + 1] = c.y;
    xyz[3 * t + 2] = c.z;
}

// One batched launch's two trace grids for scene class K at MB blocks per SM.
template <bool EXTRAS, int K, int MB>
void launch_batch_grids(const SceneSlot *slots, const BatchSegment *segs, uint32_t n_segs, Path *park,
                        unsigned int *counts, uint64_t blocks, uint64_t park_blocks, size_t smem, cudaStream_t s) {
    k_trace_batch<EXTRAS, K, MB><<<(unsigned)blocks, TRACE_THREADS, smem, s>>>(slots, segs, n_segs, park, counts);
    k_trace_batch_cont<EXTRAS, K, MB><<<(unsigned)park_blocks, TRACE_THREADS, smem, s>>>(slots, segs, n_segs, park,
                                                                                        counts);
}


}  // namespace grd
