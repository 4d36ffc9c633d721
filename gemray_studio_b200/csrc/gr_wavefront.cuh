// gr_wavefront.cuh -- wavefront transport engine.
//
// Paths live in a device pool of `cap` records (gr_trace.cuh Path, 352 B each) plus a
// 64 B event scratch per slot.  One iteration runs these kernels on the context
// stream:
//
//   regen_prep  (1 thread)  take min(free slots, unstarted tuples) new tuples
//   regen       path_init into freed slots           -> active[cur]
//   extend      step_hit over active[cur]            -> reflect | refract | finish
//   reflect     step_reflect over the reflect queue   -> active[nxt] | finish
//   refract     step_refract over the refract queue   -> active[nxt] | finish
//   finish      path_finish, write XYZ of the tuple  -> free
//   bookkeep    (1 thread)  reset consumed queues, raise the done flag
//
// Every queue is a compacted index list filled with warp-aggregated atomics, so each
// stage kernel runs full warps of ONE event type and only that stage's code -- the
// divergence and instruction-cache pressure of a one-thread-per-path megakernel
// disappear.  Results per tuple are identical to the plain kernel (same functions,
// same operation order); only the schedule differs.
#pragma once

#include <cooperative_groups.h>

#include "gr_kernels.cuh"

namespace grd {

namespace cg = cooperative_groups;

enum WaveCount : uint32_t {
    W_ACT0 = 0, W_ACT1 = 1, W_REFL = 2, W_REFR = 3, W_FIN = 4, W_FREE = 5, W_REGEN_N = 6, W_REGEN_BASE = 7,
    W_DONE = 8, W_NCOUNT = 16
};

struct WaveBuffers {
    Path *pool;
    Event *events;
    uint32_t *q_active0, *q_active1, *q_reflect, *q_refract, *q_finish, *q_free;
    uint32_t *cnt;                    // WaveCount slots
    unsigned long long *tuples;       // [0] next unstarted tuple, [1] base tuple of the current regen
    uint32_t cap;
};

__device__ __forceinline__ uint32_t *active_q(const WaveBuffers &W, uint32_t which) {
    return which ? W.q_active1 : W.q_active0;
}

// Warp-aggregated append of `value` to list/count (called by the lanes that append).
__device__ __forceinline__ void wq_push(uint32_t *list, uint32_t *count, uint32_t value) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
    base = g.shfl(base, 0);
    list[base + g.thread_rank()] = value;
}

__global__ void k_wf_reset(WaveBuffers W) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.cap; i += stride) W.q_free[i] = i;
    if (blockIdx.x == 0 && threadIdx.x < W_NCOUNT) W.cnt[threadIdx.x] = threadIdx.x == W_FREE ? W.cap : 0u;
    if (blockIdx.x == 0 && threadIdx.x < 2) W.tuples[threadIdx.x] = 0ull;
}

__global__ void k_wf_regen_prep(WaveBuffers W, uint64_t n_tuples) {
    const uint32_t free_n = W.cnt[W_FREE];
    const unsigned long long next = W.tuples[0];
    const unsigned long long left = next < n_tuples ? n_tuples - next : 0ull;
    const uint32_t take = left < free_n ? (uint32_t)left : free_n;
    W.cnt[W_REGEN_N] = take;
    W.cnt[W_REGEN_BASE] = free_n - take;
    W.cnt[W_FREE] = free_n - take;
    W.tuples[1] = next;
    W.tuples[0] = next + take;
}

__global__ void __launch_bounds__(256) k_wf_regen(SceneConst S, SceneBuffers B, LaunchRange R, WaveBuffers W,
                                                  uint32_t cur) {
    const uint32_t n = W.cnt[W_REGEN_N], base_slot = W.cnt[W_REGEN_BASE];
    const unsigned long long t0 = W.tuples[1];
    uint32_t *act = active_q(W, cur);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = W.q_free[base_slot + i];
        const uint64_t t = t0 + i;
        uint32_t pixel, sample;
        tuple_coords(R, t, pixel, sample);
        path_init<1, true>(W.pool[slot], S, B, pixel, sample, (uint32_t)t);
        wq_push(act, W.cnt + (cur ? W_ACT1 : W_ACT0), slot);
    }
}

__global__ void __launch_bounds__(256) k_wf_extend(SceneConst S, SceneBuffers B, WaveBuffers W, uint32_t cur) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint32_t n = W.cnt[cur ? W_ACT1 : W_ACT0];
    const uint32_t *act = active_q(W, cur);
    const uint32_t stride = gridDim.x * blockDim.x;
    NoCounters nc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = act[i];
        const uint32_t ev = step_hit<1, NoCounters, false, true>(W.pool[slot], S, PL, W.events[slot], nc);
        if (ev == EV_REFLECT) wq_push(W.q_reflect, W.cnt + W_REFL, slot);
        else if (ev == EV_REFRACT) wq_push(W.q_refract, W.cnt + W_REFR, slot);
        else if (ev == EV_HANDLED && (state_bits(W.pool[slot]) & F_ALIVE))  // frosted / scattered: next round
            wq_push(active_q(W, cur ^ 1u), W.cnt + (cur ? W_ACT0 : W_ACT1), slot);
        else wq_push(W.q_finish, W.cnt + W_FIN, slot);
    }
}

template <bool REFRACT>
__global__ void __launch_bounds__(256) k_wf_event(SceneConst S, WaveBuffers W, uint32_t nxt) {
    const uint32_t n = W.cnt[REFRACT ? W_REFR : W_REFL];
    const uint32_t *q = REFRACT ? W.q_refract : W.q_reflect;
    uint32_t *act = active_q(W, nxt);
    const uint32_t stride = gridDim.x * blockDim.x;
    NoCounters nc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = q[i];
        Path &P = W.pool[slot];
        if (REFRACT) step_refract<1, NoCounters, true>(P, S, W.events[slot], nc);
        else step_reflect<1, NoCounters, true>(P, S, W.events[slot], nc);
        if (state_bits(P) & F_ALIVE) wq_push(act, W.cnt + (nxt ? W_ACT1 : W_ACT0), slot);
        else wq_push(W.q_finish, W.cnt + W_FIN, slot);
    }
}

__global__ void __launch_bounds__(256) k_wf_finish(SceneConst S, SceneBuffers B, WaveBuffers W, float *__restrict__ xyz) {
    const uint32_t n = W.cnt[W_FIN];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = W.q_finish[i];
        const Path &P = W.pool[slot];
        const V3 c = path_finish<1>(P, S, B);
        const uint64_t t = p_tuple(P);
        xyz[3 * t + 0] = c.x;
        xyz[3 * t + 1] = c.y;
        xyz[3 * t + 2] = c.z;
        wq_push(W.q_free, W.cnt + W_FREE, slot);
    }
}

__global__ void k_wf_bookkeep(WaveBuffers W, uint32_t cur, uint64_t n_tuples) {
    W.cnt[cur ? W_ACT1 : W_ACT0] = 0;
    W.cnt[W_REFL] = 0;
    W.cnt[W_REFR] = 0;
    W.cnt[W_FIN] = 0;
    W.cnt[W_DONE] = (W.tuples[0] >= n_tuples && W.cnt[cur ? W_ACT0 : W_ACT1] == 0) ? 1u : 0u;
}

}  // namespace grd
