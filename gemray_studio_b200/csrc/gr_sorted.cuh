// gr_sorted.cuh -- the block-sorted transport kernel for clear isotropic stones
// (GR_KERNEL_SORTED).
//
// In the plain and staged kernels a thread owns one path from start to end, so a warp
// runs every event kind its 32 paths take at a bounce (reflect and refract, one after
// the other with part of the warp masked off) and waits for its longest path.  Here a
// block of SORT_THREADS threads owns SORT_THREADS path slots in shared memory, and any
// thread may advance any slot.  Each round of the block:
//   refill  the slots whose path ended are finished (XYZ written) and restarted with
//           the next tuples of the launch (claimed from a global counter), so slots
//           stay full until the launch's tuples run out;
//   hit     one intersection step (step_hit) for every live slot, threads taking the
//           compacted list of live slots;
//   events  the slots whose event is a reflection go to threads [0, n_reflect), the
//           refractions to the threads after them, so each warp runs one event kind
//           (only the warp on the boundary runs both).
// The lists are block-wide compactions (warp ballots and four warp counts).  Every path
// runs path_init, the step functions and path_finish in the same order as in the plain
// kernel, so every XYZ is bit-identical; only the assignment of paths to threads
// changes.
//
// Measured on B200 (c2's scene at 480x270, 64 spp, ncu captures of both forms): this
// form executes 9% fewer warp instructions than the staged kernels (19.8 threads per
// instruction), writes 62 MB of DRAM instead of 1.5 GB and hardly stalls on instruction
// fetch, but with 20 resident warps per SM and nine barriers per round its issue slots
// are only half busy (barrier stalls 3.2 cycles per issue): 11.1 ms against the staged
// kernels' 9.1 ms.  A variant with one compaction and one combined event + refill +
// intersection phase per round (three barriers) was slower still (12.5 ms): its rounds
// last as long as their slowest warp.  The staged kernels stay the default.
//
// Layout: a slot is the PATH_CLEAR_BYTES of Path a clear isotropic stone uses followed
// by its EVENT_ISO_BYTES of Event, padded to SORT_SLOT_BYTES = 304 B: 76 words, so
// eight lanes reading the same float4 row of consecutive slots hit 32 distinct banks.
// 128 slots (38 KB) plus the plane tables fit five blocks on an SM (20 warps).
#pragma once

#include "gr_launch.cuh"

namespace grd {

constexpr int SORT_THREADS = 128;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr size_t SORT_SLOT_BYTES = 304;
#ifndef GR_SORT_MIN_BLOCKS
#define GR_SORT_MIN_BLOCKS 5
#endif
static_assert(PATH_CLEAR_BYTES + EVENT_ISO_BYTES <= SORT_SLOT_BYTES, "slot holds the clear path and its event");
static_assert(SORT_SLOT_BYTES % 16 == 0 && (SORT_SLOT_BYTES / 4) % 8 == 4, "conflict-free float4 rows");

__host__ __device__ constexpr size_t sorted_smem_bytes(uint32_t n_planes) {
    return (size_t)SORT_THREADS * SORT_SLOT_BYTES + planes_smem_bytes(n_planes);
}

enum SlotState : uint8_t { SLOT_EMPTY = 0, SLOT_LIVE = 1, SLOT_ENDED = 2 };

struct SortShared {
    uint16_t list_a[SORT_THREADS];
    uint16_t list_b[SORT_THREADS];
    uint8_t state[SORT_THREADS];
    uint8_t ev[SORT_THREADS];
    uint32_t cnt_a[SORT_WARPS], cnt_b[SORT_WARPS];
    uint32_t base;
};

__device__ __forceinline__ Path &slot_path(unsigned char *slots, uint32_t i) {
    return *reinterpret_cast<Path *>(slots + (size_t)i * SORT_SLOT_BYTES);
}
__device__ __forceinline__ Event &slot_event(unsigned char *slots, uint32_t i) {
    return *reinterpret_cast<Event *>(slots + (size_t)i * SORT_SLOT_BYTES + PATH_CLEAR_BYTES);
}

// Two block-wide compactions at once: thread tid's slot joins list_a if fa, list_b if
// fb (each list in slot order).  Returns both totals (block-uniform).
__device__ __forceinline__ uint2 compact2(SortShared &sh, bool fa, bool fb) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const uint32_t ma = __ballot_sync(0xffffffffu, fa), mb = __ballot_sync(0xffffffffu, fb);
    if (lane == 0) {
        sh.cnt_a[w] = __popc(ma);
        sh.cnt_b[w] = __popc(mb);
    }
    __syncthreads();
    uint32_t oa = 0, ob = 0, ta = 0, tb = 0;
#pragma unroll
    for (uint32_t i = 0; i < SORT_WARPS; ++i) {
        const uint32_t ca = sh.cnt_a[i], cb = sh.cnt_b[i];
        oa += i < w ? ca : 0u;
        ob += i < w ? cb : 0u;
        ta += ca;
        tb += cb;
    }
    const uint32_t below = (1u << lane) - 1u;
    if (fa) sh.list_a[oa + __popc(ma & below)] = (uint16_t)tid;
    if (fb) sh.list_b[ob + __popc(mb & below)] = (uint16_t)tid;
    __syncthreads();
    return make_uint2(ta, tb);
}

template <int K>
__global__ void __launch_bounds__(SORT_THREADS, GR_SORT_MIN_BLOCKS) k_trace_sorted(SceneConst S, SceneBuffers B,
                                                                                   LaunchRange R, float *__restrict__ xyz,
                                                                                   unsigned int *__restrict__ work) {
    static_assert((K & K_ISO) && (K & K_CLEAR), "slots hold the clear isotropic record only");
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ SortShared sh;
    unsigned char *slots = dsm;
    const Planes PL = stage_plane_set(reinterpret_cast<float4 *>(dsm + SORT_THREADS * SORT_SLOT_BYTES), B.planes,
                                      S.n_planes);
    const uint32_t tid = threadIdx.x;
    NoCounters nc;
    sh.state[tid] = SLOT_EMPTY;
    bool supply = true;  // block-uniform: tuples may remain
    for (;;) {
        // refill: finish ended paths, start the next tuples in their slots and in empty ones
        const uint32_t n_free = compact2(sh, sh.state[tid] != SLOT_LIVE, false).x;
        const uint32_t claim = supply ? n_free : 0u;  // no free slot: claim nothing, keep the supply
        if (tid == 0 && claim) sh.base = atomicAdd(work, claim);
        __syncthreads();
        const uint32_t base = sh.base;
        if (claim && (uint64_t)base + claim >= R.n_tuples) supply = false;
        if (tid < n_free) {
            const uint32_t slot = sh.list_a[tid];
            Path &P = slot_path(slots, slot);
            if (sh.state[slot] == SLOT_ENDED) {
                const V3 c = path_finish<1, false, K>(P, S, B);
                const uint64_t t = p_tuple(P);
                xyz[3 * t + 0] = c.x;
                xyz[3 * t + 1] = c.y;
                xyz[3 * t + 2] = c.z;
            }
            const uint64_t t = (uint64_t)base + tid;
            if (claim && t < R.n_tuples) {
                uint32_t pixel, sample;
                tuple_coords(R, t, pixel, sample);
                path_init<1, false, K>(P, S, B, pixel, sample, (uint32_t)t);
                sh.state[slot] = SLOT_LIVE;
            } else {
                sh.state[slot] = SLOT_EMPTY;
            }
        }
        __syncthreads();
        // hit: one intersection step for every live slot
        const uint32_t n_live = compact2(sh, sh.state[tid] == SLOT_LIVE, false).x;
        if (n_live == 0) break;  // block-uniform: nothing live and nothing left to start
        if (tid < n_live) {
            const uint32_t slot = sh.list_a[tid];
            sh.ev[slot] = (uint8_t)step_hit<1, NoCounters, false, false, K>(slot_path(slots, slot), S, PL,
                                                                            slot_event(slots, slot), nc);
        }
        __syncthreads();
        // events: reflections on the first threads, refractions after them
        const bool live = sh.state[tid] == SLOT_LIVE;
        const uint2 n = compact2(sh, live && sh.ev[tid] == EV_REFLECT, live && sh.ev[tid] == EV_REFRACT);
        if (tid < n.x) {
            const uint32_t slot = sh.list_a[tid];
            step_reflect<1, NoCounters, false, K>(slot_path(slots, slot), S, slot_event(slots, slot), nc);
        } else if (tid < n.x + n.y) {
            const uint32_t slot = sh.list_b[tid - n.x];
            step_refract<1, NoCounters, false, K>(slot_path(slots, slot), S, slot_event(slots, slot), nc);
        }
        __syncthreads();
        if (live && !(state_bits(slot_path(slots, tid)) & F_ALIVE)) sh.state[tid] = SLOT_ENDED;
        __syncthreads();
    }
}

}  // namespace grd
