// gr_sorted.cuh -- the block-sorted transport kernel for clear isotropic stones
// (GR_KERNEL_SORTED).
//
// In the plain and staged kernels a thread owns one path from start to end, so a warp
// runs every event kind its 32 paths take at a bounce (reflect and refract, one after
// the other with part of the warp masked off) and waits for its longest path.  Here a
// block of SORT_THREADS threads owns SORT_THREADS path slots in shared memory, and any
// thread may advance any slot.  A slot is empty, live with a pending event (reflect or
// refract, decided by its last intersection step), or ended.  Each round of the block
// is one compaction and one work phase:
//   lists  every slot joins one of three lists (block-wide ballots and warp counts):
//          pending reflections, pending refractions, slots to refill (empty or ended);
//          the block claims as many new tuples as it has slots to refill from the
//          launch's global counter;
//   work   threads [0, n_reflect) take the reflections, the next threads the
//          refractions, the rest the refills (finish the ended path: XYZ written;
//          start a claimed tuple), and every thread then runs the next intersection
//          step of its slot -- so each warp runs one event kind, the intersection code
//          is uniform, and every slot advances one bounce per round.
// Three barriers per round.  Every path runs path_init, the step functions and
// path_finish in the same order as in the plain kernel, so every XYZ is bit-identical;
// only the assignment of paths to threads changes.
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
    uint16_t list[SORT_THREADS];  // reflections, then refractions, then refills
    uint8_t state[SORT_THREADS];
    uint8_t ev[SORT_THREADS];
    uint32_t cnt[4][SORT_WARPS];  // per warp: reflect, refract, refill, ended
    uint32_t base;                // first tuple claimed this round
};

__device__ __forceinline__ Path &slot_path(unsigned char *slots, uint32_t i) {
    return *reinterpret_cast<Path *>(slots + (size_t)i * SORT_SLOT_BYTES);
}
__device__ __forceinline__ Event &slot_event(unsigned char *slots, uint32_t i) {
    return *reinterpret_cast<Event *>(slots + (size_t)i * SORT_SLOT_BYTES + PATH_CLEAR_BYTES);
}

// The intersection step of a live slot; a path that escapes ends there.
template <int K>
__device__ __forceinline__ void slot_hit(SortShared &sh, unsigned char *slots, uint32_t slot, const SceneConst &S,
                                         const Planes &PL) {
    NoCounters nc;
    Path &P = slot_path(slots, slot);
    const uint32_t ev = step_hit<1, NoCounters, false, false, K>(P, S, PL, slot_event(slots, slot), nc);
    sh.ev[slot] = (uint8_t)ev;
    sh.state[slot] = (state_bits(P) & F_ALIVE) ? SLOT_LIVE : SLOT_ENDED;
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
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    NoCounters nc;
    sh.state[tid] = SLOT_EMPTY;
    bool supply = true;  // block-uniform: tuples may remain
    __syncthreads();
    for (;;) {
        // lists: this thread classifies its own slot
        const uint32_t my_state = sh.state[tid];
        const bool live = my_state == SLOT_LIVE;
        const bool fr = live && sh.ev[tid] == EV_REFLECT, ff = live && sh.ev[tid] == EV_REFRACT;
        const bool fn = !live, fe = my_state == SLOT_ENDED;
        const uint32_t mr = __ballot_sync(0xffffffffu, fr), mf = __ballot_sync(0xffffffffu, ff);
        const uint32_t mn = __ballot_sync(0xffffffffu, fn), me = __ballot_sync(0xffffffffu, fe);
        if (lane == 0) {
            sh.cnt[0][w] = __popc(mr);
            sh.cnt[1][w] = __popc(mf);
            sh.cnt[2][w] = __popc(mn);
            sh.cnt[3][w] = __popc(me);
        }
        __syncthreads();
        uint32_t tot[4] = {0u, 0u, 0u, 0u}, off[3] = {0u, 0u, 0u};
#pragma unroll
        for (uint32_t i = 0; i < SORT_WARPS; ++i) {
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const uint32_t c = sh.cnt[l][i];
                if (l < 3 && i < w) off[l] += c;
                tot[l] += c;
            }
        }
        const uint32_t n_r = tot[0], n_f = tot[1], n_n = tot[2], n_ended = tot[3];
        const uint32_t claim = supply ? n_n : 0u;  // no slot to refill: claim nothing, keep the supply
        const uint32_t below = (1u << lane) - 1u;
        if (fr) sh.list[off[0] + __popc(mr & below)] = (uint16_t)tid;
        if (ff) sh.list[n_r + off[1] + __popc(mf & below)] = (uint16_t)tid;
        if (fn) sh.list[n_r + n_f + off[2] + __popc(mn & below)] = (uint16_t)tid;
        if (tid == 0 && claim) sh.base = atomicAdd(work, claim);
        __syncthreads();
        if (n_r + n_f == 0 && n_ended == 0 && claim == 0) break;  // block-uniform: nothing left at all
        const uint32_t base = sh.base;
        if (claim && (uint64_t)base + claim >= R.n_tuples) supply = false;
        // work: one event (or refill) and the next intersection step per slot
        const uint32_t slot = sh.list[tid];
        Path &P = slot_path(slots, slot);
        if (tid < n_r + n_f) {
            if (tid < n_r) step_reflect<1, NoCounters, false, K>(P, S, slot_event(slots, slot), nc);
            else step_refract<1, NoCounters, false, K>(P, S, slot_event(slots, slot), nc);
            if (state_bits(P) & F_ALIVE) slot_hit<K>(sh, slots, slot, S, PL);
            else sh.state[slot] = SLOT_ENDED;
        } else {
            if (sh.state[slot] == SLOT_ENDED) {
                const V3 c = path_finish<1, false, K>(P, S, B);
                const uint64_t t = p_tuple(P);
                xyz[3 * t + 0] = c.x;
                xyz[3 * t + 1] = c.y;
                xyz[3 * t + 2] = c.z;
            }
            const uint64_t t = (uint64_t)base + (tid - n_r - n_f);
            if (claim && t < R.n_tuples) {
                uint32_t pixel, sample;
                tuple_coords(R, t, pixel, sample);
                path_init<1, false, K>(P, S, B, pixel, sample, (uint32_t)t);
                slot_hit<K>(sh, slots, slot, S, PL);
            } else {
                sh.state[slot] = SLOT_EMPTY;
            }
        }
        __syncthreads();
    }
}

}  // namespace grd
