// gr_stage.cuh -- the staged transport scheme shared by the single-scene kernels
// (gr_kernels.cuh) and the batched ones (gr_batch.cuh).
#pragma once

#include "gr_launch.cuh"

namespace grd {

// Staged kernels.  Within a warp path lengths differ widely (on the c2 brilliant the
// warp's longest path averages ~2.6x the mean), so a warp spends most of its bounce
// iterations on a few long paths with the other lanes idle.  Stage 1 runs every path
// for at most a first cap of bounces; a path still alive then is parked -- its record
// copied to a park buffer in warp-aggregated slots -- and a continuation stage
// resumes the parked paths, now packed densely, one per thread, again up to a second
// cap with its own park buffer for a final, uncapped stage.  The caps are kernel
// arguments: GR_STAGE_CAP / GR_STAGE_CAP2 by default, or the pair a resident scene
// chose by timing (StageCapTune, gr_host.cu).  A path whose
// slot would overflow a park buffer simply continues in place.  Each path runs the
// same functions in the same order as in the plain kernel, so every XYZ is
// bit-identical; only the schedule differs.
#ifndef GR_STAGE_CAP
#define GR_STAGE_CAP 12
#endif
#ifndef GR_STAGE_CAP2
#define GR_STAGE_CAP2 20
#endif

// Unroll factor of the per-channel loops in the staged kernels' bounce stages.
#ifndef GR_STEP_UNROLL
#define GR_STEP_UNROLL 1
#endif

struct ParkOut {
    Path *park;
    uint32_t cap;
    unsigned int *count;
};

// Bounces P up to `cap` (absolute bounce index), then parks it in `out` if still alive
// and a slot is free; returns true when parked.  A path that cannot be parked is run
// to its end.  Every lane of the warp must call this (the slot ballot), `active`
// false for lanes without a path.
template <bool EXTRAS, int K = K_ANY>
__device__ __forceinline__ bool run_or_park(Path &P, const SceneConst &S, const Planes &PL, bool active, uint32_t cap,
                                            const ParkOut &out) {
    NoCounters nc;
    const uint32_t lane = threadIdx.x & 31u;
    for (int round = 0; round < 2; ++round) {
        if (active) {
            while ((state_bits(P) & F_ALIVE) && p_bounce(P) < cap) {
                Event E;
                const uint32_t ev = step_hit<GR_STEP_UNROLL, NoCounters, false, EXTRAS, K>(P, S, PL, E, nc);
                if (ev == EV_REFLECT) step_reflect<GR_STEP_UNROLL, NoCounters, EXTRAS, K>(P, S, E, nc);
                else if (ev == EV_REFRACT) step_refract<GR_STEP_UNROLL, NoCounters, EXTRAS, K>(P, S, E, nc);
            }
        }
        if (round == 1 || out.cap == 0) break;
        const bool want = active && (state_bits(P) & F_ALIVE);
        const uint32_t mask = __ballot_sync(0xffffffffu, want);
        if (mask == 0u) break;
        uint32_t base = 0;
        const uint32_t leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(out.count, (unsigned)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (want) {
            const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
            if (slot < out.cap) {
                out.park[slot] = P;
                return true;
            }
        }
        cap = 0xFFFFFFFFu;  // park buffer full: finish in place
    }
    return false;
}

}  // namespace grd
