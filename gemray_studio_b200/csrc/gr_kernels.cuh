// gr_kernels.cuh -- the regeneration schedule, the film fold and the FP32 probe of the
// single-scene path (sm_100a); the plain and staged transport kernels are templates in
// gr_transport.cuh, tuple numbering and the ordered fold in gr_launch.cuh.  Included by
// gr_host.cu only (the kernels here are not templates and must be defined once).
#pragma once

#include "gr_transport.cuh"

namespace grd {

// Path-regeneration kernel.  Path lengths within a warp vary widely (on a brilliant
// the mean is ~3.7 bounces but the warp's longest path averages ~12), so a warp
// that runs each lane's path to its end idles most lanes most of the time.  Here
// each warp owns GR_REGEN_BATCH * 32 consecutive tuples; a lane whose path has ended
// waits until at least GR_REGEN_MIN_IDLE lanes are idle (or all are), then every
// idle lane finishes its path (writes its XYZ) and starts the warp's next unclaimed
// tuple, while the warp's live lanes carry on bouncing.  Each tuple still runs the
// same functions in the same order as in the plain kernel, so every XYZ is
// bit-identical; only the schedule differs.
#ifndef GR_REGEN_BATCH
#define GR_REGEN_BATCH 16
#endif
#ifndef GR_REGEN_MIN_IDLE
#define GR_REGEN_MIN_IDLE 16
#endif
constexpr uint32_t REGEN_TUPLES = 32u * GR_REGEN_BATCH;

__global__ void __launch_bounds__(TRACE_THREADS) k_trace_regen(SceneConst S, SceneBuffers B, LaunchRange R,
                                                               float *__restrict__ xyz) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t w_end0 = (warp + 1) * REGEN_TUPLES;
    const uint64_t w_end = w_end0 < R.n_tuples ? w_end0 : R.n_tuples;
    uint64_t next = warp * REGEN_TUPLES;  // warp-uniform: first unclaimed tuple
    if (next >= R.n_tuples) return;       // whole warp (n_tuples and the grid are warp-uniform)
    NoCounters nc;
    Path P;
    bool have = false;  // this lane holds a started, not yet finished path
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (;;) {
        bool alive = have && (state_bits(P) & F_ALIVE);
        const uint32_t idle = __ballot_sync(0xffffffffu, !alive);
        const uint32_t n_idle = __popc(idle);
        if (n_idle >= GR_REGEN_MIN_IDLE || idle == 0xffffffffu) {
            if (!alive) {
                if (have) {
                    const V3 c = path_finish<1>(P, S, B);
                    const uint64_t t = p_tuple(P);
                    xyz[3 * t + 0] = c.x;
                    xyz[3 * t + 1] = c.y;
                    xyz[3 * t + 2] = c.z;
                }
                const uint64_t t = next + __popc(idle & lt_mask);
                have = t < w_end;
                if (have) {
                    uint32_t pixel, sample;
                    tuple_coords(R, t, pixel, sample);
                    path_init<1, true>(P, S, B, pixel, sample, (uint32_t)t);
                }
            }
            next += n_idle;
            if (__ballot_sync(0xffffffffu, have) == 0u) break;
            alive = have && (state_bits(P) & F_ALIVE);
        }
        if (alive) {
            Event E;
            const uint32_t ev = step_hit<1, NoCounters, false, true>(P, S, PL, E, nc);
            if (ev == EV_REFLECT) step_reflect<1, NoCounters, true>(P, S, E, nc);
            else if (ev == EV_REFRACT) step_refract<1, NoCounters, true>(P, S, E, nc);
        }
    }
}

__global__ void k_film_fold(const float *__restrict__ xyz, uint32_t n_pixels, uint32_t spp, uint32_t first_pixel,
                            float *__restrict__ film, uint32_t kahan) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= n_pixels) return;
    fold_pixel(xyz, warp, spp, first_pixel + (uint32_t)warp, film, kahan);
}

static_assert(C_COUNT == GR_EVENT_COUNT, "counter layout");

// FP32 throughput probe: 8 independent FMA chains per thread (2 flops per FMA).
__global__ void k_fp32_probe(float *__restrict__ out, uint32_t iters, float seed) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.9999999f, c = 1e-7f;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    float r = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (r == 12345.678f) out[0] = r;  // keep the chains live
}

}  // namespace grd
