// gr_transport.cuh -- the single-scene transport kernels (sm_100a): the plain kernel
// (one thread per tuple) and the staged pair (capped first stage, dense continuation),
// templates over the scene class K (gr_trace.cuh) so that each class is compiled with
// only the code it runs.  Instantiated by gr_host.cu (the run-time class, counters, FP64
// re-solve, extension materials) and by gr_single_*.cu (the specialised classes).
#pragma once

#include "gr_stage.cuh"

namespace grd {

// Plain kernel: one thread traces one tuple start to finish -- the reference
// kernel's launch shape (one invocation per (pixel, sample), spectral_transport.wgsl:
// 672-691).  The Counters variant tallies events for the FLOP model; RESOLVE is the
// GR_FLAG_FP64_RESOLVE variant (FP64 re-solve of ambiguous exits and TIR decisions);
// EXTRAS the variant for scenes with frosted facets, volume scattering or a biaxial
// material.
template <class CT, bool RESOLVE = false, bool EXTRAS = false, int K = K_ANY, int MB = GR_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(TRACE_THREADS, MB) k_trace_plain(SceneConst S, SceneBuffers B, LaunchRange R,
                                                               float *__restrict__ xyz,
                                                               unsigned long long *__restrict__ tallies) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    CT ct;
    if constexpr (sizeof(CT) == sizeof(Counters)) {
        for (int i = 0; i < C_COUNT; ++i) ((Counters &)ct).c[i] = 0;
    }
    if (t < R.n_tuples) {
        uint32_t pixel, sample;
        tuple_coords(R, t, pixel, sample);
        Path P;
        path_init<1, EXTRAS, K>(P, S, B, pixel, sample, (uint32_t)t);
        tally(ct, C_PATHS);
        V3 c = trace_path<CT, RESOLVE, EXTRAS, K>(P, S, B, PL, ct);
        xyz[3 * t + 0] = c.x;
        xyz[3 * t + 1] = c.y;
        xyz[3 * t + 2] = c.z;
    }
    if constexpr (sizeof(CT) == sizeof(Counters)) {
        const uint32_t lane = threadIdx.x & 31u;
        for (int i = 0; i < C_COUNT; ++i) {
            unsigned long long v = ((Counters &)ct).c[i];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0 && v) atomicAdd(tallies + i, v);
        }
    }
}

// Staged kernels (the scheme and run_or_park are in gr_stage.cuh).
// MB: resident blocks per SM the register allocation targets (the schedule tuner's
// warps-per-SM dimension).
template <bool EXTRAS, int K = K_ANY, int MB = GR_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(TRACE_THREADS, MB) k_trace_stage1(SceneConst S, SceneBuffers B,
                                                                                     LaunchRange R,
                                                                                     float *__restrict__ xyz,
                                                                                     ParkOut out, uint32_t bounce_cap) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < R.n_tuples;
    Path P;
    if (active) {
        uint32_t pixel, sample;
        tuple_coords(R, t, pixel, sample);
        path_init<1, EXTRAS, K>(P, S, B, pixel, sample, (uint32_t)t);
    }
    if (run_or_park<EXTRAS, K>(P, S, PL, active, bounce_cap, out) || !active) return;
    const V3 c = path_finish<1, false, K>(P, S, B);
    xyz[3 * t + 0] = c.x;
    xyz[3 * t + 1] = c.y;
    xyz[3 * t + 2] = c.z;
}

// Continuation: parked paths [0, min(*count_in, cap_in)) resumed one per thread, up to
// `bounce_cap`, survivors parked in `out` (out.cap 0: run to the end).
template <bool EXTRAS, int K = K_ANY, int MB = GR_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(TRACE_THREADS, MB) k_trace_stage2(
    SceneConst S, SceneBuffers B, const Path *__restrict__ park_in, uint32_t cap_in,
    const unsigned int *__restrict__ count_in, uint32_t bounce_cap, ParkOut out, float *__restrict__ xyz) {
    const uint32_t n = min((uint32_t)*count_in, cap_in);
    if ((uint64_t)blockIdx.x * blockDim.x >= n) return;  // whole block past the parked paths
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    Path P;
    if (active) P = park_in[i];
    if (run_or_park<EXTRAS, K>(P, S, PL, active, bounce_cap, out) || !active) return;
    const V3 c = path_finish<1, false, K>(P, S, B);
    const uint64_t t = p_tuple(P);
    xyz[3 * t + 0] = c.x;
    xyz[3 * t + 1] = c.y;
    xyz[3 * t + 2] = c.z;
}

}  // namespace grd
