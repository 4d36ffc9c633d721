// gr_kernels.cuh -- the film fold and the FP32 probe of the single-scene path
// (sm_100a); the plain and staged transport kernels are templates in gr_transport.cuh,
// tuple numbering and the ordered fold in gr_launch.cuh.  Included by gr_host.cu only
// (the kernels here are not templates and must be defined once).
#pragma once

#include "gr_transport.cuh"

namespace grd {

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
