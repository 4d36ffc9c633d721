// gr_kernels.cuh -- the film fold and the FP32 probe of the single-scene path
// (sm_100a); the plain and staged transport kernels are templates in gr_transport.cuh,
// tuple numbering and the ordered fold in gr_launch.cuh.  Included by gr_host.cu only
// (the kernels here are not templates and must be defined once).
#pragma once

#include "gr_transport.cuh"

namespace grd {

// The single-scene film fold with one thread per pixel: the block's pixels' samples
// pass through shared memory in tiles of FOLD_TILE samples (each pixel's tile is one
// contiguous run of the per-tuple XYZ, loaded by the whole block), and each thread adds
// its pixel's samples in sample order -- the additions of fold_pixel (plain or Kahan,
// add mode), so the film is bit-identical, without fold_pixel's three shuffles per
// sample and warp.
constexpr uint32_t FOLD_THREADS = 128, FOLD_TILE = 8, FOLD_ROW = FOLD_TILE * 3 + 1;

// Stages floats [0, np * PER) of the tile (PER floats per pixel, from sample s0 on).
template <uint32_t PER>
__device__ __forceinline__ void fold_stage(float (*tile)[FOLD_ROW], const float *__restrict__ base, uint32_t np,
                                           uint32_t spp, uint32_t s0, uint32_t per_rt) {
    const uint32_t per = PER ? PER : per_rt;
    const uint32_t total = np * per;
    for (uint32_t f = threadIdx.x; f < total; f += FOLD_THREADS) {
        const uint32_t pi = f / per, w = f - pi * per;
        tile[pi][w] = base[((uint64_t)pi * spp + s0) * 3 + w];
    }
}

__global__ void __launch_bounds__(FOLD_THREADS) k_film_fold_tiled(const float *__restrict__ xyz, uint32_t n_pixels,
                                                                 uint32_t spp, uint32_t first_pixel,
                                                                 float *__restrict__ film, uint32_t kahan) {
    __shared__ float tile[FOLD_THREADS][FOLD_ROW];
    const uint64_t px0 = (uint64_t)blockIdx.x * FOLD_THREADS;
    const uint32_t np = (uint32_t)min((uint64_t)FOLD_THREADS, (uint64_t)n_pixels - px0);
    const uint32_t i = threadIdx.x;
    const float *base = xyz + px0 * spp * 3;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    for (uint32_t s0 = 0; s0 < spp; s0 += FOLD_TILE) {
        const uint32_t t = min(FOLD_TILE, spp - s0);
        if (t == FOLD_TILE) fold_stage<FOLD_TILE * 3>(tile, base, np, spp, s0, 0);
        else fold_stage<0>(tile, base, np, spp, s0, t * 3);
        __syncthreads();
        if (i < np) {
            for (uint32_t j = 0; j < t; ++j) {
                const float vx = tile[i][3 * j + 0], vy = tile[i][3 * j + 1], vz = tile[i][3 * j + 2];
                if (kahan) {
                    float yx = vx - cx, tx = sx + yx; cx = (tx - sx) - yx; sx = tx;
                    float yy = vy - cy, ty = sy + yy; cy = (ty - sy) - yy; sy = ty;
                    float yz = vz - cz, tz = sz + yz; cz = (tz - sz) - yz; sz = tz;
                } else {
                    sx = sx + vx;
                    sy = sy + vy;
                    sz = sz + vz;
                }
            }
        }
        __syncthreads();
    }
    if (i < np) {
        const size_t p = ((size_t)first_pixel + px0 + i) * 3;
        film[p + 0] = film[p + 0] + sx;
        film[p + 1] = film[p + 1] + sy;
        film[p + 2] = film[p + 2] + sz;
    }
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
