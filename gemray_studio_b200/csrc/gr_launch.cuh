// gr_launch.cuh -- launch-shape helpers shared by the transport kernels: the tuple
// numbering of a launch, shared-memory staging of the facet planes and the ordered
// per-pixel film fold.
//
// Work unit: a tuple t in [0, n_pixels * spp) of one launch maps to
//   pixel = first_pixel + t / spp, absolute sample = sample_offset + t % spp,
// the reference kernel's `idx = pixel * spp + s` numbering
// (renderer/shaders/spectral_transport.wgsl:672-691), and its XYZ lands in
// xyz[3 * t .. 3 * t + 3).  The fold then sums each pixel's spp samples in sample
// order and adds the sum once to the film -- the reference's per-pixel
// `sum += sample; accum[p] += sum` (renderer/gpu/frame.rs:799-814).
#pragma once

#include "gr_trace.cuh"

namespace grd {

constexpr int TRACE_THREADS = 128;

struct LaunchRange {
    uint32_t first_pixel;
    uint32_t n_pixels;
    uint32_t sample_offset;
    uint32_t spp;
    uint64_t n_tuples;  // n_pixels * spp
};

// Both shared-memory layouts of the paired scan (planes_smem_bytes(n) bytes at sp).
__device__ __forceinline__ Planes stage_plane_set(float4 *sp, const float4 *__restrict__ gp, uint32_t n) {
    float4 *pairs = sp + n;
    const uint32_t np = (n + 1u) >> 1;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sp[i] = gp[i];
    for (uint32_t j = threadIdx.x; j < np; j += blockDim.x) {
        const float4 a = gp[2 * j];
        const float4 b = 2 * j + 1 < n ? gp[2 * j + 1] : make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        pairs[2 * j] = make_float4(a.x, b.x, a.y, b.y);
        pairs[2 * j + 1] = make_float4(a.z, b.z, a.w, b.w);
    }
    __syncthreads();
    return Planes{sp, pairs, n};
}

__device__ __forceinline__ void tuple_coords(const LaunchRange &R, uint64_t t, uint32_t &pixel, uint32_t &sample) {
    uint32_t local_pixel = (uint32_t)(t / R.spp);
    uint32_t s = (uint32_t)(t - (uint64_t)local_pixel * R.spp);
    pixel = R.first_pixel + local_pixel;
    sample = R.sample_offset + s;  // u32 wrapping add, as the reference's wrapping_add
}


// One warp folds pixel `px` (local to its xyz block) into film pixel `film_pixel`.
// Add mode (cont == 0): the samples are summed in order from zero and the sum is
// added to the film once -- the reference's per-call semantics.  Continue mode
// (cont != 0): the sum starts from the film's current value (and, with Kahan, from
// the compensation kept in comp) and is written back, so successive slices of one
// sample range on a zero film form exactly one sequential sum, whatever the slicing.
__device__ __forceinline__ void fold_pixel(const float *__restrict__ xyz, uint64_t px, uint32_t spp, uint32_t film_pixel,
                                           float *__restrict__ film, uint32_t kahan, uint32_t cont = 0,
                                           float *__restrict__ comp = nullptr) {
    const uint32_t lane = threadIdx.x & 31u;
    const float *src = xyz + (size_t)px * spp * 3;
    const size_t p = (size_t)film_pixel * 3;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    if (cont) {
        sx = film[p + 0];
        sy = film[p + 1];
        sz = film[p + 2];
        if (kahan) {
            cx = comp[p + 0];
            cy = comp[p + 1];
            cz = comp[p + 2];
        }
    }
    for (uint32_t s0 = 0; s0 < spp; s0 += 32) {
        uint32_t s = s0 + lane;
        float x = 0.f, y = 0.f, z = 0.f;
        if (s < spp) {
            x = src[3 * s + 0];
            y = src[3 * s + 1];
            z = src[3 * s + 2];
        }
        uint32_t cnt = spp - s0 < 32u ? spp - s0 : 32u;
        for (uint32_t j = 0; j < cnt; ++j) {
            float vx = __shfl_sync(0xffffffffu, x, j);
            float vy = __shfl_sync(0xffffffffu, y, j);
            float vz = __shfl_sync(0xffffffffu, z, j);
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
    if (lane == 0) {
        if (cont) {
            film[p + 0] = sx;
            film[p + 1] = sy;
            film[p + 2] = sz;
            if (kahan) {
                comp[p + 0] = cx;
                comp[p + 1] = cy;
                comp[p + 2] = cz;
            }
        } else {
            film[p + 0] = film[p + 0] + sx;
            film[p + 1] = film[p + 1] + sy;
            film[p + 2] = film[p + 2] + sz;
        }
    }
}

}  // namespace grd
