// gr_tonemap.cu -- tone-mapped pixels out: rgba = ColorSpace::Srgb.encode(xyz * scale,
// ToneMap::AcesFilmic { exposure: 1 }) per pixel (renderer/tonemap.rs:52-108,
// color/space.rs:290-334, color/gamut.rs:38-71, optics/raytracer/color.rs:365-417).
// One thread per pixel; the frame is HBM-bound (12 B in, 4 B out per pixel).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "gemray_cuda.h"
#include "gr_device.cuh"
#include "gr_host.h"

namespace grd {

// sRGB XYZ->linear (color/space.rs:192-198), fused like space.rs:256-263.
__device__ __forceinline__ V3 xyz_to_srgb_linear(V3 c) {
    return v3(fmaf(3.2404542f, c.x, fmaf(-1.5371385f, c.y, -0.4985314f * c.z)),
              fmaf(-0.969266f, c.x, fmaf(1.8760108f, c.y, 0.0415560f * c.z)),
              fmaf(0.0556434f, c.x, fmaf(-0.2040259f, c.y, 1.0572252f * c.z)));
}

__device__ __forceinline__ bool in_range(V3 v, float mx) {
    return v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f && v.x <= mx && v.y <= mx && v.z <= mx;
}

// gamut.rs:71-118 project_to_gamut_bounded for the sRGB white point.
__device__ __forceinline__ V3 project_to_gamut_bounded(V3 xyz, float mx) {
    float sum = xyz.x + xyz.y + xyz.z;
    if (!isfinite(sum) || sum <= 1e-6f) return v3(0.f, 0.f, 0.f);
    float x = xyz.x / sum, y = xyz.y / sum;
    float lum = fmaxf(xyz.y, 0.0f);
    V3 lin = xyz_to_srgb_linear(xyz);
    if (in_range(lin, mx)) return lin;
    const float wx = 0.3127f, wy = 0.3290f;
    auto mapped = [&](float t) -> V3 {
        float xp = fmaf(wx - x, t, x);
        float yp = fmaf(wy - y, t, y);
        if (yp > 1e-6f) return v3((xp / yp) * lum, lum, ((1.0f - xp - yp) / yp) * lum);
        return v3((wx / wy) * lum, lum, ((1.0f - wx - wy) / wy) * lum);
    };
    V3 r = xyz_to_srgb_linear(mapped(1.0f));
    V3 resolved = v3(fmaxf(r.x, 0.0f), fmaxf(r.y, 0.0f), fmaxf(r.z, 0.0f));
    for (uint32_t i = 0; i <= 32; ++i) {
        float t = (float)i / 32.0f;
        V3 cand = xyz_to_srgb_linear(mapped(t));
        if (in_range(cand, mx)) {
            resolved = cand;
            break;
        }
    }
    return resolved;
}

// optics/raytracer/color.rs:365-372
__device__ __forceinline__ float aces(float y) {
    return (y * fmaf(2.51f, y, 0.03f)) / fmaf(y, fmaf(2.43f, y, 0.59f), 0.14f);
}

// color/space.rs:20-30 (sRGB transfer) then the `as u8` truncation of space.rs:318-326.
__device__ __forceinline__ unsigned char encode_channel(float c) {
    float lin = isfinite(c) ? fminf(fmaxf(c, 0.0f), 1.0f) : 0.0f;
    float enc = lin <= 0.0031308f ? lin * 12.92f : fmaf(1.055f, powf(lin, 1.0f / 2.4f), -0.055f);
    enc = fminf(fmaxf(enc, 0.0f), 1.0f);
    float v = enc * 255.0f;
    return (unsigned char)(v >= 255.0f ? 255 : (v > 0.0f ? (int)v : 0));
}

__global__ void k_tonemap(const float *__restrict__ xyz, float scale, uint32_t n, uchar4 *__restrict__ rgba) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 c = v3(xyz[3 * (size_t)i] * scale, xyz[3 * (size_t)i + 1] * scale, xyz[3 * (size_t)i + 2] * scale);
    uchar4 out = make_uchar4(0, 0, 0, 255);
    float sum = c.x + c.y + c.z;
    if (isfinite(sum) && sum > 1e-6f) {
        const float exposure = 1.0f;
        float lum = fmaxf(c.y, 0.0f);
        float el = fmaxf(lum * exposure, 0.0f);
        float ytm = aces(el);
        float ls = (ytm / fmaxf(el, 1e-5f)) * exposure;
        V3 toned = project_to_gamut_bounded(mul(c, ls), 1.0f);
        out.x = encode_channel(toned.x);
        out.y = encode_channel(toned.y);
        out.z = encode_channel(toned.z);
    }
    rgba[i] = out;
}

}  // namespace grd

namespace grh {
gr_status tonemap_device(const float *xyz_dev, float scale, uint32_t n, void *rgba_dev, cudaStream_t s) {
    if (n == 0) return GR_OK;
    const unsigned threads = 256;
    grd::k_tonemap<<<(n + threads - 1) / threads, threads, 0, s>>>(xyz_dev, scale, n, (uchar4 *)rgba_dev);
    return cudaGetLastError() == cudaSuccess ? GR_OK : GR_ECUDA;
}
}  // namespace grh
