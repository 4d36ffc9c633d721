// gr_stokes.cu -- the Stokes film: the polarisation state of the light a render
// collects, beside its XYZ film (gr_accumulate_stokes).
//
// The reference's film is XYZ only (renderer/gpu/frame.rs:799-814); its transport
// carries a Stokes vector per hero-wavelength channel (optics/polarization.rs:4-66
// StokesVector, spectral_transport.wgsl transport_main's per-channel state) and drops
// it at the end of the path.  The Stokes variant of the plain kernel keeps it: per
// tuple the luminance-weighted Stokes vector of the escaping light (path_finish<.., true>,
// gr_trace.cuh), folded per pixel in sample order like the XYZ film.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "gr_ctx.h"
#include "gr_launch.cuh"

using grh::fail;

namespace grd {

// The plain kernel writing XYZ (the same arithmetic as k_trace_plain) and IQUV per tuple.
template <bool EXTRAS>
__global__ void __launch_bounds__(TRACE_THREADS, GR_TRACE_MIN_BLOCKS) k_trace_stokes(SceneConst S, SceneBuffers B,
                                                                                     LaunchRange R,
                                                                                     float *__restrict__ xyz,
                                                                                     float4 *__restrict__ iquv) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= R.n_tuples) return;
    uint32_t pixel, sample;
    tuple_coords(R, t, pixel, sample);
    Path P;
    path_init<1, EXTRAS>(P, S, B, pixel, sample, (uint32_t)t);
    NoCounters nc;
    while (state_bits(P) & F_ALIVE) {
        Event E;
        const uint32_t ev = step_hit<1, NoCounters, false, EXTRAS>(P, S, PL, E, nc);
        if (ev == EV_REFLECT) step_reflect<1, NoCounters, EXTRAS>(P, S, E, nc);
        else if (ev == EV_REFRACT) step_refract<1, NoCounters, EXTRAS>(P, S, E, nc);
    }
    float4 s4;
    const V3 c = path_finish<1, true>(P, S, B, &s4);
    xyz[3 * t + 0] = c.x;
    xyz[3 * t + 1] = c.y;
    xyz[3 * t + 2] = c.z;
    iquv[t] = s4;
}

// One warp per pixel: the pixel's spp Stokes vectors summed in sample order from zero,
// the sum added once to the film (the XYZ fold's add mode, fold_pixel).
__global__ void k_stokes_fold(const float4 *__restrict__ iquv, uint32_t n_pixels, uint32_t spp, uint32_t first_pixel,
                              float4 *__restrict__ film) {
    const uint64_t px = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (px >= n_pixels) return;
    const uint32_t lane = threadIdx.x & 31u;
    const float4 *src = iquv + px * spp;
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t s0 = 0; s0 < spp; s0 += 32) {
        const float4 v = s0 + lane < spp ? src[s0 + lane] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const uint32_t cnt = spp - s0 < 32u ? spp - s0 : 32u;
        for (uint32_t j = 0; j < cnt; ++j) {
            s.x = s.x + __shfl_sync(0xffffffffu, v.x, j);
            s.y = s.y + __shfl_sync(0xffffffffu, v.y, j);
            s.z = s.z + __shfl_sync(0xffffffffu, v.z, j);
            s.w = s.w + __shfl_sync(0xffffffffu, v.w, j);
        }
    }
    if (lane == 0) {
        float4 &f = film[first_pixel + px];
        f = make_float4(f.x + s.x, f.y + s.y, f.z + s.z, f.w + s.w);
    }
}

}  // namespace grd

extern "C" {

gr_status gr_accumulate_stokes(gr_ctx *ctx, const gr_scene *sc, uint32_t sample_offset, uint32_t spp,
                               float *accum_xyz, float *accum_stokes) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!sc) return fail(GR_EINVAL, "scene is NULL");
    const uint64_t n_pixels = (uint64_t)sc->width * sc->height;
    if (spp == 0 || n_pixels == 0) return GR_OK;
    if (!accum_xyz || !accum_stokes) return fail(GR_EINVAL, "accum_xyz or accum_stokes is NULL");
    if (sc->flags & GR_FLAG_FP64_RESOLVE) return fail(GR_EINVAL, "the Stokes film has no FP64 re-solve variant");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    // films: XYZ then IQUV (16-byte aligned); per-tuple scratch: XYZ then IQUV
    const size_t xbytes = (size_t)n_pixels * 12, sbytes = (size_t)n_pixels * 16, soff = (xbytes + 255) & ~(size_t)255;
    st = ctx->film.reserve(soff + sbytes);
    if (st != GR_OK) return st;
    float *film_x = (float *)ctx->film.ptr;
    float4 *film_s = (float4 *)((char *)ctx->film.ptr + soff);
    GR_CUDA(cudaMemcpyAsync(film_x, accum_xyz, xbytes, cudaMemcpyHostToDevice, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(film_s, accum_stokes, sbytes, cudaMemcpyHostToDevice, ctx->stream));
    uint64_t budget = ctx->chunk_budget / 28;  // 12 B of XYZ + 16 B of IQUV per tuple
    if (budget > 0xFFFFFFFFull) budget = 0xFFFFFFFFull;
    uint64_t chunk_pixels = budget / spp;
    if (chunk_pixels < 1) chunk_pixels = 1;
    if (chunk_pixels > n_pixels) chunk_pixels = n_pixels;
    const uint64_t chunk_tuples = chunk_pixels * spp;
    const size_t toff = (chunk_tuples * 12 + 255) & ~(size_t)255;
    st = ctx->xyz.reserve(toff + chunk_tuples * 16);
    if (st != GR_OK) return st;
    float *txyz = (float *)ctx->xyz.ptr;
    float4 *tiquv = (float4 *)((char *)ctx->xyz.ptr + toff);
    const size_t smem = grd::planes_smem_bytes(S.n_planes);
    for (uint64_t first = 0; first < n_pixels; first += chunk_pixels) {
        const uint64_t np = n_pixels - first < chunk_pixels ? n_pixels - first : chunk_pixels;
        grd::LaunchRange R;
        R.first_pixel = (uint32_t)first;
        R.n_pixels = (uint32_t)np;
        R.sample_offset = sample_offset;
        R.spp = spp;
        R.n_tuples = np * spp;
        const unsigned blocks = (unsigned)((R.n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
        if (grd::needs_extras(S))
            grd::k_trace_stokes<true><<<blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(S, B, R, txyz, tiquv);
        else
            grd::k_trace_stokes<false><<<blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(S, B, R, txyz, tiquv);
        GR_CUDA(cudaGetLastError());
        ctx->trace_launches += 1;
        st = grh::launch_fold(txyz, (uint32_t)np, spp, (uint32_t)first, film_x, (S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u,
                              ctx->stream);
        if (st != GR_OK) return st;
        const unsigned fb = (unsigned)((np * 32 + 255) / 256);
        grd::k_stokes_fold<<<fb, 256, 0, ctx->stream>>>(tiquv, (uint32_t)np, spp, (uint32_t)first, film_s);
        GR_CUDA(cudaGetLastError());
        ctx->fold_launches += 2;
    }
    // stage both films on the host first, so a failure leaves the caller's buffers untouched
    std::vector<float> tx(n_pixels * 3), ts(n_pixels * 4);
    GR_CUDA(cudaMemcpyAsync(tx.data(), film_x, xbytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(ts.data(), film_s, sbytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(accum_xyz, tx.data(), xbytes);
    std::memcpy(accum_stokes, ts.data(), sbytes);
    return GR_OK;
}

}  // extern "C"
