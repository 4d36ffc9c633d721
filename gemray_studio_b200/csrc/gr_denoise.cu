// gr_denoise.cu -- the denoiser's guide pass and the edge-avoiding A-Trous filter.
//
// Guide pass (apps/diagram-gui/src/bridge/guide_pass.rs, generate_guide_buffers): one
// thread per pixel casts the primary ray through the pixel's corner (zero jitter) at
// the stone, through the transport kernels' plane scan, and writes (t, hit normal,
// facet index) or (1e6, 0, -1) on a miss.
//
// A-Trous (crates/gemray/src/renderer/denoise/mod.rs:154-690): 1..8 passes of a 5x5 B3
// spline kernel dilated by 2^pass, each tap gated by facet identity, a normal cosine
// power, a depth term and a colour term whose sigma tapers with the sample count; a
// pass is one thread per output pixel reading the previous pass's image (L2-resident:
// a 1080p image and its guides are ~60 MB).  Tap arithmetic follows atrous_pixel
// (:383-444) operation for operation; the depth and colour terms call CUDA's expf.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "gr_ctx.h"
#include "gr_launch.cuh"

using grh::fail;

namespace grd {

__global__ void __launch_bounds__(128) k_guide_pass(SceneConst S, const float4 *__restrict__ gplanes,
                                                    float *__restrict__ depth, float *__restrict__ normal,
                                                    int32_t *__restrict__ facet) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, gplanes, S.n_planes);
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)S.width * S.height) return;
    const uint32_t x = (uint32_t)(i % S.width), y = (uint32_t)(i / S.width);
    const float aspect = S.width_f / S.height_f;
    const float u = (((float)x + 0.0f) / S.width_f - 0.5f) * 2.0f * aspect * S.fov_tan;
    const float v = (0.5f - ((float)y + 0.0f) / S.height_f) * 2.0f * S.fov_tan;
    const V3 dir = normalize(add(add(ld3(S.cam_f), mul(ld3(S.cam_r), u)), mul(ld3(S.cam_u), v)));
    float t = 0.0f;
    int idx = -1;
    float d = 1.0e6f;
    V3 n = v3(0.f, 0.f, 0.f);
    int32_t f = -1;
    if (intersect<false>(PL, ld3(S.cam_o), dir, t, idx)) {
        d = t;
        if (idx >= 0) {  // an empty plane set hits at t = 1e30 with the zero normal, facet 0
            const float4 p = PL.aos[idx];
            n = v3(p.x, p.y, p.z);
        }
        f = idx >= 0 ? idx : 0;
    }
    depth[i] = d;
    normal[3 * i + 0] = n.x;
    normal[3 * i + 1] = n.y;
    normal[3 * i + 2] = n.z;
    facet[i] = f;
}

__device__ __forceinline__ float sanitize(float v) { return isfinite(v) ? v : 0.0f; }

// unit_normal_or_zero (:268-276), and the colour input scaled (accum * (1 / count) in
// denoise_and_tonemap_frame) or copied.
__global__ void k_denoise_prep(const float *__restrict__ normal, float *__restrict__ nn, const float *__restrict__ film,
                               float *__restrict__ color, float inv_count, uint32_t scale, uint64_t n_px) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_px) return;
    const V3 n = v3(sanitize(normal[3 * i]), sanitize(normal[3 * i + 1]), sanitize(normal[3 * i + 2]));
    const float l = sqrtf(dot(n, n));
    const bool z = l <= 1.0e-8f;
    nn[3 * i + 0] = z ? 0.0f : n.x / l;
    nn[3 * i + 1] = z ? 0.0f : n.y / l;
    nn[3 * i + 2] = z ? 0.0f : n.z / l;
    if (film) {
        for (int c = 0; c < 3; ++c) color[3 * i + c] = scale ? film[3 * i + c] * inv_count : film[3 * i + c];
    }
}

// cos_pow (:294-311): repeated squaring for power-of-two integer exponents, else powf.
__device__ __forceinline__ float cos_pow(float base, float power, uint32_t squarings, bool pow2) {
    if (pow2) {
        float v = base;
        for (uint32_t k = 0; k < squarings; ++k) v *= v;
        return v;
    }
    return powf(base, power);
}

struct AtrousConst {
    uint32_t w, h;
    float nisd, nits, power;
    uint32_t squarings, pow2;
};

__global__ void __launch_bounds__(128) k_atrous_pass(AtrousConst A, const float *__restrict__ src,
                                                     float *__restrict__ dst, const float *__restrict__ depth,
                                                     const float *__restrict__ nn, const int32_t *__restrict__ facet,
                                                     int stride) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (uint64_t)A.w * A.h) return;
    const int64_t y = (int64_t)(c / A.w), x = (int64_t)(c % A.w);
    const float B3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    const V3 cc = v3(src[3 * c], src[3 * c + 1], src[3 * c + 2]);
    const V3 scc = v3(sanitize(cc.x), sanitize(cc.y), sanitize(cc.z));
    const V3 cn = v3(nn[3 * c], nn[3 * c + 1], nn[3 * c + 2]);
    const bool cn_zero = cn.x == 0.0f && cn.y == 0.0f && cn.z == 0.0f;
    const float cdep = sanitize(depth[c]);
    const int32_t cf = facet[c];
    V3 sum = v3(0.f, 0.f, 0.f);
    float wsum = 0.0f;
#pragma unroll
    for (int ky = 0; ky < 5; ++ky) {
        const int64_t sy = y + (int64_t)(ky - 2) * stride;
        if (sy < 0 || sy >= (int64_t)A.h) continue;
#pragma unroll
        for (int kx = 0; kx < 5; ++kx) {
            const int64_t sx = x + (int64_t)(kx - 2) * stride;
            if (sx < 0 || sx >= (int64_t)A.w) continue;
            const uint64_t q = (uint64_t)sy * A.w + (uint64_t)sx;
            if (facet[q] != cf) continue;  // facet_weight 0: the tap is skipped
            const float kw = B3[ky] * B3[kx];
            const V3 qn = v3(nn[3 * q], nn[3 * q + 1], nn[3 * q + 2]);
            float wn = 1.0f;
            if (!cn_zero && !(qn.x == 0.0f && qn.y == 0.0f && qn.z == 0.0f))
                wn = cos_pow(fmaxf(clampf(dot(cn, qn), -1.0f, 1.0f), 0.0f), A.power, A.squarings, A.pow2 != 0);
            const float wd = expf(fabsf(cdep - sanitize(depth[q])) * A.nisd);
            const V3 qc = v3(src[3 * q], src[3 * q + 1], src[3 * q + 2]);
            const V3 dc = v3(scc.x - sanitize(qc.x), scc.y - sanitize(qc.y), scc.z - sanitize(qc.z));
            const float wc = expf(dot(dc, dc) * A.nits);
            const float wgt = ((kw * wn) * wd) * wc;  // kernel_w * wf * wn * wd * wc with wf = 1
            sum = add(sum, mul(qc, wgt));
            wsum = wsum + wgt;
        }
    }
    if (wsum > 1.0e-8f) {
        dst[3 * c + 0] = sum.x / wsum;
        dst[3 * c + 1] = sum.y / wsum;
        dst[3 * c + 2] = sum.z / wsum;
    } else {
        dst[3 * c + 0] = cc.x;
        dst[3 * c + 1] = cc.y;
        dst[3 * c + 2] = cc.z;
    }
}

}  // namespace grd

namespace {

gr_atrous_params default_params() {  // AtrousParams::default (:210-221)
    gr_atrous_params p;
    p.num_passes = 5;
    p.sigma_color = 0.35f;
    p.sigma_depth = 0.1f;
    p.normal_power = 64.0f;
    p.taper_reference_spp = 4.0f;
    p.taper_identity_epsilon = 0.02f;
    return p;
}

// The filter on device buffers; color_in is either the averaged image or (film,
// inv_count) to be scaled first.  out may alias neither input.
gr_status atrous_device(gr_ctx *ctx, const float *color_in, const float *film, float inv_count, const float *depth,
                        const float *normal, const int32_t *facet, uint32_t w, uint32_t h, uint32_t spp,
                        const gr_atrous_params *params_in, float *out, cudaStream_t s) {
    const uint64_t n_px = (uint64_t)w * h;
    if (n_px == 0) return GR_OK;
    const gr_atrous_params P = params_in ? *params_in : default_params();
    const size_t img = (size_t)n_px * 3 * sizeof(float);
    const float n0 = P.taper_reference_spp > 1.0e-8f ? P.taper_reference_spp : 1.0e-8f;
    const float taper = 1.0f / sqrtf(1.0f + (float)spp / n0);  // taper_strength (:244-250)
    const unsigned threads = 128;
    const unsigned blocks = (unsigned)((n_px + threads - 1) / threads);
    gr_status st = ctx->dn_a.reserve(img);
    if (st == GR_OK) st = ctx->dn_b.reserve(img);
    if (st == GR_OK) st = ctx->dn_n.reserve(img);
    if (st != GR_OK) return st;
    float *a = (float *)ctx->dn_a.ptr, *b = (float *)ctx->dn_b.ptr, *nn = (float *)ctx->dn_n.ptr;
    grd::k_denoise_prep<<<blocks, threads, 0, s>>>(normal, nn, film ? film : color_in, a, inv_count,
                                                   film ? 1u : 0u, n_px);
    GR_CUDA(cudaGetLastError());
    if (taper < P.taper_identity_epsilon) {  // the identity short-circuit: a plain copy
        GR_CUDA(cudaMemcpyAsync(out, a, img, cudaMemcpyDeviceToDevice, s));
        return GR_OK;
    }
    const uint32_t passes = P.num_passes < 1 ? 1 : (P.num_passes > 8 ? 8 : P.num_passes);
    const float sce = fmaxf(P.sigma_color * taper, 0.0f);
    const float sd = fmaxf(P.sigma_depth, 1.0e-8f);
    const float scs = fmaxf(sce * sce, 1.0e-8f);
    grd::AtrousConst A;
    A.w = w;
    A.h = h;
    A.nisd = -1.0f / sd;
    A.nits = -1.0f / (2.0f * scs);
    A.power = fmaxf(P.normal_power, 0.0f);
    A.pow2 = 0;
    A.squarings = 0;
    if (A.power == floorf(A.power) && A.power <= 4294967295.0f) {
        const uint32_t ip = (uint32_t)A.power;
        if (ip != 0 && (ip & (ip - 1)) == 0) {
            A.pow2 = 1;
            for (uint32_t k = ip; k > 1; k >>= 1) A.squarings++;
        }
    }
    for (uint32_t pass = 0; pass < passes; ++pass) {
        float *dst = pass + 1 == passes ? out : b;
        grd::k_atrous_pass<<<blocks, threads, 0, s>>>(A, a, dst, depth, nn, facet, 1 << pass);
        GR_CUDA(cudaGetLastError());
        if (pass + 1 < passes) {
            float *t = a;
            a = b;
            b = t;
        }
    }
    return GR_OK;
}

// The guide pass reads only the scene's camera, frame size and planes.  Runs on the
// context stream (its plane buffer is the context's); the caller holds ctx->mu.
gr_status guide_device(gr_ctx *ctx, const gr_scene *sc, float *depth, float *normal, int32_t *facet) {
    if (sc->n_planes > GR_MAX_PLANES) return fail(GR_EINVAL, "n_planes %u exceeds %u", sc->n_planes, GR_MAX_PLANES);
    if (sc->n_planes && !sc->planes) return fail(GR_EINVAL, "planes is NULL");
    const uint64_t n_px = (uint64_t)sc->width * sc->height;
    if (n_px == 0) return GR_OK;
    SceneConst S;
    std::memset(&S, 0, sizeof(S));
    for (int i = 0; i < 3; ++i) {
        S.cam_o[i] = sc->camera.origin[i];
        S.cam_f[i] = sc->camera.forward[i];
        S.cam_r[i] = sc->camera.right[i];
        S.cam_u[i] = sc->camera.up[i];
    }
    S.fov_tan = sc->camera.fov_tan;
    S.width = sc->width;
    S.height = sc->height;
    S.width_f = (float)sc->width;
    S.height_f = (float)sc->height;
    S.n_planes = sc->n_planes;
    gr_status st = ctx->dn_planes.reserve((size_t)(sc->n_planes ? sc->n_planes : 1) * sizeof(float4));
    if (st != GR_OK) return st;
    if (sc->n_planes)
        GR_CUDA(cudaMemcpyAsync(ctx->dn_planes.ptr, sc->planes, sc->n_planes * sizeof(gr_plane), cudaMemcpyHostToDevice,
                                ctx->stream));
    const unsigned threads = 128;
    grd::k_guide_pass<<<(unsigned)((n_px + threads - 1) / threads), threads, grd::planes_smem_bytes(S.n_planes),
                        ctx->stream>>>(S, (const float4 *)ctx->dn_planes.ptr, depth, normal, facet);
    GR_CUDA(cudaGetLastError());
    // the host planes are copied from pageable memory: wait before the caller may free them
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

// Device-pointer entry points run on the context stream (their scratch is the
// context's) ordered after the caller's stream, and the caller's stream after them.
gr_status join_in(gr_ctx *ctx, cudaStream_t user) {
    if (!user || user == ctx->stream) return GR_OK;
    if (!ctx->dn_ev) GR_CUDA(cudaEventCreateWithFlags(&ctx->dn_ev, cudaEventDisableTiming));
    GR_CUDA(cudaEventRecord(ctx->dn_ev, user));
    GR_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->dn_ev, 0));
    return GR_OK;
}
gr_status join_out(gr_ctx *ctx, cudaStream_t user) {
    if (!user || user == ctx->stream) return GR_OK;
    GR_CUDA(cudaEventRecord(ctx->dn_ev, ctx->stream));
    GR_CUDA(cudaStreamWaitEvent(user, ctx->dn_ev, 0));
    return GR_OK;
}

}  // namespace

extern "C" {

gr_status gr_guide_buffers(gr_ctx *ctx, const gr_scene *sc, float *depth, float *normal, int32_t *facet_id) {
    if (!ctx || !sc) return fail(GR_EINVAL, "ctx or scene is NULL");
    const uint64_t n_px = (uint64_t)sc->width * sc->height;
    if (n_px == 0) return GR_OK;
    if (!depth || !normal || !facet_id) return fail(GR_EINVAL, "output buffer is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    gr_status st = ctx->dn_g.reserve((size_t)n_px * 5 * sizeof(float));
    if (st != GR_OK) return st;
    float *dd = (float *)ctx->dn_g.ptr, *dn = dd + n_px;
    int32_t *df = (int32_t *)(dn + 3 * n_px);
    st = guide_device(ctx, sc, dd, dn, df);
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemcpyAsync(depth, dd, n_px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(normal, dn, n_px * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(facet_id, df, n_px * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_guide_buffers_device(gr_ctx *ctx, const gr_scene *sc, float *depth, float *normal, int32_t *facet_id,
                                  void *stream) {
    if (!ctx || !sc) return fail(GR_EINVAL, "ctx or scene is NULL");
    if ((uint64_t)sc->width * sc->height == 0) return GR_OK;
    if (!depth || !normal || !facet_id) return fail(GR_EINVAL, "output buffer is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    gr_status st = join_in(ctx, (cudaStream_t)stream);
    if (st == GR_OK) st = guide_device(ctx, sc, depth, normal, facet_id);
    if (st == GR_OK) st = join_out(ctx, (cudaStream_t)stream);
    return st;
}

gr_status gr_atrous_denoise(gr_ctx *ctx, const float *color, const float *depth, const float *normal,
                            const int32_t *facet_id, uint32_t width, uint32_t height, uint32_t spp,
                            const gr_atrous_params *params, float *out) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    const uint64_t n_px = (uint64_t)width * height;
    if (n_px == 0) return GR_OK;
    if (!color || !depth || !normal || !facet_id || !out) return fail(GR_EINVAL, "buffer is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    const size_t img = (size_t)n_px * 3 * sizeof(float);
    gr_status st = ctx->dn_in.reserve(2 * img + (size_t)n_px * (sizeof(float) + sizeof(int32_t)) + img);
    if (st != GR_OK) return st;
    float *dc = (float *)ctx->dn_in.ptr, *dn = dc + 3 * n_px, *dd = dn + 3 * n_px;
    int32_t *df = (int32_t *)(dd + n_px);
    float *dout = (float *)(df + n_px);
    cudaStream_t s = ctx->stream;
    GR_CUDA(cudaMemcpyAsync(dc, color, img, cudaMemcpyHostToDevice, s));
    GR_CUDA(cudaMemcpyAsync(dn, normal, img, cudaMemcpyHostToDevice, s));
    GR_CUDA(cudaMemcpyAsync(dd, depth, n_px * sizeof(float), cudaMemcpyHostToDevice, s));
    GR_CUDA(cudaMemcpyAsync(df, facet_id, n_px * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    st = atrous_device(ctx, dc, nullptr, 1.0f, dd, dn, df, width, height, spp, params, dout, s);
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemcpyAsync(out, dout, img, cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    return GR_OK;
}

gr_status gr_atrous_denoise_device(gr_ctx *ctx, const float *color, const float *depth, const float *normal,
                                   const int32_t *facet_id, uint32_t width, uint32_t height, uint32_t spp,
                                   const gr_atrous_params *params, float *out, void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if ((uint64_t)width * height == 0) return GR_OK;
    if (!color || !depth || !normal || !facet_id || !out) return fail(GR_EINVAL, "buffer is NULL");
    if (out == color) return fail(GR_EINVAL, "out must not alias color");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    gr_status st = join_in(ctx, (cudaStream_t)stream);
    if (st == GR_OK)
        st = atrous_device(ctx, color, nullptr, 1.0f, depth, normal, facet_id, width, height, spp, params, out,
                           ctx->stream);
    if (st == GR_OK) st = join_out(ctx, (cudaStream_t)stream);
    return st;
}

gr_status gr_denoise_tonemap_device(gr_ctx *ctx, const float *film, uint32_t sample_count, const float *depth,
                                    const float *normal, const int32_t *facet_id, uint32_t width, uint32_t height,
                                    const gr_atrous_params *params, void *rgba, void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    const uint64_t n_px = (uint64_t)width * height;
    if (n_px == 0) return GR_OK;
    if (!film || !depth || !normal || !facet_id || !rgba) return fail(GR_EINVAL, "buffer is NULL");
    if (n_px > 0xFFFFFFFFull) return fail(GR_EINVAL, "frame too large");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    gr_status st = ctx->dn_out.reserve((size_t)n_px * 3 * sizeof(float));
    if (st == GR_OK) st = join_in(ctx, (cudaStream_t)stream);
    if (st != GR_OK) return st;
    const float inv = 1.0f / (float)sample_count;  // denoise.rs: 1.0 / current_sample_count as f32
    st = atrous_device(ctx, nullptr, film, inv, depth, normal, facet_id, width, height, sample_count, params,
                       (float *)ctx->dn_out.ptr, s);
    if (st == GR_OK) st = grh::tonemap_device((const float *)ctx->dn_out.ptr, 1.0f, (uint32_t)n_px, rgba, s);
    if (st == GR_OK) st = join_out(ctx, (cudaStream_t)stream);
    return st;
}

}  // extern "C"
