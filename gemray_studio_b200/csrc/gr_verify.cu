// gr_verify.cu -- verification entry points of the engine: per-tuple event sequences
// of the transport (gr_trace_events), per-function case banks over the device
// functions the transport kernels inline (gr_case_bank) and the convex-clip ray bank
// (gr_intersect_rays).  The reference verifies its GPU port the same three ways: an
// instrumented trace (optics/raytracer/transport.rs:512-537), Tier-2 per-function ULP
// banks (renderer/gpu/transport_check/mod.rs:38-75, camera_check.rs,
// environment_check.rs) and the intersect_polyhedron case bank with its tie rule
// (renderer/gpu/polyhedron_check.rs:15-61).  Every kernel here calls the transport's
// own functions, so what is checked is what renders.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "gr_ctx.h"
#include "gr_launch.cuh"

using grh::fail;

namespace grd {

// The plain kernel's body with the recording hooks (EventRec): each tuple's facets,
// hit distances and events, and how its path ended.
template <bool EXTRAS>
__global__ void __launch_bounds__(TRACE_THREADS) k_trace_events(SceneConst S, SceneBuffers B, LaunchRange R,
                                                                EventRec rec) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, B.planes, S.n_planes);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= R.n_tuples) return;
    EventRec r = rec;
    r.t = t;
    for (uint32_t b = 0; b < r.kmax; ++b) {
        r.facets[t * r.kmax + b] = -1;
        r.ts[t * r.kmax + b] = 0.0f;
        r.events[t * r.kmax + b] = (uint8_t)GR_SEQ_NONE;
    }
    r.bounces[t] = S.max_bounces;  // overwritten by an escape or a roulette kill
    r.term[t] = GR_TERM_HIT_CAP;
    uint32_t pixel, sample;
    tuple_coords(R, t, pixel, sample);
    Path P;
    path_init<1, EXTRAS>(P, S, B, pixel, sample, (uint32_t)t);
    while (state_bits(P) & F_ALIVE) {
        Event E;
        const uint32_t ev = step_hit<1, EventRec, false, EXTRAS>(P, S, PL, E, r);
        if (ev == EV_REFLECT) step_reflect<1, EventRec, EXTRAS>(P, S, E, r);
        else if (ev == EV_REFRACT) step_refract<1, EventRec, EXTRAS>(P, S, E, r);
    }
}

// Inputs and outputs per case of each bank (the GR_BANK_* layouts of gemray_cuda.h).
constexpr uint32_t kBankArity[GR_BANK_COUNT][2] = {
    {4, 3}, {1, 3}, {1, 1}, {1, 1}, {1, 2}, {12, 1}, {6, 4}, {10, 4}, {5, 4}, {5, 4}, {9, 1}, {3, 1},
    {6, 6}, {8, 3}, {3, 1}, {9, 1}, {4, 1}, {4, 1}, {1, 1}, {6, 3}, {5, 3}, {10, 3}, {3, 3}, {1, 8},
};

// One case per thread through the device function the transport inlines.
__global__ void k_case_bank(uint32_t bank, SceneConst S, SceneBuffers B, const float *__restrict__ in, uint32_t n,
                            uint32_t ni, uint32_t no, float *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *x = in + (size_t)i * ni;
    float *y = out + (size_t)i * no;
    auto v = [&](int j) { return v3(x[j], x[j + 1], x[j + 2]); };
    auto st = [&](int j) { return Stokes{x[j], x[j + 1], x[j + 2], x[j + 3]}; };
    auto put3 = [&](V3 a, int o) { y[o] = a.x; y[o + 1] = a.y; y[o + 2] = a.z; };
    auto put4 = [&](const Stokes &a) { y[0] = a.i; y[1] = a.q; y[2] = a.u; y[3] = a.v; };
    switch (bank) {
    case GR_BANK_CAMERA_RAY: put3(camera_dir(S, x[0], x[1], x[2], x[3]), 0); break;
    case GR_BANK_CMF: put3(cmf(x[0]), 0); break;
    case GR_BANK_BLACKBODY: y[0] = blackbody(S, x[0]); break;
    case GR_BANK_DISPERSION: y[0] = dispersion(S, x[0]); break;
    case GR_BANK_ABSORPTION:
        if (S.ext_n > 0) {
            y[0] = table_lookup(B.ext_alpha_o, S.ext_n, S.ext_first, S.ext_step, x[0]);
            y[1] = table_lookup(B.ext_alpha_e, S.ext_n, S.ext_first, S.ext_step, x[0]);
        } else {
            y[0] = band_sum(S.o_bands, S.n_o_bands, x[0]);
            y[1] = band_sum(S.e_bands, S.n_e_bands, x[0]);
        }
        break;
    case GR_BANK_PLEOCHROIC: {
        // the uniaxial eigenmodes and E-field of step_hit's interior segment
        const Stokes s = st(0);
        const V3 kk = v(7);
        const V3 ea = ordinary_eigen(kk, ld3(S.c_axis));
        const V3 eb = extraordinary_eigen_from(kk, ea);
        const V3 e_hat = electric_field_direction(s, v(4), kk);
        y[0] = pleochroic_alpha(S, x[10], x[11], s, e_hat, ea, eb);
        break;
    }
    case GR_BANK_FRESNEL_REFLECTION: {
        float a, b, c;
        fresnel_reflection_abc(x[0], x[1], a, b, c);
        put4(apply_fresnel(st(2), a, b, c));
        break;
    }
    case GR_BANK_FRESNEL_TRANSMISSION: {
        float a, b, c;
        fresnel_transmission_abc(x[0], x[1], x[2], x[3], x[4], x[5], a, b, c);
        put4(apply_fresnel(st(6), a, b, c));
        break;
    }
    case GR_BANK_FRAME_ROTATION: {
        const float2 sc = m_sincos(2.0f * x[0]);
        put4(apply_rotation(st(1), sc.y, sc.x));
        break;
    }
    case GR_BANK_TIR_RETARDATION: {
        const float2 sc = m_sincos(x[0]);
        put4(apply_tir(st(1), sc.y, sc.x));
        break;
    }
    case GR_BANK_SIGNED_PSI: y[0] = signed_psi(v(0), v(3), v(6)); break;
    case GR_BANK_TIR_PHASE_DELTA: y[0] = tir_phase_delta(x[0], x[1], x[2]); break;
    case GR_BANK_EIGEN_UNIAXIAL: {
        const V3 o = ordinary_eigen(v(0), v(3));
        put3(o, 0);
        put3(extraordinary_eigen_from(v(0), o), 3);
        break;
    }
    case GR_BANK_WALK_OFF: put3(extraordinary_poynting_dir(v(0), v(3), x[6], x[7]), 0); break;
    case GR_BANK_EXTRAORDINARY_INDEX: {
        const float2 sc = m_sincos(x[2]);
        y[0] = eff_e_index(x[0], x[1], sc.x, sc.y);
        break;
    }
    case GR_BANK_THETA_C: {
        const V3 kk = v(0), normal = v(3);
        const float cos_i = clampf(dot(neg(kk), normal), 0.0f, 1.0f);
        y[0] = theta_c<1>(kk, normal, cos_i, fmaf(cos_i, -cos_i, 1.0f), x[6], x[7], ld3(S.c_axis), x[8] != 0.0f);
        break;
    }
    case GR_BANK_STUDIO: y[0] = studio_radiance(S, normalize(v(0)), x[3]); break;
    case GR_BANK_RGB_SPECTRAL: y[0] = rgb_to_spectral(x[0], x[1], x[2], x[3]); break;
    case GR_BANK_EXP_POLY: y[0] = exp_poly(x[0]); break;
    case GR_BANK_HG_SAMPLE: put3(sample_hg_direction(x[0], x[1], x[2], v(3)), 0); break;
    case GR_BANK_COSINE_HEMISPHERE: put3(cosine_weighted_hemisphere(x[0], x[1], v(2)), 0); break;
    case GR_BANK_E_FIELD: put3(electric_field_direction(st(0), v(4), v(7)), 0); break;
    case GR_BANK_VON_KRIES: put3(von_kries(v(0), S.wb), 0); break;
    case GR_BANK_WAVELENGTHS:
        for (int k = 0; k < NCH; ++k) y[k] = lambda_k(x[0], k);
        break;
    default: break;
    }
}

// The transport's clip (paired shared-memory scan) for one ray per thread.
__global__ void k_intersect_rays(const float4 *__restrict__ planes, uint32_t n_planes, const float *__restrict__ rays,
                                 uint32_t n, float *__restrict__ t_out, int32_t *__restrict__ facet_out) {
    extern __shared__ float4 s_planes[];
    const Planes PL = stage_plane_set(s_planes, planes, n_planes);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rays + 6 * (size_t)i;
    float t = 0.0f;
    int idx = -1;
    const bool hit = intersect<false>(PL, v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), t, idx);
    t_out[i] = hit ? t : 0.0f;
    facet_out[i] = hit ? idx : -1;
}

}  // namespace grd

namespace {
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

extern "C" {

gr_status gr_trace_events(gr_ctx *ctx, const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels,
                          uint32_t sample_offset, uint32_t spp, uint32_t kmax, uint32_t *bounces,
                          uint32_t *termination, int32_t *facets, float *t_hits, uint8_t *events) {
    if (!ctx || !sc) return fail(GR_EINVAL, "ctx or scene is NULL");
    if (n_pixels == 0 || spp == 0) return GR_OK;
    if (!bounces || !termination || (kmax && (!facets || !t_hits || !events))) return fail(GR_EINVAL, "NULL output");
    if ((uint64_t)first_pixel + n_pixels > (uint64_t)sc->width * sc->height)
        return fail(GR_EINVAL, "pixel range exceeds the frame");
    const uint64_t n = (uint64_t)n_pixels * spp;
    if (n > (1ull << 26) || (uint64_t)kmax * n > (1ull << 28)) return fail(GR_EINVAL, "too many tuples for one call");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    const size_t o_term = align256(n * 4), o_fac = o_term + align256(n * 4), o_ts = o_fac + align256(n * kmax * 4),
                 o_ev = o_ts + align256(n * kmax * 4), total = o_ev + align256(n * kmax + 1);
    st = ctx->xyz.reserve(total);
    if (st != GR_OK) return st;
    char *base = (char *)ctx->xyz.ptr;
    grd::EventRec rec;
    rec.bounces = (uint32_t *)base;
    rec.term = (uint32_t *)(base + o_term);
    rec.facets = (int32_t *)(base + o_fac);
    rec.ts = (float *)(base + o_ts);
    rec.events = (uint8_t *)(base + o_ev);
    rec.kmax = kmax;
    rec.t = 0;
    grd::LaunchRange R;
    R.first_pixel = first_pixel;
    R.n_pixels = n_pixels;
    R.sample_offset = sample_offset;
    R.spp = spp;
    R.n_tuples = n;
    const size_t smem = grd::planes_smem_bytes(S.n_planes);
    const unsigned blocks = (unsigned)((n + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
    if (grd::needs_extras(S))
        grd::k_trace_events<true><<<blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(S, B, R, rec);
    else
        grd::k_trace_events<false><<<blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(S, B, R, rec);
    GR_CUDA(cudaGetLastError());
    GR_CUDA(cudaMemcpyAsync(bounces, rec.bounces, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(termination, rec.term, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (kmax) {
        GR_CUDA(cudaMemcpyAsync(facets, rec.facets, n * kmax * 4, cudaMemcpyDeviceToHost, ctx->stream));
        GR_CUDA(cudaMemcpyAsync(t_hits, rec.ts, n * kmax * 4, cudaMemcpyDeviceToHost, ctx->stream));
        GR_CUDA(cudaMemcpyAsync(events, rec.events, n * kmax, cudaMemcpyDeviceToHost, ctx->stream));
    }
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_case_bank_arity(uint32_t bank, uint32_t *n_in, uint32_t *n_out) {
    if (bank >= GR_BANK_COUNT) return fail(GR_EINVAL, "unknown case bank %u", bank);
    if (!n_in || !n_out) return fail(GR_EINVAL, "NULL output");
    *n_in = grd::kBankArity[bank][0];
    *n_out = grd::kBankArity[bank][1];
    return GR_OK;
}

gr_status gr_case_bank(gr_ctx *ctx, uint32_t bank, const gr_scene *sc, const float *in, uint32_t n, float *out) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (bank >= GR_BANK_COUNT) return fail(GR_EINVAL, "unknown case bank %u", bank);
    if (n == 0) return GR_OK;
    if (!in || !out) return fail(GR_EINVAL, "NULL array");
    if (n > (1u << 24)) return fail(GR_EINVAL, "at most 2^24 cases per call");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    std::memset(&S, 0, sizeof(S));
    std::memset(&B, 0, sizeof(B));
    if (sc) {
        gr_status st = grh::prepare(ctx, sc, S, B);
        if (st != GR_OK) return st;
    }
    const size_t in_bytes = (size_t)n * grd::kBankArity[bank][0] * 4, out_bytes = (size_t)n * grd::kBankArity[bank][1] * 4;
    gr_status st = ctx->xyz.reserve(align256(in_bytes) + out_bytes);
    if (st != GR_OK) return st;
    float *din = (float *)ctx->xyz.ptr, *dout = (float *)((char *)ctx->xyz.ptr + align256(in_bytes));
    GR_CUDA(cudaMemcpyAsync(din, in, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    grd::k_case_bank<<<(n + 127) / 128, 128, 0, ctx->stream>>>(bank, S, B, din, n, grd::kBankArity[bank][0],
                                                                grd::kBankArity[bank][1], dout);
    GR_CUDA(cudaGetLastError());
    GR_CUDA(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_device_code_version(gr_ctx *ctx, uint32_t *binary_version, uint32_t *ptx_version) {
    if (!ctx || !binary_version || !ptx_version) return fail(GR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    cudaFuncAttributes a;
    GR_CUDA(cudaFuncGetAttributes(&a, grd::k_case_bank));
    *binary_version = (uint32_t)a.binaryVersion;
    *ptx_version = (uint32_t)a.ptxVersion;
    return GR_OK;
}

gr_status gr_intersect_rays(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const float *rays, uint32_t n,
                            float *t, int32_t *facet) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (n_planes > GR_MAX_PLANES) return fail(GR_EINVAL, "n_planes %u exceeds GR_MAX_PLANES", n_planes);
    if (n == 0) return GR_OK;
    if ((n_planes && !planes) || !rays || !t || !facet) return fail(GR_EINVAL, "NULL array");
    if (n > (1u << 24)) return fail(GR_EINVAL, "at most 2^24 rays per call");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    const size_t o_rays = align256((size_t)(n_planes ? n_planes : 1) * 16), o_t = o_rays + align256((size_t)n * 24),
                 o_f = o_t + align256((size_t)n * 4), total = o_f + (size_t)n * 4;
    gr_status st = ctx->xyz.reserve(total);
    if (st != GR_OK) return st;
    char *base = (char *)ctx->xyz.ptr;
    if (n_planes) GR_CUDA(cudaMemcpyAsync(base, planes, (size_t)n_planes * 16, cudaMemcpyHostToDevice, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(base + o_rays, rays, (size_t)n * 24, cudaMemcpyHostToDevice, ctx->stream));
    grd::k_intersect_rays<<<(n + 127) / 128, 128, grd::planes_smem_bytes(n_planes), ctx->stream>>>(
        (const float4 *)base, n_planes, (const float *)(base + o_rays), n, (float *)(base + o_t), (int32_t *)(base + o_f));
    GR_CUDA(cudaGetLastError());
    GR_CUDA(cudaMemcpyAsync(t, base + o_t, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(facet, base + o_f, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

}  // extern "C"
