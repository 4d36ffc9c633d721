// gr_host.cu -- the C ABI (include/gemray_cuda.h): context lifecycle, scene
// validation and encoding, chunked launches, film accumulation.
//
// Host-side physics that the reference evaluates once per scene or per ray from
// scene constants alone is evaluated here once per call with the same f32
// arithmetic (this file is compiled without FMA contraction):
//   * compute_illuminant_white_balance (optics/raytracer/color.rs:281-315),
//   * StudioRig::new (optics/studio_rig.rs:50-81),
//   * blackbody_spectrum's 560 nm normaliser (optics/raytracer/environment.rs:16-18),
//   * AbsorptionTensor3::uniaxial's axis frame (optics/birefringence.rs:202-209).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <unistd.h>

#include "gemray_cuda.h"
#include "gr_ctx.h"
#include "gr_host.h"
#include "gr_kernels.cuh"

using grd::SceneConst;

namespace grh {

thread_local std::string g_last_error;

gr_status fail(gr_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

}  // namespace grh

using grh::fail;

// ---------------------------------------------------------------------------------
// Host-side f32 helpers (glam scalar semantics).
// ---------------------------------------------------------------------------------
namespace grh {

struct H3 {
    float x, y, z;
};
static inline H3 h3(float x, float y, float z) { return H3{x, y, z}; }
static inline float hdot(H3 a, H3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline H3 hmul(H3 a, float s) { return h3(a.x * s, a.y * s, a.z * s); }
static inline H3 hsub(H3 a, H3 b) { return h3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline H3 hcross(H3 a, H3 b) { return h3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
static inline H3 hnormalize(H3 a) { return hmul(a, 1.0f / sqrtf(hdot(a, a))); }
static inline H3 hnormalize_or_zero(H3 a) {
    float r = 1.0f / sqrtf(hdot(a, a));
    if (std::isfinite(r) && r > 0.0f) return hmul(a, r);
    return h3(0.f, 0.f, 0.f);
}
static inline float hclamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
static inline float hpowi(float x, int n) {
    float r = 1.0f, sq = x;
    bool have = false;
    while (n) {
        if (n & 1) {
            r = have ? r * sq : sq;
            have = true;
        }
        n >>= 1;
        if (n) sq = sq * sq;
    }
    return r;
}
static inline float hgauss(float x, float mu, float slo, float shi) {
    float sigma = x < mu ? slo : shi;
    float t = (x - mu) / sigma;
    return expf(-0.5f * t * t);
}
// color/cie1931.rs:29-42 (scalar libm form used by the white-balance integral)
static inline H3 cmf_scalar(float l) {
    float x = fmaf(0.065f, -hgauss(l, 501.1f, 20.4f, 26.2f),
                   fmaf(1.056f, hgauss(l, 599.8f, 37.9f, 31.0f), 0.362f * hgauss(l, 442.0f, 16.0f, 26.7f)));
    float y = fmaf(0.286f, hgauss(l, 530.9f, 16.3f, 31.1f), 0.821f * hgauss(l, 568.8f, 46.9f, 40.5f));
    float z = fmaf(0.681f, hgauss(l, 459.0f, 26.0f, 13.8f), 1.217f * hgauss(l, 437.0f, 11.8f, 36.0f));
    return h3(fmaxf(x, 0.0f), fmaxf(y, 0.0f), fmaxf(z, 0.0f));
}
// optics/raytracer/environment.rs:12-21
static inline float blackbody(float lambda_nm, float temp_k) {
    float t_k = fmaxf(temp_k, 1000.0f);
    const float hck = 14388000.0f;
    float e = expf(fminf(hck / (lambda_nm * t_k), 80.0f));
    float e5 = expf(fminf(hck / (560.0f * t_k), 80.0f));
    float d = fmaxf(e - 1.0f, 1e-6f), d5 = fmaxf(e5 - 1.0f, 1e-6f);
    return hclamp(hpowi(560.0f / lambda_nm, 5) * (d5 / d), 0.01f, 20.0f);
}
static inline H3 bradford(const float m[3][3], H3 v) {
    return h3(fmaf(m[0][0], v.x, fmaf(m[0][1], v.y, m[0][2] * v.z)),
              fmaf(m[1][0], v.x, fmaf(m[1][1], v.y, m[1][2] * v.z)),
              fmaf(m[2][0], v.x, fmaf(m[2][1], v.y, m[2][2] * v.z)));
}
static const float XYZ_TO_LMS[3][3] = {{0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};

// optics/raytracer/color.rs:281-315
H3 white_balance(float temp_k) {
    H3 w = h3(0.f, 0.f, 0.f);
    for (int step = 0; step <= 400; ++step) {
        float lambda = 380.0f + (float)step;
        H3 c = cmf_scalar(lambda);
        float b = blackbody(lambda, temp_k);
        w = h3(w.x + c.x * b, w.y + c.y * b, w.z + c.z * b);
    }
    float ty = fmaxf(w.y, 1e-6f);
    const float wx = 0.3127f, wy = 0.3290f;
    H3 target = h3((wx / wy) * ty, ty, ((1.0f - wx - wy) / wy) * ty);
    H3 ls = bradford(XYZ_TO_LMS, w), lt = bradford(XYZ_TO_LMS, target);
    return h3(ls.x > 1e-6f ? lt.x / ls.x : 1.0f, ls.y > 1e-6f ? lt.y / ls.y : 1.0f, ls.z > 1e-6f ? lt.z / ls.z : 1.0f);
}

// optics/studio_rig.rs:50-81
void studio_rig(float yaw, float pitch, float key[3], float fill[3], float ring[16][3]) {
    float cos_lp = cosf(pitch), sin_lp = sinf(pitch), cos_ly = cosf(yaw), sin_ly = sinf(yaw);
    H3 k = hnormalize(h3(cos_lp * sin_ly, sin_lp, cos_lp * cos_ly));
    key[0] = k.x; key[1] = k.y; key[2] = k.z;
    const float PI = 3.14159265358979323846f;
    float fill_yaw = fmaf(PI, 0.78f, yaw);
    float fill_pitch = hclamp(pitch * 0.65f, 0.15f, 1.2f);
    H3 f = hnormalize(h3(cosf(fill_pitch) * sinf(fill_yaw), sinf(fill_pitch), cosf(fill_pitch) * cosf(fill_yaw)));
    fill[0] = f.x; fill[1] = f.y; fill[2] = f.z;
    const float step = PI * 2.0f / 16.0f;
    for (int i = 0; i < 16; ++i) {
        float angle = fmaf((float)i, step, yaw);
        H3 r = hnormalize(h3(cosf(angle) * 0.75f, sin_lp * 0.8f, sinf(angle) * 0.75f));
        ring[i][0] = r.x; ring[i][1] = r.y; ring[i][2] = r.z;
    }
}

// optics/birefringence.rs:126-131,202-209
void tensor_frame(const float c_axis[3], float ax0[3], float ax1[3], float ax2[3]) {
    H3 c = hnormalize_or_zero(h3(c_axis[0], c_axis[1], c_axis[2]));
    H3 a = fabsf(c.x) > 0.9f ? h3(0.f, 1.f, 0.f) : h3(1.f, 0.f, 0.f);
    H3 t = hnormalize_or_zero(hsub(a, hmul(c, hdot(c, a))));
    H3 b = hcross(c, t);
    ax0[0] = t.x; ax0[1] = t.y; ax0[2] = t.z;
    ax1[0] = b.x; ax1[1] = b.y; ax1[2] = b.z;
    ax2[0] = c.x; ax2[1] = c.y; ax2[2] = c.z;
}

}  // namespace grh

// ---------------------------------------------------------------------------------
// Scene encoding
// ---------------------------------------------------------------------------------
namespace grh {

gr_status validate_scene(const gr_scene *sc) {
    if (!sc) return fail(GR_EINVAL, "scene is NULL");
    if (!sc->material) return fail(GR_EINVAL, "scene.material is NULL");
    if (sc->n_planes > GR_MAX_PLANES) return fail(GR_EINVAL, "n_planes %u exceeds GR_MAX_PLANES", sc->n_planes);
    if (sc->n_planes > 0 && !sc->planes) return fail(GR_EINVAL, "scene.planes is NULL");
    if (sc->max_bounces > GR_MAX_BOUNCES) return fail(GR_EINVAL, "max_bounces %u exceeds GR_MAX_BOUNCES", sc->max_bounces);
    if ((uint64_t)sc->width * (uint64_t)sc->height > 0xFFFFFFFFull)
        return fail(GR_EINVAL, "width*height exceeds the u32 pixel index");
    const gr_material *m = sc->material;
    if (m->o_ray_band_count > GR_MAX_BANDS || m->e_ray_band_count > GR_MAX_BANDS || m->beta_ray_band_count > GR_MAX_BANDS)
        return fail(GR_EINVAL, "absorption band count exceeds GR_MAX_BANDS");
    if (m->dispersion.model_type > GR_DISP_CAUCHY) return fail(GR_EINVAL, "unknown dispersion model %u", m->dispersion.model_type);
    if (sc->env.mode > GR_ENV_LATLONG) return fail(GR_EINVAL, "unknown environment mode %u", sc->env.mode);
    if (sc->env.mode == GR_ENV_LATLONG) {
        if (!sc->env.latlong_rgb || sc->env.latlong_w == 0 || sc->env.latlong_h == 0)
            return fail(GR_EINVAL, "lat-long environment needs a non-empty map");
        if ((uint64_t)sc->env.latlong_w * sc->env.latlong_h > (1ull << 28)) return fail(GR_EINVAL, "lat-long map too large");
    }
    if (sc->material_ext) {
        const gr_material_ext *e = sc->material_ext;
        if (e->n_absorption > 0 && (!e->alpha_o_table || !e->alpha_e_table || !(e->absorption_nm_step > 0.0f)))
            return fail(GR_EINVAL, "material_ext absorption table is incomplete");
        if (e->n_absorption > (1u << 20)) return fail(GR_EINVAL, "material_ext absorption table too long");
    }
    return GR_OK;
}


void encode_scene(const gr_scene *sc, SceneConst &S) {
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
    S.max_bounces = sc->max_bounces;
    S.n_planes = sc->n_planes;
    const gr_material *m = sc->material;
    S.disp_model = m->dispersion.model_type;
    for (int i = 0; i < 3; ++i) {
        S.disp_a[i] = m->dispersion.param_a[i];
        S.disp_b[i] = m->dispersion.param_b[i];
        S.c_axis[i] = m->dispersion.c_axis_and_birefringence[i];
    }
    S.bire = m->dispersion.c_axis_and_birefringence[3];
    // transport.rs:620-621
    S.anisotropic = (m->crystal_system != GR_CRYSTAL_CUBIC && fabsf(S.bire) > 1e-4f) ? 1u : 0u;
    S.n_o_bands = m->o_ray_band_count;
    S.n_e_bands = m->e_ray_band_count;
    for (uint32_t i = 0; i < GR_MAX_BANDS; ++i) {
        S.o_bands[i][0] = m->o_ray_bands[i].center_nm;
        S.o_bands[i][1] = m->o_ray_bands[i].width_nm;
        S.o_bands[i][2] = m->o_ray_bands[i].peak;
        S.e_bands[i][0] = m->e_ray_bands[i].center_nm;
        S.e_bands[i][1] = m->e_ray_bands[i].width_nm;
        S.e_bands[i][2] = m->e_ray_bands[i].peak;
    }
    S.path_scale = m->absorption_path_scale;
    S.sigma_s = m->scattering_sigma_s;
    S.hg_g = m->scattering_g;
    S.any_frosted = 0;
    if (sc->finishes)
        for (uint32_t i = 0; i < sc->n_planes; ++i)
            if (sc->finishes[i] != 0) {
                S.frosted[i >> 5] |= 1u << (i & 31);
                S.any_frosted = 1;
            }
    S.edge_radius = m->edge_rounding_radius;
    tensor_frame(S.c_axis, S.ax0, S.ax1, S.ax2);
    const gr_material_ext *ext = sc->material_ext;
    if (ext) {
        S.ext_n = ext->n_absorption;
        S.ext_first = ext->absorption_nm_first;
        S.ext_step = ext->absorption_nm_step;
        S.has_cauchy_e = ext->has_cauchy_e ? 1u : 0u;
        for (int i = 0; i < 3; ++i) S.cauchy_e[i] = ext->cauchy_e[i];
    }
    // biaxial indicatrix and the beta-ray band set (read by biaxial materials only,
    // build_ray_wavelength_cache, refraction.rs:140-166)
    S.biaxial = m->dispersion.has_biaxial_delta ? 1u : 0u;
    S.d_beta_alpha = m->dispersion.biaxial_delta_beta_alpha;
    S.has_beta = (S.biaxial && m->has_beta_ray) ? 1u : 0u;
    S.n_b_bands = S.has_beta ? m->beta_ray_band_count : 0u;
    for (uint32_t i = 0; i < GR_MAX_BANDS; ++i) {
        S.b_bands[i][0] = m->beta_ray_bands[i].center_nm;
        S.b_bands[i][1] = m->beta_ray_bands[i].width_nm;
        S.b_bands[i][2] = m->beta_ray_bands[i].peak;
    }
    S.absorbing = (S.ext_n > 0 || S.n_o_bands > 0 || S.n_e_bands > 0 || S.n_b_bands > 0) ? 1u : 0u;
    S.env_mode = sc->env.mode;
    for (int i = 0; i < 3; ++i) S.uni_rgb[i] = sc->env.uniform_rgb[i];
    S.temp_k = sc->env.temp_k;
    S.spot_mult = sc->env.spot_mult;
    S.exposure = sc->env.exposure;
    S.wb[0] = S.wb[1] = S.wb[2] = 1.0f;  // environment.rs:238-243: maps -> Vec3::ONE
    if (sc->env.mode == GR_ENV_STUDIO) {
        H3 w = white_balance(sc->env.temp_k);
        S.wb[0] = w.x; S.wb[1] = w.y; S.wb[2] = w.z;
        studio_rig(sc->env.light_yaw, sc->env.light_pitch, S.key, S.fill, S.ring);
        float t_k = fmaxf(sc->env.temp_k, 1000.0f);
        float e5 = expf(fminf(14388000.0f / (560.0f * t_k), 80.0f));
        S.denom560 = fmaxf(e5 - 1.0f, 1e-6f);
    }
    S.map_w = sc->env.latlong_w;
    S.map_h = sc->env.latlong_h;
    S.flags = sc->flags;
}

}  // namespace grh

// ---------------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------------
// A scene kept on the device between calls (serving / benchmark): encoded
// constants plus its own copies of the planes, map and extension tables.

namespace grd {
__global__ void k_rng_records(const uint32_t *__restrict__ pixels, const uint32_t *__restrict__ samples, uint32_t n,
                              gr_rng_record *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Draws d = sample_draws(pixels[i], samples[i]);
    gr_rng_record r;
    r.seed = d.seed;
    r.jitter_x = d.jx;
    r.jitter_y = d.jy;
    r.hero_rand = d.hero;
    for (uint32_t b = 0; b < 4; ++b) {
        r.draws[b][0] = rng_draw(d.seed, b, FRESNEL_BRANCH_STREAM);
        r.draws[b][1] = rng_draw(d.seed, b, RUSSIAN_ROULETTE_STREAM);
        r.draws[b][2] = rng_draw(d.seed, b, BIREFRINGENT_SPLIT_STREAM);
        r.draws[b][3] = rng_draw(d.seed, b, MODE_COUPLING_STREAM);
    }
    out[i] = r;
}
}  // namespace grd

namespace grh {

gr_status DeviceBuffer::reserve(size_t bytes) {
    if (bytes <= cap) return GR_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&ptr, bytes);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return fail(GR_ENOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    cap = bytes;
    return GR_OK;
}
void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

// Upload the scene's device-side arrays into the context's buffers.
gr_status upload_scene(gr_ctx *ctx, const gr_scene *sc, const SceneConst &S, grd::SceneBuffers &B) {
    std::memset(&B, 0, sizeof(B));
    size_t pbytes = (size_t)(sc->n_planes ? sc->n_planes : 1) * sizeof(float4);
    gr_status st = ctx->planes.reserve(pbytes);
    if (st != GR_OK) return st;
    if (sc->n_planes) {
        static_assert(sizeof(gr_plane) == sizeof(float4), "plane layout");
        GR_CUDA(cudaMemcpyAsync(ctx->planes.ptr, sc->planes, sc->n_planes * sizeof(gr_plane), cudaMemcpyHostToDevice,
                                ctx->stream));
    }
    B.planes = (const float4 *)ctx->planes.ptr;
    if (S.env_mode == GR_ENV_LATLONG) {
        size_t mbytes = (size_t)S.map_w * S.map_h * 3 * sizeof(float);
        st = ctx->map.reserve(mbytes);
        if (st != GR_OK) return st;
        GR_CUDA(cudaMemcpyAsync(ctx->map.ptr, sc->env.latlong_rgb, mbytes, cudaMemcpyHostToDevice, ctx->stream));
        B.map = (const float *)ctx->map.ptr;
    }
    if (S.ext_n > 0) {
        size_t ebytes = (size_t)S.ext_n * 2 * sizeof(float);
        st = ctx->ext.reserve(ebytes);
        if (st != GR_OK) return st;
        float *d = (float *)ctx->ext.ptr;
        GR_CUDA(cudaMemcpyAsync(d, sc->material_ext->alpha_o_table, S.ext_n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        GR_CUDA(cudaMemcpyAsync(d + S.ext_n, sc->material_ext->alpha_e_table, S.ext_n * sizeof(float), cudaMemcpyHostToDevice,
                                ctx->stream));
        B.ext_alpha_o = d;
        B.ext_alpha_e = d + S.ext_n;
    }
    return GR_OK;
}


int resolve_kernel(int mode, uint64_t n_tuples) {
    if (mode != GR_KERNEL_AUTO) return mode;
    return n_tuples < GR_AUTO_STAGED_MIN_TUPLES ? GR_KERNEL_PLAIN : GR_KERNEL_STAGED;
}

int scene_class(const SceneConst &S) {
    if (grd::needs_extras(S)) return -1;
    const bool iso = !S.anisotropic && !S.biaxial, clear = !S.absorbing;
    return ((iso && clear) ? (grd::K_ISO | grd::K_CLEAR) : 0) | grd::k_env(S.env_mode);
}

// The kernel a single-scene launch of this scene runs: GR_KERNEL_SORTED only for clear
// isotropic stones (its slots hold that class's record; other scenes take AUTO's choice).
static int scene_kernel(int mode, const SceneConst &S, uint64_t n_tuples) {
    if (mode == GR_KERNEL_SORTED) {
        const int K = scene_class(S);
        const bool ok = K >= 0 && (K & grd::K_CLEAR) && S.max_bounces > 0 && !(S.flags & GR_FLAG_FP64_RESOLVE);
        if (!ok) mode = GR_KERNEL_AUTO;
    }
    return resolve_kernel(mode, n_tuples);
}

int trace_kernel_launches(int mode, const SceneConst &S, uint64_t n_tuples) {
    const int k = scene_kernel(mode, S, n_tuples);
    const bool staged = k == GR_KERNEL_STAGED && S.max_bounces > 0 && !(S.flags & GR_FLAG_FP64_RESOLVE);
    return staged ? 3 : 1;  // stages 1, 2 and 3
}

uint64_t staged_park_slots(uint64_t n_tuples) {
    uint64_t cap1 = (n_tuples + 7) / 8;
    const uint64_t max_cap = (4ull << 30) / sizeof(grd::Path);
    if (cap1 > max_cap) cap1 = max_cap;
    if (cap1 < 1024) cap1 = 1024;
    return cap1;
}

size_t staged_park_bytes(uint64_t n_tuples) {
    const uint64_t cap1 = staged_park_slots(n_tuples);
    return (size_t)(cap1 + (cap1 + 3) / 4) * sizeof(grd::Path) + 256;
}

// Trace tuples [0, R.n_tuples) of one chunk into xyz (device).

gr_status launch_trace(gr_ctx *ctx, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                       float *xyz, cudaStream_t stream, int mode, grh::DeviceBuffer *park_buf, StageCaps caps) {
    if (caps.first == 0) caps = StageCaps{GR_STAGE_CAP, GR_STAGE_CAP2};
    if (R.n_tuples == 0) return GR_OK;
    mode = scene_kernel(mode, S, R.n_tuples);
    size_t smem = grd::planes_smem_bytes(S.n_planes);
    const bool extras = grd::needs_extras(S);
    const uint64_t plain_blocks = (R.n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS;
    if (S.flags & GR_FLAG_FP64_RESOLVE) {  // the re-solve variant exists for the plain kernel only
        if (extras)
            grd::k_trace_plain<grd::NoCounters, true, true><<<(unsigned)plain_blocks, grd::TRACE_THREADS, smem, stream>>>(
                S, B, R, xyz, nullptr);
        else
            grd::k_trace_plain<grd::NoCounters, true><<<(unsigned)plain_blocks, grd::TRACE_THREADS, smem, stream>>>(
                S, B, R, xyz, nullptr);
        GR_CUDA(cudaGetLastError());
        return GR_OK;
    }
    const int K = scene_class(S);
    const bool clear = K >= 0 && (K & grd::K_CLEAR);
    if (mode == GR_KERNEL_PLAIN || S.max_bounces == 0) {
        if (extras) {
            grd::k_trace_plain<grd::NoCounters, false, true><<<(unsigned)plain_blocks, grd::TRACE_THREADS, smem, stream>>>(
                S, B, R, xyz, nullptr);
            GR_CUDA(cudaGetLastError());
            return GR_OK;
        }
        return clear ? launch_single_clear(K, S, B, R, xyz, stream, nullptr)
                     : launch_single_general(K, S, B, R, xyz, stream, nullptr);
    }
    if (mode == GR_KERNEL_SORTED) {
        // the tuple counter of the sorted blocks sits in the park buffer's header, so a
        // frame stream (own park buffer and stream) never shares it with the context
        grh::DeviceBuffer &pk = park_buf ? *park_buf : ctx->park;
        gr_status st = pk.reserve(256);
        if (st != GR_OK) return st;
        return launch_single_clear(K, S, B, R, xyz, stream, nullptr, (unsigned int *)pk.ptr + 2, ctx->sm_count);
    }
    if (mode == GR_KERNEL_STAGED) {
        // park buffers: stage 1 parks up to 1/8 of the launch's paths (at most 4 GiB),
        // stage 2 up to 1/4 of that; overflowing paths finish where they are
        const uint64_t cap1 = staged_park_slots(R.n_tuples);
        const uint64_t cap2 = caps.second == 0xFFFFFFFFu ? 0 : (cap1 + 3) / 4;
        grh::DeviceBuffer &pk = park_buf ? *park_buf : ctx->park;
        gr_status st = pk.reserve((size_t)(cap1 + cap2) * sizeof(grd::Path) + 256);
        if (st != GR_OK) return st;
        unsigned int *counts = (unsigned int *)pk.ptr;
        grd::Path *park1 = (grd::Path *)((char *)pk.ptr + 256);
        grd::Path *park2 = park1 + cap1;
        GR_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned int), stream));
        if (!extras) {
            const StagedLaunch sl{park1, park2, counts, cap1, cap2, caps.first, caps.second, caps.blocks};
            return clear ? launch_single_clear(K, S, B, R, xyz, stream, &sl)
                         : launch_single_general(K, S, B, R, xyz, stream, &sl);
        }
        const grd::ParkOut out1{park1, (uint32_t)cap1, counts};
        const grd::ParkOut out2{park2, (uint32_t)cap2, counts + 1};
        const grd::ParkOut none{nullptr, 0, nullptr};
        const unsigned b2 = (unsigned)((cap1 + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
        const unsigned b3 = (unsigned)((cap2 + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS);
        {
            grd::k_trace_stage1<true><<<(unsigned)plain_blocks, grd::TRACE_THREADS, smem, stream>>>(S, B, R, xyz, out1,
                                                                                                  caps.first);
            grd::k_trace_stage2<true><<<b2, grd::TRACE_THREADS, smem, stream>>>(S, B, park1, (uint32_t)cap1, counts,
                                                                                caps.second, out2, xyz);
            if (cap2)
                grd::k_trace_stage2<true><<<b3, grd::TRACE_THREADS, smem, stream>>>(S, B, park2, (uint32_t)cap2,
                                                                                    counts + 1, 0xFFFFFFFFu, none, xyz);
        }
        GR_CUDA(cudaGetLastError());
        return GR_OK;
    }
    return fail(GR_EINVAL, "unknown kernel mode %d", mode);
}

gr_status launch_fold(const float *xyz, uint32_t n_pixels, uint32_t spp, uint32_t first_pixel, float *film,
                      uint32_t kahan, cudaStream_t stream) {
    if (n_pixels == 0) return GR_OK;
    const uint64_t blocks = ((uint64_t)n_pixels + grd::FOLD_THREADS - 1) / grd::FOLD_THREADS;
    grd::k_film_fold_tiled<<<(unsigned)blocks, grd::FOLD_THREADS, 0, stream>>>(xyz, n_pixels, spp, first_pixel, film,
                                                                              kahan);
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

// Next free (start, stop) event pair for a timed launch, or NULL when timing is off.
cudaEvent_t *timing_slot(gr_ctx *ctx, std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &pool, size_t &used) {
    if (!ctx->timing) return nullptr;
    if (used == pool.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return nullptr;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return nullptr;
        }
        pool.emplace_back(a, b);
    }
    return &pool[used++].first;
}

// The shared body of gr_accumulate / gr_accumulate_device: trace every pixel's
// [sample_offset, sample_offset + spp) samples chunk by chunk and add each pixel's
// folded sum into film_dev.
gr_status render_into(gr_ctx *ctx, const gr_scene *sc, const SceneConst &S, const grd::SceneBuffers &B,
                      uint32_t sample_offset, uint32_t spp, float *film_dev, cudaStream_t stream,
                      StageCaps caps = StageCaps{}) {
    const uint64_t n_pixels = (uint64_t)sc->width * sc->height;
    uint64_t budget_tuples = ctx->chunk_budget / (3 * sizeof(float));
    if (budget_tuples > 0xFFFFFFFFull) budget_tuples = 0xFFFFFFFFull;  // tuple ids are u32 within a launch
    uint64_t chunk_pixels = budget_tuples / spp;
    if (chunk_pixels < 1) chunk_pixels = 1;
    if (chunk_pixels > n_pixels) chunk_pixels = n_pixels;
    gr_status st = ctx->xyz.reserve((size_t)chunk_pixels * spp * 3 * sizeof(float));
    if (st != GR_OK) return st;
    for (uint64_t first = 0; first < n_pixels; first += chunk_pixels) {
        uint64_t np = n_pixels - first < chunk_pixels ? n_pixels - first : chunk_pixels;
        grd::LaunchRange R;
        R.first_pixel = (uint32_t)first;
        R.n_pixels = (uint32_t)np;
        R.sample_offset = sample_offset;
        R.spp = spp;
        R.n_tuples = np * spp;
        cudaEvent_t *tev = timing_slot(ctx, ctx->trace_ev, ctx->trace_used);
        if (tev) cudaEventRecord(tev[0], stream);
        st = launch_trace(ctx, S, B, R, (float *)ctx->xyz.ptr, stream, ctx->kernel_mode, nullptr, caps);
        if (st != GR_OK) return st;
        if (tev) cudaEventRecord(tev[1], stream);
        ctx->trace_launches += trace_kernel_launches(ctx->kernel_mode, S, R.n_tuples);
        cudaEvent_t *fev = timing_slot(ctx, ctx->fold_ev, ctx->fold_used);
        if (fev) cudaEventRecord(fev[0], stream);
        st = launch_fold((const float *)ctx->xyz.ptr, (uint32_t)np, spp, (uint32_t)first, film_dev,
                         (S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u, stream);
        if (st != GR_OK) return st;
        if (fev) cudaEventRecord(fev[1], stream);
        ctx->fold_launches++;
    }
    return GR_OK;
}

gr_status prepare(gr_ctx *ctx, const gr_scene *sc, SceneConst &S, grd::SceneBuffers &B) {
    gr_status st = validate_scene(sc);
    if (st != GR_OK) return st;
    encode_scene(sc, S);
    return upload_scene(ctx, sc, S, B);
}

// The candidate a trial times: trials [0, kScheduleBlockCount) the first cap pair at
// each blocks-per-SM target, then the other pairs at the fastest of those targets (-1
// while that target is not known yet).
int trial_candidate(const StageCapTune &T, int n) {
    if (n < kScheduleBlockCount) return n;
    int fast = 0;
    for (int b = 0; b < kScheduleBlockCount; ++b) {
        if (!T.trial[b].done) return -1;
        if (T.ms_per_mtuple[b] < T.ms_per_mtuple[fast]) fast = b;
    }
    return (n - kScheduleBlockCount + 1) * kScheduleBlockCount + fast;
}

void tune_harvest(gr_ctx *ctx, StageCapTune &T) {
    if (T.best >= 0) return;
    bool all = T.n_trials == StageCapTune::kTrials;
    for (int i = 0; i < T.n_trials; ++i) {
        auto &tr = T.trial[i];
        if (tr.ended && !tr.done && cudaEventQuery(tr.stop) == cudaSuccess) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, tr.start, tr.stop) == cudaSuccess && tr.tuples)
                T.ms_per_mtuple[tr.candidate] = ms / (float)((double)tr.tuples * 1e-6);
            tr.done = true;
        }
        all = all && tr.done;
    }
    cudaGetLastError();  // a query of an unfinished event is not an error to keep
    if (!all) return;
    int best = 0;
    for (int c = 1; c < kScheduleCandidates; ++c)
        if (T.ms_per_mtuple[c] < T.ms_per_mtuple[best]) best = c;
    T.best = best;
    if (T.key) ctx->tuned[T.key] = TunedSchedule{best, T.ms_per_mtuple[best]};
}

void tune_init(gr_ctx *ctx, StageCapTune &T, uint64_t key) {
    tune_release(T);
    T = StageCapTune{};
    T.key = key;
    auto it = ctx->tuned.find(key);
    if (key && it != ctx->tuned.end()) T.best = it->second.candidate;
}

uint32_t scene_stage_cap(const ResidentScene &rs) {
    return rs.tune.best >= 0 ? schedule_candidate(rs.tune.best).first : (uint32_t)GR_STAGE_CAP;
}

StageCaps scene_stage_caps(const ResidentScene &rs) {
    return rs.tune.best >= 0 ? schedule_candidate(rs.tune.best) : StageCaps{};
}

StageCaps tune_begin(gr_ctx *ctx, StageCapTune &T, const SceneConst &S, uint64_t n_pixels, uint32_t spp,
                     cudaStream_t s, int &trial) {
    trial = -1;
    const uint64_t budget_tuples = ctx->chunk_budget / (3 * sizeof(float));
    const uint64_t first_chunk = std::min<uint64_t>(n_pixels, std::max<uint64_t>(1, budget_tuples / spp)) * spp;
    if (trace_kernel_launches(ctx->kernel_mode, S, first_chunk) != 3) return StageCaps{};  // not staged
    tune_harvest(ctx, T);
    if (T.best >= 0) return schedule_candidate(T.best);
    if (T.staged_calls++ == 0 || T.n_trials == StageCapTune::kTrials) return StageCaps{};
    const int c = trial_candidate(T, T.n_trials);
    if (c < 0) return StageCaps{};  // the second round waits for the first round's times
    auto &tr = T.trial[T.n_trials];
    if ((!tr.start && cudaEventCreate(&tr.start) != cudaSuccess) || (!tr.stop && cudaEventCreate(&tr.stop) != cudaSuccess)) {
        cudaGetLastError();
        return StageCaps{};  // untimed: stay on the built-in schedule
    }
    tr.candidate = c;
    tr.tuples = n_pixels * spp;
    tr.ended = tr.done = false;
    trial = T.n_trials++;
    cudaEventRecord(tr.start, s);
    return schedule_candidate(c);
}

void tune_end(StageCapTune &T, int trial, cudaStream_t s) {
    if (trial < 0) return;
    cudaEventRecord(T.trial[trial].stop, s);
    T.trial[trial].ended = true;
}

uint64_t stone_key(const gr_scene *sc) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a, 64 bit
    auto mix = [&h](const void *p, size_t n) {
        const unsigned char *b = (const unsigned char *)p;
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    };
    mix(&sc->n_planes, sizeof(sc->n_planes));
    mix(&sc->max_bounces, sizeof(sc->max_bounces));
    mix(&sc->flags, sizeof(sc->flags));
    mix(&sc->env.mode, sizeof(sc->env.mode));  // the environment kind selects the kernels
    if (sc->planes) mix(sc->planes, (size_t)sc->n_planes * sizeof(gr_plane));
    if (sc->finishes) mix(sc->finishes, (size_t)sc->n_planes * sizeof(uint32_t));
    if (sc->material) mix(sc->material, sizeof(gr_material));
    if (const gr_material_ext *e = sc->material_ext) {
        // its values and tables, not its table pointers (which differ between processes)
        mix(&e->n_absorption, sizeof(e->n_absorption));
        mix(&e->absorption_nm_first, sizeof(e->absorption_nm_first));
        mix(&e->absorption_nm_step, sizeof(e->absorption_nm_step));
        if (e->n_absorption && e->alpha_o_table) mix(e->alpha_o_table, (size_t)e->n_absorption * sizeof(float));
        if (e->n_absorption && e->alpha_e_table) mix(e->alpha_e_table, (size_t)e->n_absorption * sizeof(float));
        mix(&e->has_cauchy_e, sizeof(e->has_cauchy_e));
        mix(e->cauchy_e, sizeof(e->cauchy_e));
    }
    return h;
}

void tune_release(StageCapTune &T) {
    for (auto &tr : T.trial) {
        if (tr.start) cudaEventDestroy(tr.start);
        if (tr.stop) cudaEventDestroy(tr.stop);
        tr.start = tr.stop = nullptr;
    }
}

StageCapTune &accum_tune(gr_ctx *ctx, const gr_scene *sc) {
    const uint64_t key = stone_key(sc);
    auto it = ctx->accum_tune.find(key);
    if (it != ctx->accum_tune.end()) return it->second;
    if (ctx->accum_tune.size() >= gr_ctx::kMaxAccumTunes) {
        for (auto &kv : ctx->accum_tune) tune_release(kv.second);
        ctx->accum_tune.clear();
    }
    StageCapTune &T = ctx->accum_tune[key];
    tune_init(ctx, T, key);
    return T;
}
}  // namespace grh

// ---------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------
// Device pointers of a resident scene in the layout the kernels take.
grd::SceneBuffers resident_buffers(ResidentScene *rs) {
    grd::SceneBuffers B;
    std::memset(&B, 0, sizeof(B));
    B.planes = (const float4 *)rs->planes.ptr;
    B.map = (const float *)rs->map.ptr;
    if (rs->S.ext_n) {
        B.ext_alpha_o = (const float *)rs->ext.ptr;
        B.ext_alpha_e = (const float *)rs->ext.ptr + rs->S.ext_n;
    }
    return B;
}

extern "C" {

uint32_t gr_abi_version(void) { return GR_ABI_VERSION; }

const char *gr_last_error_string(void) { return grh::g_last_error.c_str(); }

namespace {
gr_status tuning_save_locked(gr_ctx *ctx, const char *path);
gr_status tuning_load_locked(gr_ctx *ctx, const char *path, uint32_t *n_loaded);
}  // namespace

gr_status gr_create(gr_ctx **out, const gr_create_opts *opts) {
    if (!out) return fail(GR_EINVAL, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(GR_NO_DEVICE, "no CUDA device: %s", e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
    }
    int dev = 0;
    if (opts && opts->device >= 0) dev = opts->device;
    if (dev >= count) return fail(GR_NO_DEVICE, "device %d out of range (%d devices)", dev, count);
    cudaDeviceProp prop;
    GR_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) return fail(GR_NO_DEVICE, "device %d (%s, sm_%d%d) is not sm_100", dev, prop.name, prop.major, prop.minor);
    GR_CUDA(cudaSetDevice(dev));
    gr_ctx *ctx = new gr_ctx();
    ctx->device = dev;
    if (opts && opts->chunk_budget_bytes) ctx->chunk_budget = opts->chunk_budget_bytes;
    if (opts && opts->serve_budget_bytes) ctx->serve_budget = opts->serve_budget_bytes;
    // The context stream sits between the stream priorities: the request loop's bulk
    // lane (gr_serve.cu) takes the highest, so its blocks are scheduled before the
    // ticks queued here.
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    e = cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, (prio_lo + prio_hi) / 2);
    if (e != cudaSuccess) {
        delete ctx;
        return fail(GR_ECUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
    }
    ctx->sm_count = prop.multiProcessorCount;
    char buf[512];
    snprintf(buf, sizeof(buf), "%.256s (CUDA, sm_%d%d, %d SMs)", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    ctx->label = buf;
    // GR_TUNING_CACHE: a per-device schedule table read now and written back (merged)
    // by gr_destroy; a table for another device or schedule set is left to be replaced
    const char *cache = getenv("GR_TUNING_CACHE");
    if (cache && *cache) {
        ctx->tuning_cache = cache;
        tuning_load_locked(ctx, cache, nullptr);
        grh::g_last_error.clear();
    }
    *out = ctx;
    return GR_OK;
}

gr_status gr_destroy(gr_ctx *ctx) {
    if (!ctx) return GR_OK;
    grh::serve_shutdown(ctx);  // joins the request loop, which takes ctx->mu itself
    grh::streams_shutdown(ctx);
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ctx->xyz.release();
        ctx->film.release();
        ctx->planes.release();
        ctx->map.release();
        ctx->ext.release();
        ctx->counter.release();
        ctx->rgba.release();
        ctx->metrics.release();
        ctx->park.release();
        for (grh::DeviceBuffer *b : {&ctx->dn_a, &ctx->dn_b, &ctx->dn_n, &ctx->dn_g, &ctx->dn_in, &ctx->dn_out,
                                     &ctx->dn_planes})
            b->release();
        if (ctx->dn_ev) cudaEventDestroy(ctx->dn_ev);
        for (int k = 0; k < gr_ctx::kStageSlots; ++k) {
            if (ctx->stage_host[k]) cudaFreeHost(ctx->stage_host[k]);
            if (ctx->stage_ev[k]) cudaEventDestroy(ctx->stage_ev[k]);
        }
        for (BatchGraph &g : ctx->batch_graphs) cudaGraphExecDestroy(g.exec);
        ctx->batch_graphs.clear();
        ctx->batch_tables.release();
        ctx->batch_park.release();
        if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
        ctx->host_stage = nullptr;
        for (auto &p : ctx->trace_ev) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
        for (auto &p : ctx->fold_ev) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
        if (!ctx->tuning_cache.empty()) {
            for (auto &kv : ctx->scenes) grh::tune_harvest(ctx, kv.second->tune);
            for (auto &kv : ctx->accum_tune) grh::tune_harvest(ctx, kv.second);
            if (!ctx->tuned.empty()) tuning_save_locked(ctx, ctx->tuning_cache.c_str());
        }
        for (auto &kv : ctx->accum_tune) grh::tune_release(kv.second);
        ctx->accum_tune.clear();
        for (auto &kv : ctx->scenes) {
            grh::tune_release(kv.second->tune);
            kv.second->planes.release();
            kv.second->map.release();
            kv.second->ext.release();
            delete kv.second;
        }
        ctx->scenes.clear();
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return GR_OK;
}

const char *gr_device_label(gr_ctx *ctx) { return ctx ? ctx->label.c_str() : ""; }

gr_status gr_accumulate(gr_ctx *ctx, const gr_scene *sc, uint32_t sample_offset, uint32_t spp, float *accum) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!sc) return fail(GR_EINVAL, "scene is NULL");
    const uint64_t n_pixels = (uint64_t)sc->width * sc->height;
    if (spp == 0 || n_pixels == 0) return GR_OK;  // frame.rs:678-680
    if (!accum) return fail(GR_EINVAL, "accum is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    const size_t fbytes = (size_t)n_pixels * 3 * sizeof(float);
    st = ctx->film.reserve(fbytes);
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemcpyAsync(ctx->film.ptr, accum, fbytes, cudaMemcpyHostToDevice, ctx->stream));
    StageCapTune &T = grh::accum_tune(ctx, sc);
    int trial = -1;
    const StageCaps caps = grh::tune_begin(ctx, T, S, n_pixels, spp, ctx->stream, trial);
    st = grh::render_into(ctx, sc, S, B, sample_offset, spp, (float *)ctx->film.ptr, ctx->stream, caps);
    grh::tune_end(T, trial, ctx->stream);
    if (st != GR_OK) {
        cudaStreamSynchronize(ctx->stream);
        return st;
    }
    // Copy into the context's pinned staging buffer first (a failure leaves accum
    // untouched; a pinned target takes the copy at full link speed and is not
    // allocated and zeroed per call), then into the caller's buffer.
    if (ctx->host_stage_cap < fbytes) {
        if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
        ctx->host_stage = nullptr;
        ctx->host_stage_cap = 0;
        GR_CUDA(cudaHostAlloc(&ctx->host_stage, fbytes, cudaHostAllocDefault));
        ctx->host_stage_cap = fbytes;
    }
    GR_CUDA(cudaMemcpyAsync(ctx->host_stage, ctx->film.ptr, fbytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(accum, ctx->host_stage, fbytes);
    return GR_OK;
}

gr_status gr_accumulate_device(gr_ctx *ctx, const gr_scene *sc, uint32_t sample_offset, uint32_t spp,
                               float *accum_dev, void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!sc) return fail(GR_EINVAL, "scene is NULL");
    const uint64_t n_pixels = (uint64_t)sc->width * sc->height;
    if (spp == 0 || n_pixels == 0) return GR_OK;
    if (!accum_dev) return fail(GR_EINVAL, "accum_xyz_device is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    if (s != ctx->stream) {
        // Order the caller's stream after the scene upload on the context stream.
        cudaEvent_t ev;
        GR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, ctx->stream);
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    StageCapTune &T = grh::accum_tune(ctx, sc);
    int trial = -1;
    const StageCaps caps = grh::tune_begin(ctx, T, S, n_pixels, spp, s, trial);
    st = grh::render_into(ctx, sc, S, B, sample_offset, spp, accum_dev, s, caps);
    grh::tune_end(T, trial, s);
    if (st != GR_OK) return st;
    if (s != ctx->stream) {
        // Later uploads on the context stream must wait for this work.
        cudaEvent_t ev;
        GR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, s);
        cudaStreamWaitEvent(ctx->stream, ev, 0);
        cudaEventDestroy(ev);
    }
    return GR_OK;
}

gr_status gr_trace_samples(gr_ctx *ctx, const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels,
                           uint32_t sample_offset, uint32_t spp, float *xyz_out) {
    if (!ctx || !sc) return fail(GR_EINVAL, "ctx or scene is NULL");
    if (n_pixels == 0 || spp == 0) return GR_OK;
    if (!xyz_out) return fail(GR_EINVAL, "xyz_out is NULL");
    if ((uint64_t)first_pixel + n_pixels > (uint64_t)sc->width * sc->height)
        return fail(GR_EINVAL, "pixel range exceeds the frame");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    uint64_t n_tuples = (uint64_t)n_pixels * spp;
    size_t bytes = (size_t)n_tuples * 3 * sizeof(float);
    st = ctx->xyz.reserve(bytes);
    if (st != GR_OK) return st;
    grd::LaunchRange R;
    R.first_pixel = first_pixel;
    R.n_pixels = n_pixels;
    R.sample_offset = sample_offset;
    R.spp = spp;
    R.n_tuples = n_tuples;
    st = grh::launch_trace(ctx, S, B, R, (float *)ctx->xyz.ptr, ctx->stream, ctx->kernel_mode);
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemcpyAsync(xyz_out, ctx->xyz.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_tonemap(gr_ctx *ctx, const float *xyz, float scale, uint32_t n_px, uint8_t *rgba) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (n_px == 0) return GR_OK;
    if (!xyz || !rgba) return fail(GR_EINVAL, "xyz or rgba is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    size_t in_bytes = (size_t)n_px * 3 * sizeof(float), out_bytes = (size_t)n_px * 4;
    gr_status st = ctx->film.reserve(in_bytes);
    if (st != GR_OK) return st;
    st = ctx->rgba.reserve(out_bytes);
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemcpyAsync(ctx->film.ptr, xyz, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    st = grh::tonemap_device((const float *)ctx->film.ptr, scale, n_px, ctx->rgba.ptr, ctx->stream);
    if (st != GR_OK) return fail(st, "tone-map launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    GR_CUDA(cudaMemcpyAsync(rgba, ctx->rgba.ptr, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_rng_records(gr_ctx *ctx, const uint32_t *pixels, const uint32_t *samples, uint32_t n,
                         gr_rng_record *out) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (n == 0) return GR_OK;
    if (!pixels || !samples || !out) return fail(GR_EINVAL, "NULL array");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    size_t in_bytes = (size_t)n * sizeof(uint32_t), out_bytes = (size_t)n * sizeof(gr_rng_record);
    gr_status st = ctx->xyz.reserve(2 * in_bytes + out_bytes + 16);
    if (st != GR_OK) return st;
    char *base = (char *)ctx->xyz.ptr;
    uint32_t *dp = (uint32_t *)base, *ds = (uint32_t *)(base + in_bytes);
    gr_rng_record *dout = (gr_rng_record *)(base + ((2 * in_bytes + 15) & ~(size_t)15));
    GR_CUDA(cudaMemcpyAsync(dp, pixels, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    GR_CUDA(cudaMemcpyAsync(ds, samples, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    grd::k_rng_records<<<(n + 127) / 128, 128, 0, ctx->stream>>>(dp, ds, n, dout);
    GR_CUDA(cudaGetLastError());
    GR_CUDA(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_scene_upload(gr_ctx *ctx, const gr_scene *sc, uint64_t *out_id) {
    if (!ctx || !out_id) return fail(GR_EINVAL, "ctx or out_id is NULL");
    gr_status st = grh::validate_scene(sc);
    if (st != GR_OK) return st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    ResidentScene *rs = new ResidentScene();
    grh::encode_scene(sc, rs->S);
    size_t pbytes = (size_t)(sc->n_planes ? sc->n_planes : 1) * sizeof(float4);
    size_t mbytes = rs->S.env_mode == GR_ENV_LATLONG ? (size_t)rs->S.map_w * rs->S.map_h * 3 * sizeof(float) : 0;
    size_t ebytes = (size_t)rs->S.ext_n * 2 * sizeof(float);
    uint64_t total = pbytes + mbytes + ebytes;
    if (ctx->resident_bytes + total > ctx->serve_budget) {
        delete rs;
        return fail(GR_EBUSY, "resident scene (%llu B) exceeds the device-memory budget", (unsigned long long)total);
    }
    if ((st = rs->planes.reserve(pbytes)) != GR_OK || (mbytes && (st = rs->map.reserve(mbytes)) != GR_OK) ||
        (ebytes && (st = rs->ext.reserve(ebytes)) != GR_OK)) {
        rs->planes.release();
        rs->map.release();
        rs->ext.release();
        delete rs;
        return st;
    }
    cudaError_t e = cudaSuccess;
    if (sc->n_planes) e = cudaMemcpy(rs->planes.ptr, sc->planes, sc->n_planes * sizeof(gr_plane), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && mbytes) e = cudaMemcpy(rs->map.ptr, sc->env.latlong_rgb, mbytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ebytes) {
        e = cudaMemcpy(rs->ext.ptr, sc->material_ext->alpha_o_table, rs->S.ext_n * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy((float *)rs->ext.ptr + rs->S.ext_n, sc->material_ext->alpha_e_table,
                           rs->S.ext_n * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        rs->planes.release();
        rs->map.release();
        rs->ext.release();
        delete rs;
        return fail(GR_ECUDA, "scene upload failed: %s", cudaGetErrorString(e));
    }
    rs->bytes = total;
    rs->stone = grh::stone_key(sc);
    grh::tune_init(ctx, rs->tune, rs->stone);
    ctx->resident_bytes += total;
    uint64_t id = ctx->next_scene_id++;
    ctx->scenes[id] = rs;
    *out_id = id;
    return GR_OK;
}

gr_status gr_scene_release(gr_ctx *ctx, uint64_t id) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    if (it->second->users)
        return fail(GR_EBUSY, "scene %llu is in use by %u open frame stream(s) or bulk render(s)",
                    (unsigned long long)id, it->second->users);
    GR_CUDA(cudaSetDevice(ctx->device));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    ResidentScene *rs = it->second;
    ctx->resident_bytes -= rs->bytes;
    grh::tune_release(rs->tune);
    rs->planes.release();
    rs->map.release();
    rs->ext.release();
    delete rs;
    ctx->scenes.erase(it);
    return GR_OK;
}


}  // extern "C"

namespace grh {
gr_status render_resident_locked(gr_ctx *ctx, ResidentScene *rs, uint32_t sample_offset, uint32_t spp, float *film_dev,
                                 cudaStream_t s) {
    const uint64_t n_pixels = (uint64_t)rs->S.width * rs->S.height;
    gr_scene shape;
    std::memset(&shape, 0, sizeof(shape));
    shape.width = rs->S.width;
    shape.height = rs->S.height;
    int trial = -1;
    const StageCaps caps = tune_begin(ctx, rs->tune, rs->S, n_pixels, spp, s, trial);
    gr_status st = render_into(ctx, &shape, rs->S, resident_buffers(rs), sample_offset, spp, film_dev, s, caps);
    tune_end(rs->tune, trial, s);
    return st;
}
}  // namespace grh

extern "C" {

gr_status gr_render_resident(gr_ctx *ctx, uint64_t id, uint32_t sample_offset, uint32_t spp, float *film_dev,
                             void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    ResidentScene *rs = it->second;
    const uint64_t n_pixels = (uint64_t)rs->S.width * rs->S.height;
    if (spp == 0 || n_pixels == 0) return GR_OK;
    if (!film_dev) return fail(GR_EINVAL, "film is NULL");
    GR_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return grh::render_resident_locked(ctx, rs, sample_offset, spp, film_dev, s);
}

gr_status gr_scene_stage_caps(gr_ctx *ctx, uint64_t id, uint32_t *cap_first, uint32_t *cap_second) {
    if (!ctx || !cap_first || !cap_second) return fail(GR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    StageCapTune &T = it->second->tune;
    grh::tune_harvest(ctx, T);
    const StageCaps c = T.best < 0 ? StageCaps{} : schedule_candidate(T.best);
    *cap_first = c.first;
    *cap_second = c.second;
    return GR_OK;
}

gr_status gr_scene_schedule(gr_ctx *ctx, uint64_t id, uint32_t *cap_first, uint32_t *cap_second,
                            uint32_t *blocks_per_sm) {
    if (!ctx || !cap_first || !cap_second || !blocks_per_sm) return fail(GR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    StageCapTune &T = it->second->tune;
    grh::tune_harvest(ctx, T);
    const StageCaps c = T.best < 0 ? StageCaps{} : schedule_candidate(T.best);
    *cap_first = c.first;
    *cap_second = c.second;
    *blocks_per_sm = c.blocks;
    return GR_OK;
}

gr_status gr_scene_set_schedule(gr_ctx *ctx, uint64_t id, uint32_t cap_first, uint32_t cap_second,
                                uint32_t blocks_per_sm) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    ResidentScene *rs = it->second;
    if (cap_first == 0 && cap_second == 0 && blocks_per_sm == 0) {
        // open again: forget the stone's entry and time the candidates afresh
        ctx->tuned.erase(rs->stone);
        grh::tune_init(ctx, rs->tune, rs->stone);
        return GR_OK;
    }
    const int c = schedule_index(cap_first, cap_second, blocks_per_sm);
    if (c < 0)
        return fail(GR_EINVAL, "schedule (%u, %u, %u blocks/SM) is not a candidate", cap_first, cap_second,
                    blocks_per_sm);
    grh::tune_init(ctx, rs->tune, rs->stone);
    rs->tune.best = c;
    return GR_OK;
}

namespace {
// The identity line of a tuning table: what its timings are valid for.
std::string tuning_identity(const gr_ctx *ctx) {
    char buf[640];
    snprintf(buf, sizeof(buf), "gemray-schedules %d %s", GR_SCHEDULE_SET, ctx->label.c_str());
    return buf;
}

// Reads a tuning table's entries into `out` (entries naming no candidate are skipped);
// GR_EINVAL when it was written for another schedule set or device.
gr_status read_table(const char *path, const std::string &id, std::map<uint64_t, TunedSchedule> &out, uint32_t *n) {
    *n = 0;
    FILE *f = fopen(path, "r");
    if (!f) return fail(GR_ENOTFOUND, "cannot read %s", path);
    char line[1024];
    std::string head = fgets(line, sizeof(line), f) ? line : "";
    while (!head.empty() && (head.back() == '\n' || head.back() == '\r')) head.pop_back();
    if (head != id) {
        fclose(f);
        return fail(GR_EINVAL, "%s was not written for this schedule set and device (%s)", path, id.c_str());
    }
    while (fgets(line, sizeof(line), f)) {
        unsigned long long key = 0;
        unsigned first = 0, second = 0, blocks = 0;
        float ms = 0.0f;
        if (sscanf(line, "%llx %u %u %u %g", &key, &first, &second, &blocks, &ms) != 5 || key == 0) continue;
        const int c = schedule_index(first, second, blocks);
        if (c < 0) continue;
        out[key] = TunedSchedule{c, ms};
        ++*n;
    }
    fclose(f);
    return GR_OK;
}

// Writes the context's entries, merged over those the file already holds for this
// schedule set and device, through a temporary file renamed into place.
gr_status tuning_save_locked(gr_ctx *ctx, const char *path) {
    std::map<uint64_t, TunedSchedule> all;
    uint32_t n = 0;
    const std::string id = tuning_identity(ctx);
    read_table(path, id, all, &n);  // a missing or foreign table is replaced
    for (auto &kv : ctx->tuned) all[kv.first] = kv.second;
    const std::string tmp = std::string(path) + ".tmp." + std::to_string((long long)getpid());
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return fail(GR_EINVAL, "cannot write %s", tmp.c_str());
    fprintf(f, "%s\n", id.c_str());
    for (auto &kv : all) {
        const StageCaps c = schedule_candidate(kv.second.candidate);
        fprintf(f, "%016llx %u %u %u %.6g\n", (unsigned long long)kv.first, c.first, c.second, c.blocks,
                (double)kv.second.ms_per_mtuple);
    }
    const bool ok = fflush(f) == 0;
    fclose(f);
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return fail(GR_EINVAL, "cannot write %s", path);
    }
    return GR_OK;
}

gr_status tuning_load_locked(gr_ctx *ctx, const char *path, uint32_t *n_loaded) {
    uint32_t n = 0;
    if (n_loaded) *n_loaded = 0;
    const gr_status st = read_table(path, tuning_identity(ctx), ctx->tuned, &n);
    if (st != GR_OK) return st;
    // stones already resident or met by gr_accumulate, and still open, take their entry
    for (auto &kv : ctx->scenes) {
        StageCapTune &T = kv.second->tune;
        auto t = ctx->tuned.find(T.key);
        if (T.best < 0 && T.key && t != ctx->tuned.end()) T.best = t->second.candidate;
    }
    for (auto &kv : ctx->accum_tune) {
        auto t = ctx->tuned.find(kv.first);
        if (kv.second.best < 0 && t != ctx->tuned.end()) kv.second.best = t->second.candidate;
    }
    if (n_loaded) *n_loaded = n;
    return GR_OK;
}
}  // namespace

gr_status gr_tuning_save(gr_ctx *ctx, const char *path) {
    if (!ctx || !path) return fail(GR_EINVAL, "ctx or path is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (auto &kv : ctx->scenes) grh::tune_harvest(ctx, kv.second->tune);
    for (auto &kv : ctx->accum_tune) grh::tune_harvest(ctx, kv.second);
    return tuning_save_locked(ctx, path);
}

gr_status gr_tuning_load(gr_ctx *ctx, const char *path, uint32_t *n_loaded) {
    if (!ctx || !path) return fail(GR_EINVAL, "ctx or path is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    return tuning_load_locked(ctx, path, n_loaded);
}

gr_status gr_tuning_count(gr_ctx *ctx, uint32_t *n_entries) {
    if (!ctx || !n_entries) return fail(GR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (auto &kv : ctx->scenes) grh::tune_harvest(ctx, kv.second->tune);
    for (auto &kv : ctx->accum_tune) grh::tune_harvest(ctx, kv.second);
    *n_entries = (uint32_t)ctx->tuned.size();
    return GR_OK;
}

gr_status gr_render_resident_static(gr_ctx *ctx, uint64_t id, uint32_t sample_offset, uint32_t spp, float *film_dev,
                                    void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (spp > GR_STATIC_SCRATCH_TUPLES)
        return fail(GR_EINVAL, "spp %u does not fit the static scratch: at most %u samples per pixel per call", spp,
                    (unsigned)GR_STATIC_SCRATCH_TUPLES);
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)id);
    ResidentScene *rs = it->second;
    const uint64_t n_pixels = (uint64_t)rs->S.width * rs->S.height;
    if (spp == 0 || n_pixels == 0) return GR_OK;
    if (!film_dev) return fail(GR_EINVAL, "film is NULL");
    GR_CUDA(cudaSetDevice(ctx->device));
    float *scratch = nullptr;
    GR_CUDA((cudaError_t)grh::static_scratch(ctx->device, &scratch));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    const grd::SceneBuffers B = resident_buffers(rs);
    uint64_t chunk_pixels = GR_STATIC_SCRATCH_TUPLES / spp;
    if (chunk_pixels > n_pixels) chunk_pixels = n_pixels;
    for (uint64_t first = 0; first < n_pixels; first += chunk_pixels) {
        const uint64_t np = n_pixels - first < chunk_pixels ? n_pixels - first : chunk_pixels;
        grd::LaunchRange R;
        R.first_pixel = (uint32_t)first;
        R.n_pixels = (uint32_t)np;
        R.sample_offset = sample_offset;
        R.spp = spp;
        R.n_tuples = np * spp;
        gr_status st = grh::launch_trace(ctx, rs->S, B, R, scratch, s, GR_KERNEL_PLAIN);
        if (st != GR_OK) return st;
        ctx->trace_launches += 1;
        st = grh::launch_fold(scratch, (uint32_t)np, spp, (uint32_t)first, film_dev,
                              (rs->S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u, s);
        if (st != GR_OK) return st;
        ctx->fold_launches += 1;
    }
    return GR_OK;
}

gr_status gr_event_counts(gr_ctx *ctx, const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels,
                          uint32_t sample_offset, uint32_t spp, uint64_t *counts, uint32_t n_counts) {
    if (!ctx || !sc || !counts) return fail(GR_EINVAL, "NULL argument");
    if (n_counts < GR_EVENT_COUNT) return fail(GR_EINVAL, "counts needs %u entries", GR_EVENT_COUNT);
    if ((uint64_t)first_pixel + n_pixels > (uint64_t)sc->width * sc->height)
        return fail(GR_EINVAL, "pixel range exceeds the frame");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    SceneConst S;
    grd::SceneBuffers B;
    gr_status st = grh::prepare(ctx, sc, S, B);
    if (st != GR_OK) return st;
    uint64_t n_tuples = (uint64_t)n_pixels * spp;
    if (n_tuples == 0 || S.max_bounces == 0) {
        for (uint32_t i = 0; i < GR_EVENT_COUNT; ++i) counts[i] = 0;
        return GR_OK;
    }
    st = ctx->xyz.reserve((size_t)n_tuples * 3 * sizeof(float));
    if (st != GR_OK) return st;
    st = ctx->counter.reserve(sizeof(unsigned long long) * (1 + GR_EVENT_COUNT));
    if (st != GR_OK) return st;
    GR_CUDA(cudaMemsetAsync(ctx->counter.ptr, 0, sizeof(unsigned long long) * (1 + GR_EVENT_COUNT), ctx->stream));
    grd::LaunchRange R;
    R.first_pixel = first_pixel;
    R.n_pixels = n_pixels;
    R.sample_offset = sample_offset;
    R.spp = spp;
    R.n_tuples = n_tuples;
    unsigned long long *dc = (unsigned long long *)ctx->counter.ptr;
    size_t smem = grd::planes_smem_bytes(S.n_planes);
    uint64_t blocks = (n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS;
    if (grd::needs_extras(S))
        grd::k_trace_plain<grd::Counters, false, true><<<(unsigned)blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(
            S, B, R, (float *)ctx->xyz.ptr, dc + 1);
    else
        grd::k_trace_plain<grd::Counters><<<(unsigned)blocks, grd::TRACE_THREADS, smem, ctx->stream>>>(
            S, B, R, (float *)ctx->xyz.ptr, dc + 1);
    GR_CUDA(cudaGetLastError());
    unsigned long long host[1 + GR_EVENT_COUNT];
    GR_CUDA(cudaMemcpyAsync(host, dc, sizeof(host), cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    for (uint32_t i = 0; i < GR_EVENT_COUNT; ++i) counts[i] = host[1 + i];
    return GR_OK;
}

gr_status gr_probe_fp32_peak(gr_ctx *ctx, double *tflops) {
    if (!ctx || !tflops) return fail(GR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    gr_status st = ctx->counter.reserve(64);
    if (st != GR_OK) return st;
    const unsigned threads = 256, blocks = (unsigned)ctx->sm_count * 8;
    const uint32_t iters = 4096;
    cudaEvent_t a, b;
    GR_CUDA(cudaEventCreate(&a));
    GR_CUDA(cudaEventCreate(&b));
    grd::k_fp32_probe<<<blocks, threads, 0, ctx->stream>>>((float *)ctx->counter.ptr, 64, 1.0f);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a, ctx->stream);
        grd::k_fp32_probe<<<blocks, threads, 0, ctx->stream>>>((float *)ctx->counter.ptr, iters, 1.0f);
        cudaEventRecord(b, ctx->stream);
        GR_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    GR_CUDA(cudaGetLastError());
    double flops = (double)blocks * threads * iters * 16.0 * 8.0 * 2.0;
    *tflops = flops / (best * 1e-3) / 1e12;
    return GR_OK;
}

gr_status gr_timing_enable(gr_ctx *ctx, uint32_t on) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->timing = on != 0;
    ctx->trace_used = ctx->fold_used = 0;
    ctx->trace_launches = ctx->fold_launches = 0;
    return GR_OK;
}

gr_status gr_timing_read(gr_ctx *ctx, double *trace_ms, double *fold_ms, uint64_t *trace_launches,
                         uint64_t *fold_launches) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    double t = 0.0, f = 0.0;
    for (size_t i = 0; i < ctx->trace_used; ++i) {
        GR_CUDA(cudaEventSynchronize(ctx->trace_ev[i].second));
        float ms = 0.f;
        GR_CUDA(cudaEventElapsedTime(&ms, ctx->trace_ev[i].first, ctx->trace_ev[i].second));
        t += ms;
    }
    for (size_t i = 0; i < ctx->fold_used; ++i) {
        GR_CUDA(cudaEventSynchronize(ctx->fold_ev[i].second));
        float ms = 0.f;
        GR_CUDA(cudaEventElapsedTime(&ms, ctx->fold_ev[i].first, ctx->fold_ev[i].second));
        f += ms;
    }
    if (trace_ms) *trace_ms = t;
    if (fold_ms) *fold_ms = f;
    if (trace_launches) *trace_launches = ctx->trace_launches;
    if (fold_launches) *fold_launches = ctx->fold_launches;
    ctx->trace_used = ctx->fold_used = 0;
    ctx->trace_launches = ctx->fold_launches = 0;
    return GR_OK;
}

gr_status gr_optical_metrics(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const gr_material *material,
                             const gr_pose *poses, uint32_t n_poses, uint32_t flags, gr_metrics_out *out) {
    if (!ctx || !material || (n_poses && (!poses || !out))) return fail(GR_EINVAL, "NULL argument");
    if (n_planes > GR_MAX_PLANES) return fail(GR_EINVAL, "n_planes %u exceeds GR_MAX_PLANES", n_planes);
    if (n_planes && !planes) return fail(GR_EINVAL, "planes is NULL");
    if (n_poses == 0) return GR_OK;
    if (n_planes == 0) {
        // color/metrics.rs:1090-1103: no geometry -> the reference's placeholder values
        for (uint32_t i = 0; i < n_poses; ++i) out[i] = gr_metrics_out{85.0f, 25.0f, 75.0f, 5.0f, 5.0f};
        return GR_OK;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    gr_status st = grh::metrics_device(planes, n_planes, material, poses, n_poses, out, flags, ctx->stream, ctx->metrics);
    if (st == GR_ECUDA) return fail(st, "metrics launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return st;
}

gr_status gr_angular_profile(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const gr_material *material,
                             float cam_yaw, float light_yaw, float light_pitch, float *brilliance_19,
                             float *extinction_19, float *windowing_19) {
    if (!brilliance_19 || !extinction_19 || !windowing_19) return fail(GR_EINVAL, "NULL curve");
    gr_pose poses[19];
    const float to_rad = 3.14159265358979323846f / 180.0f;  // f32::to_radians
    for (int i = 0; i < 19; ++i) poses[i] = gr_pose{cam_yaw, (5.0f * (float)i) * to_rad, light_yaw, light_pitch};
    gr_metrics_out m[19];
    gr_status st = gr_optical_metrics(ctx, planes, n_planes, material, poses, 19, 0u, m);
    if (st != GR_OK) return st;
    for (int i = 0; i < 19; ++i) {
        brilliance_19[i] = m[i].brilliance_pct;
        extinction_19[i] = m[i].extinction_pct;
        windowing_19[i] = m[i].windowing_pct;
    }
    return GR_OK;
}

gr_status gr_set_kernel(gr_ctx *ctx, uint32_t kernel) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (kernel != GR_KERNEL_PLAIN && kernel != GR_KERNEL_WAVEFRONT && kernel != GR_KERNEL_REGEN &&
        kernel != GR_KERNEL_STAGED && kernel != GR_KERNEL_AUTO && kernel != GR_KERNEL_SORTED)
        return fail(GR_EINVAL, "unknown kernel %u", kernel);
    std::lock_guard<std::mutex> lk(ctx->mu);
    // the retired wavefront and regeneration schedules run AUTO's choice
    ctx->kernel_mode = (kernel == GR_KERNEL_WAVEFRONT || kernel == GR_KERNEL_REGEN) ? (int)GR_KERNEL_AUTO : (int)kernel;
    return GR_OK;
}

gr_status gr_synchronize(gr_ctx *ctx) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    GR_CUDA(cudaSetDevice(ctx->device));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

void *gr_stream(gr_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

}  // extern "C"
