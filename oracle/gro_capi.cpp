// gro_capi.cpp -- C entry points of the oracle for the Python test suite and the
// CPU-baseline leg of bench.py.
//
// TEST INFRASTRUCTURE ONLY (see gr_oracle.hpp).  Threading mirrors the reference
// worker's `trace_into` (apps/gemray-worker/src/render_core/mod.rs:220-317): one
// thread per core claiming rows through an atomic counter; each pixel's samples are
// summed in sample order from zero and the sum is then added once to the film.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "gr_oracle.hpp"
#include "gro_scene.hpp"

using namespace gro;

namespace {

template <class R>
void trace_pixel_samples(const gr_scene &sc, const MaterialCtx<R> &mc, const EnvCtx<R> &env, uint32_t pixel,
                         uint32_t sample_offset, uint32_t spp, float *per_sample /* spp*3 or null */,
                         double sum_out[3], EventLog *logs) {
    uint32_t x = pixel % sc.width, y = pixel / sc.width;
    PixelRotations rot = pixel_rotations(pixel);
    V3<R> sum;
    for (uint32_t s = 0; s < spp; ++s) {
        uint32_t sample_num = sample_offset + s;
        SampleDraws d = sample_draws(pixel, sample_num, rot);
        Ray<float> ray = generate_ray(sc.camera, (float)x, (float)y, (float)sc.width, (float)sc.height, d.jitter_x,
                                      d.jitter_y);
        EventLog *lg = logs ? &logs[s] : nullptr;
        if (lg) std::memset(lg, 0, sizeof(EventLog));
        V3<R> xyz = trace_spectral_ray<R>(ray, sc.planes, sc.n_planes, mc, env, sc.max_bounces, d.seed, d.hero_rand, lg,
                                          sc.finishes);
        if (per_sample) {
            per_sample[3 * s + 0] = (float)xyz.x;
            per_sample[3 * s + 1] = (float)xyz.y;
            per_sample[3 * s + 2] = (float)xyz.z;
        }
        sum = sum + xyz;
    }
    sum_out[0] = (double)sum.x; sum_out[1] = (double)sum.y; sum_out[2] = (double)sum.z;
}

template <class R>
int accumulate_impl(const gr_scene *sc, uint32_t sample_offset, uint32_t spp, float *accum_f, double *accum_d,
                    int threads) {
    if (!sc || (!accum_f && !accum_d)) return GR_EINVAL;
    if (spp == 0 || sc->width == 0 || sc->height == 0) return GR_OK;
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<R> mc = make_material<R>(sc->material, sc->material_ext);
    EnvCtx<R> env = make_env<R>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    std::atomic<uint32_t> next_row(0);
    auto worker = [&]() {
        for (;;) {
            uint32_t y = next_row.fetch_add(1);
            if (y >= sc->height) break;
            for (uint32_t x = 0; x < sc->width; ++x) {
                uint32_t p = y * sc->width + x;
                double s[3];
                trace_pixel_samples<R>(*sc, mc, env, p, sample_offset, spp, nullptr, s, nullptr);
                for (int c = 0; c < 3; ++c) {
                    if (accum_f) accum_f[3 * (size_t)p + c] = (float)((R)accum_f[3 * (size_t)p + c] + (R)s[c]);
                    if (accum_d) accum_d[3 * (size_t)p + c] += s[c];
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

}  // namespace

extern "C" {

uint32_t gro_hash_u32(uint32_t x) { return hash_u32(x); }

float gro_rng_draw(uint32_t seed, uint32_t bounce, uint32_t stream) { return rng_draw(seed, bounce, stream); }

float gro_radical_inverse(uint32_t n, uint32_t base) { return radical_inverse_base(n, base); }

// Bulk sampler: (pixel[i], sample[i]) -> seed, jitter_x, jitter_y, hero_rand.
void gro_sample_draws(const uint32_t *pixels, const uint32_t *samples, uint64_t n, uint32_t *seed, float *jx,
                      float *jy, float *hero) {
    for (uint64_t i = 0; i < n; ++i) {
        PixelRotations r = pixel_rotations(pixels[i]);
        SampleDraws d = sample_draws(pixels[i], samples[i], r);
        seed[i] = d.seed; jx[i] = d.jitter_x; jy[i] = d.jitter_y; hero[i] = d.hero_rand;
    }
}

void gro_camera_new(float yaw, float pitch, float distance, float fov_deg, gr_camera *out) {
    *out = camera_new(yaw, pitch, distance, fov_deg);
}

uint32_t gro_standard_round_brilliant(gr_plane *out, uint32_t cap) {
    std::vector<gr_plane> p = standard_round_brilliant();
    for (uint32_t i = 0; i < p.size() && i < cap; ++i) out[i] = p[i];
    return (uint32_t)p.size();
}

int gro_builtin_material(const char *name, gr_material *out) { return builtin_material(name, out) ? 0 : -1; }

void gro_white_balance(float temp_k, float out[3]) {
    V3<float> w = compute_illuminant_white_balance<float>(temp_k);
    out[0] = w.x; out[1] = w.y; out[2] = w.z;
}

// White-furnace analytic target (crates/gemray/tests/raytracer_tests.rs:2594-2600):
// sum over lambda = 380..780 nm of cie_1931_cmf(lambda) * rgb_to_spectral_radiance(
// [L0, L0, L0], lambda), then / 106.856, in the reference's f32 order.
void gro_furnace_target(float l0, float out[3]) {
    float t[3] = {0.0f, 0.0f, 0.0f};
    for (int step = 0; step <= 400; ++step) {
        const float lambda = 380.0f + (float)step;
        const float spec = rgb_to_spectral<float>(l0, l0, l0, lambda);
        float c[3];
        cmf_scalar<float>(lambda, c);
        for (int k = 0; k < 3; ++k) t[k] = t[k] + c[k] * spec;
    }
    for (int k = 0; k < 3; ++k) out[k] = t[k] / 106.856f;
}

float gro_studio_env(const float dir[3], float lambda, float temp_k, float spot_mult, float exposure, float yaw,
                     float pitch) {
    StudioRig<float> rig = studio_rig_new<float>(yaw, pitch);
    return studio_radiance<float>(V3<float>(dir[0], dir[1], dir[2]), lambda, temp_k, spot_mult, exposure, rig);
}

// Studio radiance with the blackbody factor supplied by the caller (isolates libm
// rounding of the blackbody from the rest of environment.rs:280-321).
float gro_studio_env_spec(const float dir[3], float spec, float spot_mult, float exposure, float yaw, float pitch) {
    StudioRig<float> rig = studio_rig_new<float>(yaw, pitch);
    V3<float> d = V3<float>(dir[0], dir[1], dir[2]).normalize();
    float bg = rmax(::fmaf(0.012f, ::fmaf(d.y, 0.5f, 0.5f), 0.015f), 0.005f) * exposure;
    float rad = bg * spec;
    float key_dot = rmax(d.dot(rig.key), 0.0f);
    if (key_dot > 0.0f) rad = ::fmaf(powi(key_dot, 28) * 12.0f * spot_mult * exposure, spec, rad);
    float fill_dot = rmax(d.dot(rig.fill), 0.0f);
    if (fill_dot > 0.0f) rad = ::fmaf(powi(fill_dot, 18) * 4.5f * exposure, spec, rad);
    for (int i = 0; i < 16; ++i) {
        float ring_dot = rmax(d.dot(rig.ring[i]), 0.0f);
        if (ring_dot > 0.96f) rad = ::fmaf(powi((ring_dot - 0.96f) / 0.04f, 6) * 22.0f * spot_mult * exposure, spec, rad);
    }
    return rad;
}

float gro_exp_poly(float x) { return M<float>::exp_poly(x); }

// One traced sample with an explicit ray (the golden tests' entry point,
// trace_spectral_ray / trace_spectral_ray_with_finish, transport.rs:420-454; the
// scene's finishes, when given, select frosted facets).  precision 32 or 64.
int gro_trace_ray(const gr_scene *sc, const float origin[3], const float dir[3], uint32_t seed, float hero_rand,
                  uint32_t max_bounces, int precision, double xyz_out[3], uint32_t *bounces, uint32_t *termination) {
    Ray<float> ray;
    ray.origin = V3<float>(origin[0], origin[1], origin[2]);
    ray.dir = V3<float>(dir[0], dir[1], dir[2]);
    EventLog lg;
    std::memset(&lg, 0, sizeof(lg));
    if (precision == 64) {
        MaterialCtx<double> mc = make_material<double>(sc->material, sc->material_ext);
        EnvCtx<double> env = make_env<double>(sc->env);
        V3<double> x = trace_spectral_ray<double>(ray, sc->planes, sc->n_planes, mc, env, max_bounces, seed, hero_rand, &lg,
                                                  sc->finishes);
        xyz_out[0] = x.x; xyz_out[1] = x.y; xyz_out[2] = x.z;
    } else {
        MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
        EnvCtx<float> env = make_env<float>(sc->env);
        V3<float> x = trace_spectral_ray<float>(ray, sc->planes, sc->n_planes, mc, env, max_bounces, seed, hero_rand, &lg,
                                                 sc->finishes);
        xyz_out[0] = x.x; xyz_out[1] = x.y; xyz_out[2] = x.z;
    }
    if (bounces) *bounces = lg.bounces;
    if (termination) *termination = lg.termination;
    return 0;
}

// The sample loop of the reference's CPU property tests (raytracer_tests.rs:2322-2372,
// 2411-2460, 2710-2760; scattering.rs scattering_tests): a grid x grid view through the
// scene's camera at pixel centres, sample s of pixel p seeded hash(p ^ hash(s ^ salt)),
// hero_rand = hash(seed) / 4294967295, radiance summed in a Vec3 of f32 and divided
// once by the sample count.  Declined materials return GR_DECLINED_MATERIAL.
int gro_probe_grid(const gr_scene *sc, uint32_t grid, uint32_t spp, uint32_t salt, uint32_t max_bounces,
                   float mean_out[3]) {
    if (!sc || !mean_out || grid == 0 || spp == 0) return GR_EINVAL;
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    const float g = (float)grid;
    V3<float> sum(0.f, 0.f, 0.f);
    uint32_t count = 0;
    for (uint32_t iy = 0; iy < grid; ++iy) {
        for (uint32_t ix = 0; ix < grid; ++ix) {
            const Ray<float> ray = generate_ray(sc->camera, (float)ix, (float)iy, g, g, 0.5f, 0.5f);
            const uint32_t pixel_id = iy * grid + ix;
            for (uint32_t s = 0; s < spp; ++s) {
                const uint32_t seed = hash_u32(pixel_id ^ hash_u32(s ^ salt));
                const float hero = (float)hash_u32(seed) / 4294967295.0f;
                EventLog lg;
                std::memset(&lg, 0, sizeof(lg));
                sum = sum + trace_spectral_ray<float>(ray, sc->planes, sc->n_planes, mc, env, max_bounces, seed, hero,
                                                      &lg, sc->finishes);
                ++count;
            }
        }
    }
    const float c = (float)count;
    mean_out[0] = sum.x / c; mean_out[1] = sum.y / c; mean_out[2] = sum.z / c;
    return GR_OK;
}

// downsample_preview (apps/gemray-worker/src/stream_emit/downsample.rs:17-53): the box
// mean of the running total over each preview pixel's source block, summed row by row
// from zero in f32 and divided by the count as f32.
void gro_downsample_preview(const float *src, uint32_t w, uint32_t h, uint32_t tw, uint32_t th, float *out) {
    const size_t TW = tw ? tw : 1, TH = th ? th : 1;
    for (size_t i = 0; i < 3 * TW * TH; ++i) out[i] = 0.0f;
    if (w == 0 || h == 0) return;
    for (size_t oy = 0; oy < TH; ++oy) {
        const size_t y0 = oy * h / TH;
        size_t y1 = (oy + 1) * h / TH;
        if (y1 < y0 + 1) y1 = y0 + 1;
        if (y1 > h) y1 = h;
        for (size_t ox = 0; ox < TW; ++ox) {
            const size_t x0 = ox * w / TW;
            size_t x1 = (ox + 1) * w / TW;
            if (x1 < x0 + 1) x1 = x0 + 1;
            if (x1 > w) x1 = w;
            float s[3] = {0.0f, 0.0f, 0.0f};
            uint32_t count = 0;
            for (size_t y = y0; y < y1; ++y)
                for (size_t x = x0; x < x1; ++x) {
                    const float *p = src + 3 * (y * w + x);
                    s[0] = s[0] + p[0];
                    s[1] = s[1] + p[1];
                    s[2] = s[2] + p[2];
                    ++count;
                }
            float *o = out + 3 * (oy * TW + ox);
            if (count) {
                const float c = (float)count;
                o[0] = s[0] / c; o[1] = s[1] / c; o[2] = s[2] / c;
            }
        }
    }
}

// The denoiser's guide pass (apps/diagram-gui/src/bridge/guide_pass.rs:
// generate_guide_buffers): per pixel the primary ray through the pixel's corner
// (generate_ray with zero jitter) against the stone -- t, the hit plane's normal and
// its index, or (1e6, 0, -1) on a miss.
void gro_guide_buffers(const gr_scene *sc, float *depth, float *normal, int32_t *facet) {
    const float w = (float)sc->width, h = (float)sc->height;
    for (uint32_t y = 0; y < sc->height; ++y)
        for (uint32_t x = 0; x < sc->width; ++x) {
            const size_t i = (size_t)y * sc->width + x;
            const Ray<float> ray = generate_ray(sc->camera, (float)x, (float)y, w, h, 0.0f, 0.0f);
            const Hit<float> hit = intersect_polyhedron<float>(ray, sc->planes, sc->n_planes);
            depth[i] = hit.hit ? hit.t : 1.0e6f;
            normal[3 * i + 0] = hit.hit ? hit.normal.x : 0.0f;
            normal[3 * i + 1] = hit.hit ? hit.normal.y : 0.0f;
            normal[3 * i + 2] = hit.hit ? hit.normal.z : 0.0f;
            facet[i] = hit.hit ? hit.facet : -1;
        }
}

// Edge-avoiding A-Trous denoiser (crates/gemray/src/renderer/denoise/mod.rs:154-690),
// single-threaded (the reference's result is thread-count invariant): taper of the
// colour sigma with spp, identity copy below the taper epsilon, 1..8 passes of the
// dilated 5x5 B3 kernel gated by facet id, normal cosine power, depth and colour.
namespace atrous {
static inline float sanitize(float v) { return std::isfinite(v) ? v : 0.0f; }
static inline float cos_pow(float base, float power) {  // :294-311
    if (power >= 0.0f && power == std::floor(power) && power <= 4294967295.0f) {
        const uint32_t ip = (uint32_t)power;
        if (ip != 0 && (ip & (ip - 1)) == 0) {
            float v = base;
            for (uint32_t k = ip; k > 1; k >>= 1) v *= v;
            return v;
        }
    }
    return ::powf(base, power);
}
}  // namespace atrous

float gro_taper_strength(uint32_t spp, float n0_in) {  // :244-250
    const float n0 = rmax(n0_in, 1.0e-8f);
    return 1.0f / ::sqrtf(1.0f + (float)spp / n0);
}

float gro_cos_pow(float base, float power) { return atrous::cos_pow(base, power); }

void gro_atrous_denoise(const float *color, const float *depth, const float *normal, const int32_t *facet, uint32_t w,
                        uint32_t h, uint32_t spp, uint32_t num_passes_in, float sigma_color, float sigma_depth_in,
                        float normal_power, float taper_ref, float taper_eps, float *out) {
    using namespace atrous;
    const size_t len = (size_t)w * h;
    if (len == 0) return;
    const float taper = gro_taper_strength(spp, taper_ref);
    const uint32_t num_passes = num_passes_in < 1 ? 1 : (num_passes_in > 8 ? 8 : num_passes_in);
    if (taper < taper_eps) {
        std::memcpy(out, color, len * 3 * sizeof(float));
        return;
    }
    const float sce = rmax(sigma_color * taper, 0.0f);
    std::vector<float> ping(color, color + 3 * len), pong(3 * len), nn(3 * len);
    for (size_t i = 0; i < len; ++i) {  // unit_normal_or_zero (:268-276)
        const V3<float> n(sanitize(normal[3 * i]), sanitize(normal[3 * i + 1]), sanitize(normal[3 * i + 2]));
        const float l = ::sqrtf(n.dot(n));
        const bool z = l <= 1.0e-8f;
        nn[3 * i + 0] = z ? 0.0f : n.x / l;
        nn[3 * i + 1] = z ? 0.0f : n.y / l;
        nn[3 * i + 2] = z ? 0.0f : n.z / l;
    }
    const float sd = rmax(sigma_depth_in, 1.0e-8f);
    const float scs = rmax(sce * sce, 1.0e-8f);
    const float nisd = -1.0f / sd;
    const float nits = -1.0f / (2.0f * scs);
    const float np = rmax(normal_power, 0.0f);
    static const float B3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    for (uint32_t pass = 0; pass < num_passes; ++pass) {
        const int64_t stride = (int64_t)1 << pass;
        for (int64_t y = 0; y < (int64_t)h; ++y)
            for (int64_t x = 0; x < (int64_t)w; ++x) {  // atrous_pixel (:383-444)
                const size_t c = (size_t)y * w + x;
                const V3<float> cc(ping[3 * c], ping[3 * c + 1], ping[3 * c + 2]);
                const V3<float> cn(nn[3 * c], nn[3 * c + 1], nn[3 * c + 2]);
                const bool cn_zero = cn.x == 0.0f && cn.y == 0.0f && cn.z == 0.0f;
                const float cdep = sanitize(depth[c]);
                V3<float> sum(0.0f, 0.0f, 0.0f);
                float wsum = 0.0f;
                for (int ky = 0; ky < 5; ++ky) {
                    const int64_t sy = y + (ky - 2) * stride;
                    if (sy < 0 || sy >= (int64_t)h) continue;
                    for (int kx = 0; kx < 5; ++kx) {
                        const int64_t sx = x + (kx - 2) * stride;
                        if (sx < 0 || sx >= (int64_t)w) continue;
                        const size_t q = (size_t)sy * w + sx;
                        const float kw = B3[ky] * B3[kx];
                        const float wf = facet[c] == facet[q] ? 1.0f : 0.0f;
                        if (wf == 0.0f) continue;
                        const V3<float> qn(nn[3 * q], nn[3 * q + 1], nn[3 * q + 2]);
                        float wn = 1.0f;
                        if (!cn_zero && !(qn.x == 0.0f && qn.y == 0.0f && qn.z == 0.0f))
                            wn = cos_pow(rmax(clampr(cn.dot(qn), -1.0f, 1.0f), 0.0f), np);
                        const float wd = ::expf(std::fabs(cdep - sanitize(depth[q])) * nisd);
                        const V3<float> qc(ping[3 * q], ping[3 * q + 1], ping[3 * q + 2]);
                        const V3<float> dc(sanitize(cc.x) - sanitize(qc.x), sanitize(cc.y) - sanitize(qc.y),
                                           sanitize(cc.z) - sanitize(qc.z));
                        const float wc = ::expf(dc.dot(dc) * nits);
                        const float wgt = (((kw * wf) * wn) * wd) * wc;
                        sum = sum + qc * wgt;
                        wsum = wsum + wgt;
                    }
                }
                float *o = &pong[3 * c];
                if (wsum > 1.0e-8f) {
                    o[0] = sum.x / wsum; o[1] = sum.y / wsum; o[2] = sum.z / wsum;
                } else {
                    o[0] = cc.x; o[1] = cc.y; o[2] = cc.z;
                }
            }
        ping.swap(pong);
    }
    std::memcpy(out, ping.data(), len * 3 * sizeof(float));
}

// shading_normal_near_edge (optics/raytracer/intersect.rs:196-229), for the edge
// rounding unit tests.
void gro_shading_normal(const gr_plane *planes, uint32_t n, const float hp[3], int hit_idx, const float hn[3],
                        float radius, float out[3]) {
    const V3<float> r = shading_normal_near_edge<float>(planes, n, V3<float>(hp[0], hp[1], hp[2]), hit_idx,
                                                        V3<float>(hn[0], hn[1], hn[2]), radius);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// BiaxialIndicatrix entry points (optics/birefringence.rs:349-839) for the property
// tests: an indicatrix from three principal indices and a frame given as columns
// (ax0, ax1, ax2), or from a material at a wavelength (materials.rs:1508-1519).
static Indicatrix<float> ind_from(float na, float nb, float ng, const float axes[9]) {
    Indicatrix<float> I;
    I.na = na; I.nb = nb; I.ng = ng;
    I.ax0 = V3<float>(axes[0], axes[1], axes[2]);
    I.ax1 = V3<float>(axes[3], axes[4], axes[5]);
    I.ax2 = V3<float>(axes[6], axes[7], axes[8]);
    return I;
}

void gro_biaxial_wave_indices(float na, float nb, float ng, const float axes[9], const float wn[3], float out[2]) {
    wave_indices(ind_from(na, nb, ng, axes), V3<float>(wn[0], wn[1], wn[2]), out[0], out[1]);
}

void gro_biaxial_eigen(float na, float nb, float ng, const float axes[9], const float wn[3], float d_slow[3],
                       float d_fast[3]) {
    V3<float> s, f;
    eigen_polarizations(ind_from(na, nb, ng, axes), V3<float>(wn[0], wn[1], wn[2]), s, f);
    d_slow[0] = s.x; d_slow[1] = s.y; d_slow[2] = s.z;
    d_fast[0] = f.x; d_fast[1] = f.y; d_fast[2] = f.z;
}

void gro_biaxial_poynting(float na, float nb, float ng, const float axes[9], const float wn[3], int want_slow,
                          float out[3]) {
    const V3<float> d = mode_poynting_dir(ind_from(na, nb, ng, axes), V3<float>(wn[0], wn[1], wn[2]), want_slow != 0);
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

int gro_material_indicatrix(const gr_material *m, float lambda_nm, float n_out[3], float axes_out[9]) {
    if (!m || !m->dispersion.has_biaxial_delta) return -1;
    const V3<float> c(m->dispersion.c_axis_and_birefringence[0], m->dispersion.c_axis_and_birefringence[1],
                      m->dispersion.c_axis_and_birefringence[2]);
    const Indicatrix<float> I = make_indicatrix<float>(dispersion_evaluate<float>(m->dispersion, lambda_nm),
                                                       m->dispersion.biaxial_delta_beta_alpha,
                                                       m->dispersion.c_axis_and_birefringence[3], c);
    n_out[0] = I.na; n_out[1] = I.nb; n_out[2] = I.ng;
    const V3<float> ax[3] = {I.ax0, I.ax1, I.ax2};
    for (int i = 0; i < 3; ++i) { axes_out[3 * i] = ax[i].x; axes_out[3 * i + 1] = ax[i].y; axes_out[3 * i + 2] = ax[i].z; }
    return 0;
}

// The two direction samplers of the frosted and scattering paths (scattering.rs:
// 356-362 cosine_weighted_hemisphere, 428-443 sample_henyey_greenstein_direction).
void gro_cosine_hemisphere(float u1, float u2, const float n[3], float out[3]) {
    const V3<float> d = cosine_weighted_hemisphere<float>(u1, u2, V3<float>(n[0], n[1], n[2]));
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

void gro_sample_hg(float u1, float u2, float g, const float fwd[3], float out[3]) {
    const V3<float> d = sample_hg_direction<float>(u1, u2, g, V3<float>(fwd[0], fwd[1], fwd[2]));
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

// CPU baseline: the listed rows only; threads claim 16-pixel runs of those rows from
// an atomic counter (the reference worker claims whole rows, apps/gemray-worker/src/
// render_core/mod.rs:241-316 -- pixel runs keep every core busy on a small row
// sample).  accum is the full W*H*3 film; each pixel's samples are summed in sample
// order and added once.
int gro_accumulate_rows(const gr_scene *sc, const uint32_t *rows, uint32_t n_rows, uint32_t sample_offset,
                        uint32_t spp, float *accum, int threads) {
    if (!sc || !rows || !accum) return GR_EINVAL;
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    const uint32_t RUN = 16;
    const uint64_t runs_per_row = (sc->width + RUN - 1) / RUN;
    const uint64_t total = runs_per_row * n_rows;
    std::atomic<uint64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            uint64_t i = next.fetch_add(1);
            if (i >= total) break;
            uint32_t y = rows[i / runs_per_row];
            if (y >= sc->height) continue;
            uint32_t x0 = (uint32_t)(i % runs_per_row) * RUN;
            for (uint32_t x = x0; x < x0 + RUN && x < sc->width; ++x) {
                uint32_t p = y * sc->width + x;
                double s[3];
                trace_pixel_samples<float>(*sc, mc, env, p, sample_offset, spp, nullptr, s, nullptr);
                for (int c = 0; c < 3; ++c) accum[3 * (size_t)p + c] = accum[3 * (size_t)p + c] + (float)s[c];
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

// Film accumulation, FP32: accum (W*H*3 floats) += per-pixel sample sums.
int gro_accumulate(const gr_scene *sc, uint32_t sample_offset, uint32_t spp, float *accum, int threads) {
    return accumulate_impl<float>(sc, sample_offset, spp, accum, nullptr, threads);
}

// Film accumulation, FP64 oracle: accum (W*H*3 doubles) += per-pixel sample sums.
int gro_accumulate_f64(const gr_scene *sc, uint32_t sample_offset, uint32_t spp, double *accum, int threads) {
    return accumulate_impl<double>(sc, sample_offset, spp, nullptr, accum, threads);
}

// Per-sample XYZ of pixels [first_pixel, first_pixel+n_pixels), samples
// [offset, offset+spp) -> xyz_out[(p*spp + s)*3 + c] (FP32 oracle), plus optional
// per-sample bounce counts / termination reasons / event counts.
int gro_trace_samples(const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels, uint32_t sample_offset,
                      uint32_t spp, float *xyz_out, uint32_t *bounces, uint32_t *term, uint32_t *counts /* 6 per sample */,
                      int threads) {
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        std::vector<EventLog> logs(spp);
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= n_pixels) break;
            uint32_t p = first_pixel + i;
            double s[3];
            trace_pixel_samples<float>(*sc, mc, env, p, sample_offset, spp, xyz_out + (size_t)i * spp * 3, s, logs.data());
            for (uint32_t k = 0; k < spp; ++k) {
                size_t o = (size_t)i * spp + k;
                if (bounces) bounces[o] = logs[k].bounces;
                if (term) term[o] = logs[k].termination;
                if (counts) {
                    counts[6 * o + 0] = logs[k].n_tir;
                    counts[6 * o + 1] = logs[k].n_reflect;
                    counts[6 * o + 2] = logs[k].n_refract;
                    counts[6 * o + 3] = logs[k].n_inside_abs;
                    counts[6 * o + 4] = logs[k].n_escape;
                    counts[6 * o + 5] = logs[k].n_chan_tir;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

}  // extern "C"

// Per-sample XYZ and luminance-weighted Stokes vector (I, Q, U, V) of the FP32 tracer
// (the Stokes film's oracle), (pixel, sample) order: xyz n*3, iquv n*4; and the films:
// accum_xyz (W*H*3) and accum_iquv (W*H*4) += each pixel's sample-order sums.
template <class R>
static void stokes_pixel(const gr_scene &sc, const MaterialCtx<R> &mc, const EnvCtx<R> &env, uint32_t pixel,
                         uint32_t sample_offset, uint32_t spp, float *xyz, float *iquv, float sum_x[3], float sum_s[4]) {
    const uint32_t x = pixel % sc.width, y = pixel / sc.width;
    const PixelRotations rot = pixel_rotations(pixel);
    for (int c = 0; c < 3; ++c) sum_x[c] = 0.0f;
    for (int c = 0; c < 4; ++c) sum_s[c] = 0.0f;
    for (uint32_t s = 0; s < spp; ++s) {
        const SampleDraws d = sample_draws(pixel, sample_offset + s, rot);
        const Ray<float> ray = generate_ray(sc.camera, (float)x, (float)y, (float)sc.width, (float)sc.height, d.jitter_x,
                                            d.jitter_y);
        R so[4];
        const V3<R> v = trace_spectral_ray<R>(ray, sc.planes, sc.n_planes, mc, env, sc.max_bounces, d.seed, d.hero_rand,
                                              nullptr, sc.finishes, so);
        const float fx[3] = {(float)v.x, (float)v.y, (float)v.z};
        for (int c = 0; c < 3; ++c) {
            if (xyz) xyz[3 * s + c] = fx[c];
            sum_x[c] = sum_x[c] + fx[c];
        }
        for (int c = 0; c < 4; ++c) {
            if (iquv) iquv[4 * s + c] = (float)so[c];
            sum_s[c] = sum_s[c] + (float)so[c];
        }
    }
}

extern "C" int gro_trace_samples_stokes(const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels,
                                        uint32_t sample_offset, uint32_t spp, float *xyz_out, float *iquv_out,
                                        int threads) {
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= n_pixels) break;
            float sx[3], ss[4];
            stokes_pixel<float>(*sc, mc, env, first_pixel + i, sample_offset, spp, xyz_out + (size_t)i * spp * 3,
                                iquv_out + (size_t)i * spp * 4, sx, ss);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

extern "C" int gro_accumulate_stokes(const gr_scene *sc, uint32_t sample_offset, uint32_t spp, float *accum_xyz,
                                     float *accum_iquv, int threads) {
    if (!sc || !accum_xyz || !accum_iquv) return GR_EINVAL;
    if (spp == 0 || sc->width == 0 || sc->height == 0) return GR_OK;
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    const uint32_t n = sc->width * sc->height;
    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        for (;;) {
            const uint32_t p = next.fetch_add(1);
            if (p >= n) break;
            float sx[3], ss[4];
            stokes_pixel<float>(*sc, mc, env, p, sample_offset, spp, nullptr, nullptr, sx, ss);
            for (int c = 0; c < 3; ++c) accum_xyz[3 * (size_t)p + c] = accum_xyz[3 * (size_t)p + c] + sx[c];
            for (int c = 0; c < 4; ++c) accum_iquv[4 * (size_t)p + c] = accum_iquv[4 * (size_t)p + c] + ss[c];
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

extern "C" {

// Per-sample XYZ of the FP64 twin (values rounded to f32), for per-sample agreement
// checks against the f32 engine.
int gro_trace_samples_f64(const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels, uint32_t sample_offset,
                          uint32_t spp, float *xyz_out, int threads) {
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<double> mc = make_material<double>(sc->material, sc->material_ext);
    EnvCtx<double> env = make_env<double>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= n_pixels) break;
            double s[3];
            trace_pixel_samples<double>(*sc, mc, env, first_pixel + i, sample_offset, spp,
                                        xyz_out + (size_t)i * spp * 3, s, nullptr);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

// tonemap_to_rgba (renderer/tonemap.rs:52-108): rgba[i] = encode(xyz[i] * scale).
void gro_tonemap(const float *xyz, float scale, uint32_t n, uint8_t *rgba) {
    for (uint32_t i = 0; i < n; ++i) {
        V3<float> c(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
        srgb_encode(c * scale, rgba + 4 * (size_t)i);
    }
}

// Sampler records (renderer/gpu/rng_check.rs cpu_record): seed, jitter, hero and
// the Fresnel / roulette / split / coupling draws of bounces 0..3 (20 words each).
void gro_rng_records(const uint32_t *pixels, const uint32_t *samples, uint32_t n, uint32_t *out) {
    for (uint32_t i = 0; i < n; ++i) {
        PixelRotations r = pixel_rotations(pixels[i]);
        SampleDraws d = sample_draws(pixels[i], samples[i], r);
        uint32_t *o = out + 20 * (size_t)i;
        float f[19];
        f[0] = d.jitter_x; f[1] = d.jitter_y; f[2] = d.hero_rand;
        const uint32_t streams[4] = {FRESNEL_BRANCH_STREAM, RUSSIAN_ROULETTE_STREAM, BIREFRINGENT_SPLIT_STREAM,
                                     MODE_COUPLING_STREAM};
        for (uint32_t b = 0; b < 4; ++b)
            for (int k = 0; k < 4; ++k) f[3 + 4 * b + k] = rng_draw(d.seed, b, streams[k]);
        o[0] = d.seed;
        std::memcpy(o + 1, f, sizeof(f));
    }
}

// Material cache of one wavelength (build_ray_wavelength_cache, refraction.rs:127-174,
// with the extension's tabulated absorption and Cauchy n_e): out = n_o, n_e,
// alpha_o, alpha_e.  precision 32 or 64.
int gro_material_channel(const gr_material *m, const gr_material_ext *ext, float lambda_nm, int precision,
                         double out[4]) {
    if (!m || !out) return GR_EINVAL;
    if (precision == 64) {
        MaterialCtx<double> mc = make_material<double>(m, ext);
        double lam[8];
        for (double &l : lam) l = (double)lambda_nm;
        WaveCache<double> wc = build_cache(mc, lam);
        out[0] = wc.n_o[0]; out[1] = wc.n_o[0] + wc.n_e_delta[0];
        out[2] = wc.tensor[0].alpha.x; out[3] = wc.tensor[0].alpha.z;
    } else {
        MaterialCtx<float> mc = make_material<float>(m, ext);
        float lam[8];
        for (float &l : lam) l = lambda_nm;
        WaveCache<float> wc = build_cache(mc, lam);
        out[0] = wc.n_o[0]; out[1] = wc.n_o[0] + wc.n_e_delta[0];
        out[2] = wc.tensor[0].alpha.x; out[3] = wc.tensor[0].alpha.z;
    }
    return GR_OK;
}

// Per-sample event sequences of the FP32 tracer (the instrumented trace,
// transport.rs:512-537): the layout of gr_trace_events -- per tuple the final bounce
// index and termination, and per logged bounce (b < min(kmax, 64)) the facet, its
// hit distance and the event; unrecorded slots -1 / 0 / 0xFF.
int gro_trace_events(const gr_scene *sc, uint32_t first_pixel, uint32_t n_pixels, uint32_t sample_offset,
                     uint32_t spp, uint32_t kmax, uint32_t *bounces, uint32_t *term, int32_t *facets, float *t_hits,
                     uint8_t *events, int threads) {
    if (!sc || !bounces || !term || (kmax && (!facets || !t_hits || !events))) return GR_EINVAL;
    if (!material_supported(sc->material, sc->finishes, sc->n_planes)) return GR_DECLINED_MATERIAL;
    MaterialCtx<float> mc = make_material<float>(sc->material, sc->material_ext);
    EnvCtx<float> env = make_env<float>(sc->env);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    std::atomic<uint32_t> next(0);
    auto worker = [&]() {
        std::vector<EventLog> logs(spp);
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= n_pixels) break;
            double s[3];
            trace_pixel_samples<float>(*sc, mc, env, first_pixel + i, sample_offset, spp, nullptr, s, logs.data());
            for (uint32_t k = 0; k < spp; ++k) {
                const size_t o = (size_t)i * spp + k;
                const EventLog &lg = logs[k];
                bounces[o] = lg.bounces;
                term[o] = lg.termination;
                const uint32_t rec = lg.bounces + (lg.termination == TERM_RUSSIAN_ROULETTE ? 1u : 0u);
                for (uint32_t b = 0; b < kmax; ++b) {
                    const bool have = b < rec && b < 64;
                    facets[o * kmax + b] = have ? lg.facets[b] : -1;
                    t_hits[o * kmax + b] = have ? lg.ts[b] : 0.0f;
                    events[o * kmax + b] = have ? lg.events[b] : (uint8_t)0xFF;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return GR_OK;
}

}  // extern "C"

namespace {

// One case of a per-function bank (the layouts of GR_BANK_* in gemray_cuda.h) in
// precision R, each through the oracle's restatement of the reference function.
template <class R>
void bank_case(uint32_t bank, const gr_scene *sc, const float *x, double *y) {
    auto v = [&](int i) { return V3<R>(R(x[i]), R(x[i + 1]), R(x[i + 2])); };
    auto st = [&](int i) { return Stokes<R>{R(x[i]), R(x[i + 1]), R(x[i + 2]), R(x[i + 3])}; };
    auto put3 = [&](const V3<R> &a, int o) { y[o] = a.x; y[o + 1] = a.y; y[o + 2] = a.z; };
    auto put4 = [&](const Stokes<R> &a) { y[0] = a.i; y[1] = a.q; y[2] = a.u; y[3] = a.v; };
    switch (bank) {
    case GR_BANK_CAMERA_RAY: {
        Ray<R> r = generate_ray_t<R>(sc->camera, R(x[0]), R(x[1]), R((float)sc->width), R((float)sc->height), R(x[2]),
                                     R(x[3]));
        put3(r.dir, 0);
        break;
    }
    case GR_BANK_CMF: {
        R lam[8], c[8][3];
        for (R &l : lam) l = R(x[0]);
        cmf_x8(lam, c);
        y[0] = c[0][0]; y[1] = c[0][1]; y[2] = c[0][2];
        break;
    }
    case GR_BANK_BLACKBODY: y[0] = blackbody_spectrum(R(x[0]), R(sc->env.temp_k)); break;
    case GR_BANK_DISPERSION: y[0] = dispersion_evaluate(sc->material->dispersion, R(x[0])); break;
    case GR_BANK_ABSORPTION: {
        const gr_material *m = sc->material;
        const gr_material_ext *e = sc->material_ext;
        if (e && e->n_absorption > 0) {
            y[0] = table_lookup(e->alpha_o_table, e->n_absorption, e->absorption_nm_first, e->absorption_nm_step, R(x[0]));
            y[1] = table_lookup(e->alpha_e_table, e->n_absorption, e->absorption_nm_first, e->absorption_nm_step, R(x[0]));
        } else {
            y[0] = spectral_absorption(m->o_ray_bands, m->o_ray_band_count, R(x[0]));
            y[1] = spectral_absorption(m->e_ray_bands, m->e_ray_band_count, R(x[0]));
        }
        break;
    }
    case GR_BANK_PLEOCHROIC: {
        const MaterialCtx<R> mc = make_material<R>(sc->material, sc->material_ext);
        const Stokes<R> s = st(0);
        const V3<R> k = v(7);
        const Tensor3<R> t = tensor_uniaxial(R(x[10]), R(x[11]), mc.c_axis);
        const V3<R> e_hat = electric_field_direction(s, v(4), k);
        const V3<R> ea = ordinary_eigen_polarization(k, mc.c_axis), eb = extraordinary_eigen_polarization(k, mc.c_axis);
        y[0] = effective_pleochroic_alpha(t, e_hat, ea, eb, s.degree_of_polarization());
        break;
    }
    case GR_BANK_FRESNEL_REFLECTION: put4(apply_matrix(st(2), fresnel_reflection(R(x[0]), R(x[1])))); break;
    case GR_BANK_FRESNEL_TRANSMISSION:
        put4(apply_matrix(st(6), fresnel_transmission(R(x[0]), R(x[1]), R(x[2]), R(x[3]), R(x[4]), R(x[5]))));
        break;
    case GR_BANK_FRAME_ROTATION: put4(apply_matrix(st(1), frame_rotation(R(x[0])))); break;
    case GR_BANK_TIR_RETARDATION: put4(apply_matrix(st(1), tir_retardation(R(x[0])))); break;
    case GR_BANK_SIGNED_PSI: y[0] = signed_frame_rotation_psi(v(0), v(3), v(6)); break;
    case GR_BANK_TIR_PHASE_DELTA: y[0] = tir_phase_delta(R(x[0]), R(x[1]), R(x[2])); break;
    case GR_BANK_EIGEN_UNIAXIAL:
        put3(ordinary_eigen_polarization(v(0), v(3)), 0);
        put3(extraordinary_eigen_polarization(v(0), v(3)), 3);
        break;
    case GR_BANK_WALK_OFF: put3(extraordinary_poynting_dir(v(0), v(3), R(x[6]), R(x[7])), 0); break;
    case GR_BANK_EXTRAORDINARY_INDEX: y[0] = effective_extraordinary_index(R(x[0]), R(x[1]), R(x[2])); break;
    case GR_BANK_THETA_C: {
        const MaterialCtx<R> mc = make_material<R>(sc->material, sc->material_ext);
        const V3<R> k = v(0), n = v(3);
        const R cos_i = clampr((-k).dot(n), R(0), R(1));
        y[0] = theta_c_for_bounce(k, n, cos_i, R(x[6]), R(x[7]), mc.c_axis, x[8] != 0.0f);
        break;
    }
    case GR_BANK_STUDIO: {
        const StudioRig<R> rig = studio_rig_new(R(sc->env.light_yaw), R(sc->env.light_pitch));
        y[0] = studio_radiance(v(0), R(x[3]), R(sc->env.temp_k), R(sc->env.spot_mult), R(sc->env.exposure), rig);
        break;
    }
    case GR_BANK_RGB_SPECTRAL: y[0] = rgb_to_spectral(R(x[0]), R(x[1]), R(x[2]), R(x[3])); break;
    case GR_BANK_EXP_POLY: y[0] = M<R>::exp_poly(R(x[0])); break;
    case GR_BANK_HG_SAMPLE: put3(sample_hg_direction(R(x[0]), R(x[1]), R(x[2]), v(3)), 0); break;
    case GR_BANK_COSINE_HEMISPHERE: put3(cosine_weighted_hemisphere(R(x[0]), R(x[1]), v(2)), 0); break;
    case GR_BANK_E_FIELD: put3(electric_field_direction(st(0), v(4), v(7)), 0); break;
    case GR_BANK_VON_KRIES: {
        const EnvCtx<R> env = make_env<R>(sc->env);
        put3(apply_von_kries(v(0), env.white_balance), 0);
        break;
    }
    case GR_BANK_WAVELENGTHS: {
        R lam[8];
        wrapped_hero_wavelengths<R>(x[0], lam);
        for (int k = 0; k < 8; ++k) y[k] = lam[k];
        break;
    }
    default: break;
    }
}

const uint32_t kBankArity[GR_BANK_COUNT][2] = {
    {4, 3}, {1, 3}, {1, 1}, {1, 1}, {1, 2}, {12, 1}, {6, 4}, {10, 4}, {5, 4}, {5, 4}, {9, 1}, {3, 1},
    {6, 6}, {8, 3}, {3, 1}, {9, 1}, {4, 1}, {4, 1}, {1, 1}, {6, 3}, {5, 3}, {10, 3}, {3, 3}, {1, 8},
};

}  // namespace

extern "C" {

// Case bank `bank` over n input rows in precision 32 (the reference's f32 arithmetic)
// or 64 (the FP64 oracle); out receives n rows of the bank's outputs as doubles.
int gro_case_bank(uint32_t bank, int precision, const gr_scene *sc, const float *in, uint32_t n, double *out) {
    if (bank >= GR_BANK_COUNT || !in || !out) return GR_EINVAL;
    const uint32_t ni = kBankArity[bank][0], no = kBankArity[bank][1];
    for (uint32_t i = 0; i < n; ++i) {
        if (precision == 64) bank_case<double>(bank, sc, in + (size_t)i * ni, out + (size_t)i * no);
        else bank_case<float>(bank, sc, in + (size_t)i * ni, out + (size_t)i * no);
    }
    return GR_OK;
}

int gro_case_bank_arity(uint32_t bank, uint32_t *n_in, uint32_t *n_out) {
    if (bank >= GR_BANK_COUNT) return GR_EINVAL;
    *n_in = kBankArity[bank][0];
    *n_out = kBankArity[bank][1];
    return GR_OK;
}

// intersect_polyhedron (intersect.rs:93-132) for n rays (origin[3], dir[3] each) in
// precision 32 or 64: t (rounded to f32) and the facet, -1 on a miss.
int gro_intersect_rays(const gr_plane *planes, uint32_t n_planes, const float *rays, uint32_t n, int precision,
                       float *t, int32_t *facet) {
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = rays + 6 * (size_t)i;
        if (precision == 64) {
            Ray<double> ray;
            ray.origin = V3<double>(r[0], r[1], r[2]);
            ray.dir = V3<double>(r[3], r[4], r[5]);
            const Hit<double> h = intersect_polyhedron(ray, planes, n_planes);
            t[i] = h.hit ? (float)h.t : 0.0f;
            facet[i] = h.hit ? h.facet : -1;
        } else {
            Ray<float> ray;
            ray.origin = V3<float>(r[0], r[1], r[2]);
            ray.dir = V3<float>(r[3], r[4], r[5]);
            const Hit<float> h = intersect_polyhedron(ray, planes, n_planes);
            t[i] = h.hit ? h.t : 0.0f;
            facet[i] = h.hit ? h.facet : -1;
        }
    }
    return GR_OK;
}

// evaluate_gem_optical_metrics (color/metrics.rs:1082-1237): out = brilliance %,
// fire index, scintillation %, windowing %, extinction %.
void gro_metrics(const gr_plane *planes, uint32_t n, const gr_material *m, float cam_yaw, float cam_pitch,
                 float light_yaw, float light_pitch, float out[5]) {
    MetricsOut o = evaluate_gem_optical_metrics(planes, n, m, cam_yaw, cam_pitch, light_yaw, light_pitch);
    out[0] = o.brilliance; out[1] = o.fire; out[2] = o.scintillation; out[3] = o.windowing; out[4] = o.extinction;
}

}  // extern "C"
