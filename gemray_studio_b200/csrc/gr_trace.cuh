// gr_trace.cuh -- the per-path transport loop (optics/raytracer/transport.rs:684-940)
// for polished facets of isotropic and uniaxial materials, written as a resumable
// state machine: path_init() builds a path from its (pixel, sample) tuple,
// path_step() advances it by one bounce, path_finish() integrates it to XYZ.  The
// plain kernel runs init/step.../finish per thread; the persistent kernel
// regenerates finished lanes between steps so warps stay full.
#pragma once

#include "gr_device.cuh"

namespace grd {

constexpr int NCH = 8;

struct Path {
    Stokes st[NCH];
    float pdf[NCH];
    float n_o[NCH];
    float ne_d[NCH];  // n_e - n_o per channel
    float a_o[NCH], a_e[NCH];
    V3 o, d, k, prev_plane;
    float hero;
    float rad_scale[NCH];  // radiance multiplier at escape (intensity at escape)
    uint32_t seed, bounce, tuple;
    bool inside, is_e, have_prev, absorbing, alive, escaped;
    V3 escape_dir;
};

// Build the path of tuple (pixel, sample): sampler draws, camera ray, the
// per-sample wavelength cache (refraction.rs:127-174).
__device__ __forceinline__ void path_init(Path &P, const SceneConst &S, const SceneBuffers &B, uint32_t pixel,
                                          uint32_t sample, uint32_t tuple) {
    Draws dr = sample_draws(pixel, sample);
    uint32_t x = pixel % S.width, y = pixel / S.width;
    // camera.rs:95-114
    float aspect = S.width_f / S.height_f;
    float u = (((float)x + dr.jx) / S.width_f - 0.5f) * 2.0f * aspect * S.fov_tan;
    float v = (0.5f - ((float)y + dr.jy) / S.height_f) * 2.0f * S.fov_tan;
    V3 dir = normalize(add(add(ld3(S.cam_f), mul(ld3(S.cam_r), u)), mul(ld3(S.cam_u), v)));
    P.o = ld3(S.cam_o);
    P.d = dir;
    P.k = dir;
    P.prev_plane = v3(0.f, 0.f, 0.f);
    P.hero = dr.hero;
    P.seed = dr.seed;
    P.bounce = 0;
    P.tuple = tuple;
    P.inside = false;
    P.is_e = false;
    P.have_prev = false;
    P.alive = true;
    P.escaped = false;
    bool any = false;
#pragma unroll
    for (int k = 0; k < NCH; ++k) {
        P.st[k] = Stokes{1.0f, 0.0f, 0.0f, 0.0f};
        P.pdf[k] = 1.0f;
        float lam = lambda_k(P.hero, k);
        float n_o = dispersion(S, lam);
        P.n_o[k] = n_o;
        if (S.has_cauchy_e) {
            float lum = lam * 1e-3f;
            float l2 = lum * lum, l4 = l2 * l2;
            float n_e = S.cauchy_e[0] + S.cauchy_e[1] / l2 + S.cauchy_e[2] / l4;
            P.ne_d[k] = n_e - n_o;
        } else {
            P.ne_d[k] = S.bire;
        }
        float ao = 0.0f, ae = 0.0f;
        if (S.absorbing) {
            if (S.ext_n > 0) {
                ao = table_lookup(B.ext_alpha_o, S.ext_n, S.ext_first, S.ext_step, lam);
                ae = table_lookup(B.ext_alpha_e, S.ext_n, S.ext_first, S.ext_step, lam);
            } else {
                ao = band_sum(S.o_bands, S.n_o_bands, lam);
                ae = band_sum(S.e_bands, S.n_e_bands, lam);
            }
        }
        P.a_o[k] = ao;
        P.a_e[k] = ae;
        any = any || (ao != 0.0f) || (ae != 0.0f);
    }
    // Every alpha exactly zero makes the Beer-Lambert factor exp_poly(-0) == 1.0
    // for every channel, so skipping the absorption step is bit-identical.
    P.absorbing = any;
}

// Convex clip against planes staged in shared memory (intersect.rs:93-132,
// simd/slab.rs:101-152).  Returns false on a miss.
__device__ __forceinline__ bool intersect(const float4 *__restrict__ planes, uint32_t n, V3 o, V3 d, float &t_hit,
                                          int &idx_hit) {
    float t_near = -1e30f, t_far = 1e30f;
    int near_idx = -1, far_idx = -1;
    bool outside = false;
    for (uint32_t i = 0; i < n; ++i) {
        float4 p = planes[i];
        float denom = (p.x * d.x + p.y * d.y) + p.z * d.z;
        float side = p.w + ((p.x * o.x + p.y * o.y) + p.z * o.z);
        if (fabsf(denom) > 1e-7f) {
            float t = (-side) / denom;
            if (denom < 0.0f) {
                if (t > t_near) { t_near = t; near_idx = (int)i; }
            } else if (t < t_far) {
                t_far = t; far_idx = (int)i;
            }
        } else if (side > 0.0f) {
            outside = true;
            break;
        }
    }
    if (outside || t_near > t_far) return false;
    if (t_near > 1e-4f) {
        t_hit = t_near;
        idx_hit = near_idx;
        return true;
    }
    if (t_far > 1e-4f) {
        t_hit = t_far;
        idx_hit = far_idx;
        return true;
    }
    return false;
}

__device__ __forceinline__ V3 plane_normal(const float4 *planes, int idx) {
    if (idx < 0) return v3(0.f, 0.f, 0.f);
    float4 p = planes[idx];
    return v3(p.x, p.y, p.z);
}

// intersect.rs:196-229 (edge rounding; identity when radius <= 0)
__device__ __forceinline__ V3 shading_normal(const float4 *planes, uint32_t n, V3 hp, int hit_idx, V3 hn, float radius) {
    if (radius <= 0.0f) return hn;
    float nearest = __int_as_float(0x7f800000);
    V3 nn = hn;
    for (uint32_t i = 0; i < n; ++i) {
        if ((int)i == hit_idx) continue;
        float4 p = planes[i];
        V3 pn = v3(p.x, p.y, p.z);
        float dist = -(p.w + dot(pn, hp));
        if (dist < nearest) { nearest = dist; nn = pn; }
    }
    if (nearest >= radius) return hn;
    float t = clampf(1.0f - nearest / radius, 0.0f, 1.0f);
    float smooth_t = t * t * fmaf(2.0f, -t, 3.0f);
    V3 bis = normalize_or_zero(add(hn, nn));
    return normalize_or_zero(add(mul(hn, 1.0f - smooth_t), mul(bis, smooth_t)));
}

// Per-thread event tallies for the instrumented kernel variant (the FLOP model's
// inputs, cf. trace_spectral_ray_with_finish_instrumented, transport.rs:512-537).
enum CounterIndex {
    C_PATHS = 0, C_BOUNCES, C_ESCAPES, C_TIR, C_REFLECT, C_REFRACT, C_ABSORB, C_CH_TIR, C_CH_REFR, C_ROULETTE,
    C_ROTATIONS, C_ANISO_BOUNCES, C_WALKOFF, C_ROULETTE_KILLS, C_COUNT
};
struct Counters {
    uint32_t c[C_COUNT];
};
struct NoCounters {};
template <class CT> __device__ __forceinline__ void tally(CT &, int, uint32_t = 1) {}
template <> __device__ __forceinline__ void tally<Counters>(Counters &ct, int i, uint32_t v) { ct.c[i] += v; }

// One bounce of transport.rs:781-929.  Marks the path dead on escape, Russian
// roulette or the bounce cap.
template <class CT = NoCounters>
__device__ __forceinline__ void path_step(Path &P, const SceneConst &S, const float4 *__restrict__ planes, CT &ct) {
    const uint32_t bounce = P.bounce;
    float t_hit = 0.0f;
    int fidx = 0;
    tally(ct, C_BOUNCES);
    if (!intersect(planes, S.n_planes, P.o, P.d, t_hit, fidx)) {
        tally(ct, C_ESCAPES);
        // accumulate_miss_radiance (transport.rs:67-90): radiance_k = I_k * L_k
        P.escaped = true;
        P.escape_dir = P.d;
#pragma unroll
        for (int k = 0; k < NCH; ++k) P.rad_scale[k] = intensity(P.st[k]);
        P.alive = false;
        return;
    }
    V3 hp = add(P.o, smul(t_hit, P.d));
    V3 normal = shading_normal(planes, S.n_planes, hp, fidx, plane_normal(planes, fidx), S.edge_radius);
    const V3 kk = P.k;

    // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:71-89)
    V3 cur_plane = normalize_or_zero(cross(kk, normal));
    if (P.have_prev && dot(cur_plane, cur_plane) > 1e-6f && dot(P.prev_plane, P.prev_plane) > 1e-6f) {
        float cos_psi = clampf(dot(P.prev_plane, cur_plane), -1.0f, 1.0f);
        float sin_psi = dot(cross(P.prev_plane, cur_plane), normalize_or_zero(kk));
        float psi = atan2f(sin_psi, cos_psi);
        float s2, c2;
        sincosf(2.0f * psi, &s2, &c2);
#pragma unroll
        for (int k = 0; k < NCH; ++k) P.st[k] = apply_rotation(P.st[k], c2, s2);
        tally(ct, C_ROTATIONS);
    }
    P.prev_plane = cur_plane;
    P.have_prev = true;

    // apply_interior_segment (transport.rs:586-605) -> apply_absorption (absorption.rs:115-141)
    if (P.inside) {
        normal = neg(normal);
        if (P.absorbing) {
            tally(ct, C_ABSORB);
            V3 c_axis = ld3(S.c_axis);
            V3 ea = ordinary_eigen(kk, c_axis);
            V3 eb = extraordinary_eigen_from(kk, ea);
            float scaled = t_hit * S.path_scale;
            float alpha[NCH];
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                V3 e_hat = electric_field_direction(P.st[k], cur_plane, kk);
                float p = clampf(dop(P.st[k]), 0.0f, 1.0f);
                float a_pol = quad_form(S, P.a_o[k], P.a_e[k], e_hat);
                float a_unp = midpoint(quad_form(S, P.a_o[k], P.a_e[k], ea), quad_form(S, P.a_o[k], P.a_e[k], eb));
                alpha[k] = fmaf(p, a_pol - a_unp, a_unp);
            }
#pragma unroll
            for (int k = 0; k < NCH; ++k) P.st[k] = scale(P.st[k], exp_poly(-alpha[k] * scaled));
        }
    }

    // compute_bounce_refraction_geometry (refraction.rs:428-547), uniaxial branch
    const bool inside = P.inside;
    const bool aniso = S.anisotropic != 0;
    float cos_i = clampf(dot(neg(kk), normal), 0.0f, 1.0f);
    float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    float sin_i = sqrtf(fmaxf(one_m_c2, 0.0f));
    float n_o_hero = P.n_o[0];
    float n_e_hero = n_o_hero + P.ne_d[0];
    float n_med[NCH];
    if (aniso) {
        tally(ct, C_ANISO_BOUNCES);
        V3 c_axis = ld3(S.c_axis);
        float theta;
        if (!inside) {
            // theta_c_for_bounce entry fixed point (refraction.rs:248-269)
            float n_guess = n_o_hero;
            theta = 0.0f;
#pragma unroll
            for (int it = 0; it < 2; ++it) {
                float eta = 1.0f / n_guess;
                float s2 = eta * eta * one_m_c2;
                if (s2 > 1.0f) break;
                float ct = sqrtf(fmaxf(1.0f - s2, 0.0f));
                V3 wd = normalize(add(smul(eta, kk), smul(fmaf(eta, cos_i, -ct), normal)));
                theta = acosf(fabsf(clampf(dot(wd, c_axis), -1.0f, 1.0f)));
                float sth, cth;
                sincosf(theta, &sth, &cth);
                n_guess = eff_e_index(n_o_hero, n_e_hero, sth, cth);
            }
        } else {
            theta = acosf(fabsf(clampf(dot(kk, c_axis), -1.0f, 1.0f)));
        }
        float sth, cth;
        sincosf(theta, &sth, &cth);
        const bool use_o = inside && !P.is_e;
#pragma unroll
        for (int k = 0; k < NCH; ++k)
            n_med[k] = use_o ? P.n_o[k] : eff_e_index(P.n_o[k], P.n_o[k] + P.ne_d[k], sth, cth);
    } else {
#pragma unroll
        for (int k = 0; k < NCH; ++k) n_med[k] = P.n_o[k];
    }
    const float n1 = inside ? n_med[0] : 1.0f;
    const float n2 = inside ? 1.0f : n_med[0];
    float eta0 = n1 / n2;
    const float sin2_t = eta0 * eta0 * one_m_c2;

    V3 new_k, new_s;
    bool new_inside = inside;
    bool has_update = false, update_val = false;
    if (sin2_t > 1.0f) {
        // apply_tir_bounce (refraction.rs:599-637)
        tally(ct, C_TIR);
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            float n1k = inside ? n_med[k] : 1.0f, n2k = inside ? 1.0f : n_med[k];
            float etak = n1k / n2k;
            float s2k = etak * etak * one_m_c2;
            if (s2k > 1.0f) {
                tally(ct, C_CH_TIR);
                float dk = tir_phase_delta(n1k, cos_i, sin_i);
                float sd, cd;
                sincosf(dk, &sd, &cd);
                P.st[k] = apply_tir(P.st[k], cd, sd);
            } else {
                float ct = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                float rs, rp, a, b, c;
                fresnel_rs_rp(n1k, n2k, cos_i, ct, rs, rp);
                fresnel_reflection_abc(rs, rp, a, b, c);
                P.st[k] = apply_fresnel(P.st[k], a, b, c);
                P.pdf[k] = P.pdf[k] * r_unpol(rs, rp);
            }
        }
        new_k = sub(kk, smul(2.0f * dot(kk, normal), normal));
        new_s = (inside && aniso && P.is_e) ? extraordinary_poynting_dir(new_k, ld3(S.c_axis), n_o_hero, n_e_hero)
                                            : new_k;
    } else {
        // apply_partial_fresnel_bounce (refraction.rs:1036-1086)
        float cos_t = sqrtf(1.0f - sin2_t);
        float rs, rp;
        fresnel_rs_rp(n1, n2, cos_i, cos_t, rs, rp);
        const float ru = r_unpol(rs, rp);
        float rng_b = rng_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
        if (rng_b < ru) {
            // apply_partial_reflect_bounce (refraction.rs:650-690)
            tally(ct, C_REFLECT);
            const float inv = 1.0f / ru;
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                float n1k = inside ? n_med[k] : 1.0f, n2k = inside ? 1.0f : n_med[k];
                float etak = n1k / n2k;
                float s2k = etak * etak * one_m_c2;
                if (s2k > 1.0f) {
                    tally(ct, C_CH_TIR);
                    float dk = tir_phase_delta(n1k, cos_i, sin_i);
                    float sd, cd;
                    sincosf(dk, &sd, &cd);
                    P.st[k] = scale(apply_tir(P.st[k], cd, sd), inv);
                } else {
                    float ct = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                    float rsk, rpk, a, b, c;
                    fresnel_rs_rp(n1k, n2k, cos_i, ct, rsk, rpk);
                    P.pdf[k] = P.pdf[k] * r_unpol(rsk, rpk);
                    fresnel_reflection_abc(rsk, rpk, a, b, c);
                    P.st[k] = scale(apply_fresnel(P.st[k], a, b, c), inv);
                }
            }
            new_k = sub(kk, smul(2.0f * dot(kk, normal), normal));
            new_s = (inside && aniso && P.is_e)
                        ? extraordinary_poynting_dir(new_k, ld3(S.c_axis), n_o_hero, n_e_hero)
                        : new_k;
        } else {
            // apply_refract_bounce (refraction.rs:748-867)
            tally(ct, C_REFRACT);
            const bool entering_aniso = !inside && aniso;
            bool use_e = P.is_e;
            if (entering_aniso) use_e = rng_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f;
            const bool ordinary_entry = entering_aniso && !use_e;
            const bool extra_entry = entering_aniso && use_e;
            float n2_dir = ordinary_entry ? n_o_hero : n2;
            float eta_dir = n1 / n2_dir;
            float s2d = fminf(eta_dir * eta_dir * one_m_c2, 1.0f);
            float ctd = sqrtf(fmaxf(1.0f - s2d, 0.0f));
            V3 refr = normalize(add(smul(eta_dir, kk), smul(fmaf(eta_dir, cos_i, -ctd), normal)));
            V3 c_axis = ld3(S.c_axis);
            V3 final_dir = extra_entry ? extraordinary_poynting_dir(refr, c_axis, n_o_hero, n_e_hero) : refr;
            if (extra_entry) tally(ct, C_WALKOFF, 9);
            const float tinv = 1.0f / (1.0f - ru);
            const float TOL = 1.0f - 1e-6f;
            // apply_refract_channel (refraction.rs:883-1011)
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                float n1k = inside ? n_med[k] : 1.0f;
                float n2k = ordinary_entry ? P.n_o[k] : (inside ? 1.0f : n_med[k]);
                float ratio = n1k / n2k;
                float s2k = (ratio * ratio) * one_m_c2;
                if (s2k > 1.0f) {
                    P.st[k] = scale(P.st[k], 0.0f);
                    P.pdf[k] = 0.0f;
                    continue;
                }
                tally(ct, C_CH_REFR);
                float ctk = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                V3 rk = normalize(add(smul(ratio, kk), smul(fmaf(ratio, cos_i, -ctk), normal)));
                V3 fk = extra_entry ? extraordinary_poynting_dir(rk, c_axis, P.n_o[k], P.n_o[k] + P.ne_d[k]) : rk;
                if (dot(fk, final_dir) >= TOL) {
                    float ts = (2.0f * n1k * cos_i) / fmaf(n2k, ctk, n1k * cos_i);
                    float tp = (2.0f * n1k * cos_i) / fmaf(n1k, ctk, n2k * cos_i);
                    float a, b, c;
                    fresnel_transmission_abc(n1k, n2k, cos_i, ctk, ts, tp, a, b, c);
                    P.st[k] = scale(apply_fresnel(P.st[k], a, b, c), tinv);
                    float rsk, rpk;
                    fresnel_rs_rp(n1k, n2k, cos_i, ctk, rsk, rpk);
                    P.pdf[k] = P.pdf[k] * (1.0f - r_unpol(rsk, rpk));
                } else {
                    P.st[k] = scale(P.st[k], 0.0f);
                    P.pdf[k] = 0.0f;
                }
            }
            new_k = refr;
            new_s = final_dir;
            new_inside = !inside;
            if (entering_aniso) {
                has_update = true;
                update_val = use_e;
            }
        }
    }
    const bool was_internal_reflection = inside && !has_update && new_inside == inside;
    P.d = new_s;
    P.o = add(hp, mul(new_s, 1e-4f));
    P.k = new_k;
    P.inside = new_inside;
    if (has_update) P.is_e = update_val;
    // maybe_apply_internal_mode_coupling (transport.rs:343-353)
    if (aniso && was_internal_reflection) P.is_e = rng_draw(P.seed, bounce, MODE_COUPLING_STREAM) < 0.5f;

    // apply_russian_roulette (transport.rs:204-220)
    if (bounce > 4) {
        tally(ct, C_ROULETTE);
        float mx = 0.0f;
#pragma unroll
        for (int k = 0; k < NCH; ++k) mx = fmaxf(mx, intensity(P.st[k]));
        float q = clampf(mx, 0.05f, 1.0f);
        float rr = rng_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM);
        if (rr > q) {
            tally(ct, C_ROULETTE_KILLS);
            P.alive = false;
            return;
        }
        const float iq = 1.0f / q;
#pragma unroll
        for (int k = 0; k < NCH; ++k) P.st[k] = scale(P.st[k], iq);
    }
    P.bounce = bounce + 1;
    if (P.bounce >= S.max_bounces) P.alive = false;
}

// Escape radiance, spectral MIS and CIE integration (transport.rs:67-90,931-939,
// raytracer/color.rs:122-164) for a finished path.
__device__ __forceinline__ V3 path_finish(const Path &P, const SceneConst &S, const SceneBuffers &B) {
    float rad[NCH];
    if (P.escaped) {
        if (S.env_mode == GR_ENV_STUDIO) {
            V3 dn = normalize(P.escape_dir);
#pragma unroll
            for (int k = 0; k < NCH; ++k) rad[k] = fmaf(P.rad_scale[k], studio_radiance(S, dn, lambda_k(P.hero, k)), 0.0f);
        } else {
            float rgb[3];
            if (S.env_mode == GR_ENV_UNIFORM) {
                rgb[0] = S.uni_rgb[0]; rgb[1] = S.uni_rgb[1]; rgb[2] = S.uni_rgb[2];
            } else {
                latlong_rgb(S, B.map, P.escape_dir, rgb);
            }
#pragma unroll
            for (int k = 0; k < NCH; ++k)
                rad[k] = fmaf(P.rad_scale[k], rgb_to_spectral(rgb[0], rgb[1], rgb[2], lambda_k(P.hero, k)), 0.0f);
        }
    } else {
#pragma unroll
        for (int k = 0; k < NCH; ++k) rad[k] = 0.0f;
    }
    float sum = -0.0f;
#pragma unroll
    for (int k = 0; k < NCH; ++k) sum = sum + P.pdf[k];
    float w = sum <= 1e-12f ? 1.0f : 8.0f * P.pdf[0] / sum;
    const float norm = (400.0f / 8.0f) / 106.856f;
    V3 xyz = v3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < NCH; ++k) {
        float wr = rad[k] * w;
        xyz = add(xyz, mul(cmf(lambda_k(P.hero, k)), wr * norm));
    }
    return von_kries(xyz, S.wb);
}

}  // namespace grd
