// gr_scene_builders.cpp -- host-only scene helpers exported through the C ABI:
// the pinhole camera (optics/raytracer/camera.rs:62-93), the standard round brilliant
// (geometry/cuts.rs:45-129, GpuFacetPlane::new at geometry/plane.rs:12-19) and the 13
// built-in materials (optics/materials.rs:136-1250) encoded as GpuGemMaterial
// (renderer/buffers.rs:313-385).  Compiled without FMA contraction, f32 libm.
#include <cmath>
#include <cstring>

#include "gemray_cuda.h"

namespace {

struct F3 {
    float x, y, z;
};
inline float fdot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline F3 fscale(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
inline F3 fnormalize(F3 a) { return fscale(a, 1.0f / sqrtf(fdot(a, a))); }
inline F3 fcross(F3 a, F3 b) { return F3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }

inline float deg2rad(float d) { return d * (3.14159265358979323846f / 180.0f); }

inline gr_plane plane_of(F3 n, float d) {
    F3 u = fnormalize(n);
    gr_plane p;
    p.normal[0] = u.x;
    p.normal[1] = u.y;
    p.normal[2] = u.z;
    p.d = d;
    return p;
}

struct Band {
    float c, w, p;
};

enum Abs { ABS_ISOTROPIC, ABS_UNIAXIAL, ABS_BIAXIAL };

struct Spec {
    const char *name;
    uint32_t crystal, optical, model;
    float a[3], b[3];
    float bire;
    Abs abs;
    int no, ne, nb;
    Band o[3], e[3], beta[3];
    float c_axis[3];
    int has_biax;
    float biax;
};

// legacy_rgb_bands (optics/absorption.rs): lobes at 620/540/450 nm.
#define RGB3(r, g, b) {{620.f, 55.f, r}, {540.f, 45.f, g}, {450.f, 45.f, b}}

const Spec kSpecs[] = {
    {"Diamond", 0, 0, GR_DISP_SELLMEIER3, {4.3356f, 0.3306f, 0.0f}, {0.011236f, 0.030625f, 1.0f}, 0.0f, ABS_ISOTROPIC, 0, 0, 0,
     {}, {}, {}, {0, 1, 0}, 0, 0},
    {"Sapphire", 3, 2, GR_DISP_SELLMEIER3, {1.431349f, 0.650547f, 5.341402f}, {0.00528f, 0.01424f, 325.015f}, -0.0081f,
     ABS_UNIAXIAL, 1, 1, 0, {{580.f, 90.f, 3.0f}}, {{700.f, 95.f, 2.1f}}, {}, {0, 1, 0}, 0, 0},
    {"Ruby", 3, 2, GR_DISP_SELLMEIER3, {1.431349f, 0.650547f, 5.341402f}, {0.00528f, 0.01424f, 325.015f}, -0.0081f,
     ABS_UNIAXIAL, 2, 2, 0, {{410.f, 30.f, 3.0f}, {556.f, 45.f, 2.5f}}, {{400.f, 30.f, 2.9f}, {550.f, 45.f, 1.4f}}, {},
     {0, 1, 0}, 0, 0},
    {"Emerald", 2, 2, GR_DISP_CAUCHY, {1.566794f, 0.004273f, 0.0f}, {0, 0, 0}, -0.0060f, ABS_ISOTROPIC, 2, 0, 0,
     {{430.f, 30.f, 2.8f}, {600.f, 40.f, 2.6f}}, {}, {}, {0, 1, 0}, 0, 0},
    {"Zircon", 1, 1, GR_DISP_CAUCHY, {1.890963f, 0.011820f, 0.0f}, {0, 0, 0}, 0.0590f, ABS_ISOTROPIC, 3, 0, 0,
     RGB3(0.2f, 0.6f, 1.8f), {}, {}, {0, 1, 0}, 0, 0},
    {"Alexandrite", 4, 3, GR_DISP_SELLMEIER3, {0.78522f, 1.21202f, 16.81f}, {0.0f, 0.01262f, 1000.0f}, 0.0076f, ABS_BIAXIAL,
     2, 2, 2, {{565.f, 40.f, 1.9f}, {420.f, 32.f, 1.8f}}, {{595.f, 40.f, 3.1f}, {430.f, 32.f, 1.5f}},
     {{560.f, 40.f, 0.65f}, {422.f, 32.f, 3.5f}}, {0, 1, 0}, 1, 0.001951f},
    {"Topaz", 4, 3, GR_DISP_CAUCHY, {1.614872f, 0.004273f, 0.0f}, {0, 0, 0}, 0.0080f, ABS_ISOTROPIC, 3, 0, 0,
     RGB3(1.2f, 0.4f, 0.1f), {}, {}, {0, 1, 0}, 1, 0.0024f},
    {"Spinel", 0, 0, GR_DISP_SELLMEIER3, {1.8938f, 3.0755f, 0.0f}, {0.009884f, 250.462f, 1.0f}, 0.0f, ABS_ISOTROPIC, 3, 0, 0,
     RGB3(0.4f, 2.2f, 1.6f), {}, {}, {0, 1, 0}, 0, 0},
    {"Quartz", 3, 1, GR_DISP_SELLMEIER3, {0.2860414f, 1.0704408f, 1.1020224f}, {0.0f, 0.0100586f, 100.0f}, 0.0091f,
     ABS_ISOTROPIC, 3, 0, 0, RGB3(0.8f, 1.8f, 0.6f), {}, {}, {0, 1, 0}, 0, 0},
    {"Tourmaline", 3, 2, GR_DISP_CAUCHY, {1.624481f, 0.005183f, 0.0f}, {0, 0, 0}, -0.0210f, ABS_UNIAXIAL, 2, 2, 0,
     {{720.f, 55.f, 3.0f}, {430.f, 45.f, 1.8f}}, {{720.f, 55.f, 1.0f}, {430.f, 45.f, 0.6f}}, {}, {1, 0, 0}, 0, 0},
    {"Tanzanite", 4, 3, GR_DISP_CAUCHY, {1.674589f, 0.009123f, 0.0f}, {0, 0, 0}, 0.0130f, ABS_BIAXIAL, 2, 3, 2,
     {{595.f, 45.f, 1.3f}, {528.f, 35.f, 1.8f}}, {{595.f, 45.f, 1.6f}, {528.f, 35.f, 1.0f}, {455.f, 40.f, 2.6f}},
     {{595.f, 45.f, 3.2f}, {528.f, 35.f, 2.8f}}, {0, 1, 0}, 1, 0.0070f},
    {"Synthetic Moissanite", 2, 1, GR_DISP_SELLMEIER3, {1.163887f, 4.408433f, 21.53f}, {0.0f, 0.03178f, 1000.0f}, 0.0415f,
     ABS_ISOTROPIC, 0, 0, 0, {}, {}, {}, {0, 1, 0}, 0, 0},
    {"Cubic Zirconia", 0, 0, GR_DISP_SELLMEIER3, {1.347091f, 2.117788f, 9.452943f}, {0.003912f, 0.027802f, 591.489f}, 0.0f,
     ABS_ISOTROPIC, 0, 0, 0, {}, {}, {}, {0, 1, 0}, 0, 0},
};

void put_bands(gr_band *dst, uint32_t *count, const Band *src, int n) {
    for (uint32_t i = 0; i < GR_MAX_BANDS; ++i) {
        dst[i].center_nm = 0.0f;
        dst[i].width_nm = 1.0f;
        dst[i].peak = 0.0f;
    }
    for (int i = 0; i < n; ++i) {
        dst[i].center_nm = src[i].c;
        dst[i].width_nm = src[i].w;
        dst[i].peak = src[i].p;
    }
    *count = (uint32_t)n;
}

}  // namespace

extern "C" {

gr_status gr_camera_new(float yaw, float pitch, float distance, float fov_deg, gr_camera *out) {
    if (!out) return GR_EINVAL;
    float cos_p = cosf(pitch), sin_p = sinf(pitch), cos_y = cosf(yaw), sin_y = sinf(yaw);
    F3 origin{distance * cos_p * sin_y, distance * sin_p, distance * cos_p * cos_y};
    F3 forward = fnormalize(F3{-origin.x, -origin.y, -origin.z});
    F3 world_up = fabsf(cos_p) < 1e-4f ? F3{0.f, 0.f, -1.f} : F3{0.f, 1.f, 0.f};
    F3 right = fnormalize(fcross(forward, world_up));
    F3 up = fnormalize(fcross(right, forward));
    out->origin[0] = origin.x; out->origin[1] = origin.y; out->origin[2] = origin.z;
    out->forward[0] = forward.x; out->forward[1] = forward.y; out->forward[2] = forward.z;
    out->right[0] = right.x; out->right[1] = right.y; out->right[2] = right.z;
    out->up[0] = up.x; out->up[1] = up.y; out->up[2] = up.z;
    out->fov_tan = tanf(deg2rad(fov_deg) * 0.5f);
    return GR_OK;
}

uint32_t gr_standard_round_brilliant(gr_plane *out, uint32_t cap) {
    gr_plane planes[74];
    uint32_t n = 0;
    const float gear = 96.0f;
    const float PI = 3.14159265358979323846f;
    planes[n++] = plane_of(F3{0.f, 1.f, 0.f}, -0.32f);
    auto ring = [&](float deg, const float *idx, int cnt, float d, float ysign) {
        float a = deg2rad(deg);
        for (int i = 0; i < cnt; ++i) {
            float phi = 2.0f * PI * idx[i] / gear;
            planes[n++] = plane_of(F3{sinf(a) * cosf(phi), ysign > 0 ? cosf(a) : -cosf(a), sinf(a) * sinf(phi)}, d);
        }
    };
    const float stars[8] = {6, 18, 30, 42, 54, 66, 78, 90};
    const float mains[8] = {0, 12, 24, 36, 48, 60, 72, 84};
    const float halves[16] = {95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85};
    ring(15.0f, stars, 8, -0.45f, 1.f);
    ring(34.5f, mains, 8, -0.59f, 1.f);
    ring(41.0f, halves, 16, -0.67f, 1.f);
    for (int i = 0; i < 16; ++i) {
        float phi = 2.0f * PI * (float)i / 16.0f;
        planes[n++] = plane_of(F3{cosf(phi), 0.f, sinf(phi)}, -1.0f);
    }
    ring(41.0f, mains, 8, -0.67f, -1.f);
    ring(42.5f, halves, 16, -0.68f, -1.f);
    planes[n++] = plane_of(F3{0.f, -1.f, 0.f}, -0.88f);
    if (out)
        for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = planes[i];
    return n;
}

gr_status gr_builtin_material(const char *name, gr_material *out) {
    if (!name || !out) return GR_EINVAL;
    for (const Spec &s : kSpecs) {
        if (strcmp(s.name, name) != 0) continue;
        gr_material m;
        memset(&m, 0, sizeof(m));
        m.dispersion.model_type = s.model;
        if (s.model == GR_DISP_CAUCHY) {
            for (int i = 0; i < 3; ++i) m.dispersion.param_a[i] = s.a[i];
        } else {
            for (int i = 0; i < 3; ++i) {
                m.dispersion.param_a[i] = s.a[i];
                m.dispersion.param_b[i] = s.b[i];
            }
        }
        for (int i = 0; i < 3; ++i) m.dispersion.c_axis_and_birefringence[i] = s.c_axis[i];
        m.dispersion.c_axis_and_birefringence[3] = s.bire;
        m.dispersion.is_anisotropic = (s.crystal != GR_CRYSTAL_CUBIC && fabsf(s.bire) > 1e-4f) ? 1u : 0u;
        m.dispersion.biaxial_delta_beta_alpha = s.has_biax ? s.biax : 0.0f;
        m.dispersion.has_biaxial_delta = s.has_biax ? 1u : 0u;
        m.crystal_system = s.crystal;
        m.optical_character = s.optical;
        m.is_pleochroic = s.abs == ABS_ISOTROPIC ? 0u : 1u;
        if (s.abs == ABS_ISOTROPIC) {
            put_bands(m.o_ray_bands, &m.o_ray_band_count, s.o, s.no);
            put_bands(m.e_ray_bands, &m.e_ray_band_count, s.o, s.no);
            put_bands(m.beta_ray_bands, &m.beta_ray_band_count, s.beta, 0);
        } else {
            put_bands(m.o_ray_bands, &m.o_ray_band_count, s.o, s.no);
            put_bands(m.e_ray_bands, &m.e_ray_band_count, s.e, s.ne);
            put_bands(m.beta_ray_bands, &m.beta_ray_band_count, s.beta, s.abs == ABS_BIAXIAL ? s.nb : 0);
            m.has_beta_ray = s.abs == ABS_BIAXIAL ? 1u : 0u;
        }
        m.absorption_path_scale = 1.0f;
        *out = m;
        return GR_OK;
    }
    return GR_ENOTFOUND;
}

}  // extern "C"
