// gro_scene.hpp -- oracle restatement of the reference's scene inputs.
//
// TEST INFRASTRUCTURE ONLY (see gr_oracle.hpp).  Restates
//   * StandardGemCuts::standard_round_brilliant (crates/gemray/src/geometry/cuts.rs:45-129),
//   * GpuFacetPlane::new (geometry/plane.rs:12-19),
//   * the 13 built-in materials (optics/materials.rs:136-1250) encoded as
//     GpuGemMaterial (renderer/buffers.rs:313-420),
// so the golden pins of the oracle do not depend on the product's own scene builders
// (which the tests compare against these).
#pragma once

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "gr_oracle.hpp"

namespace gro {

// plane.rs:12-19
static inline gr_plane make_plane(V3<float> n, float d) {
    V3<float> u = n.normalize();
    gr_plane p;
    p.normal[0] = u.x; p.normal[1] = u.y; p.normal[2] = u.z;
    p.d = d;
    return p;
}

static inline float to_radians(float deg) { return deg * (3.14159265358979323846f / 180.0f); }

// cuts.rs:45-129 -- 74 planes.
static inline std::vector<gr_plane> standard_round_brilliant() {
    std::vector<gr_plane> planes;
    const float gear = 96.0f;
    const float PI = 3.14159265358979323846f;
    planes.push_back(make_plane(V3<float>(0.f, 1.f, 0.f), -0.32f));
    auto ring = [&](float angle_deg, const std::vector<float> &idx, float d, bool crown) {
        float a = to_radians(angle_deg);
        for (float g : idx) {
            float phi = 2.0f * PI * g / gear;
            V3<float> n(::sinf(a) * ::cosf(phi), crown ? ::cosf(a) : -::cosf(a), ::sinf(a) * ::sinf(phi));
            planes.push_back(make_plane(n, d));
        }
    };
    ring(15.0f, {6, 18, 30, 42, 54, 66, 78, 90}, -0.45f, true);
    ring(34.5f, {0, 12, 24, 36, 48, 60, 72, 84}, -0.59f, true);
    ring(41.0f, {95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85}, -0.67f, true);
    for (int i = 0; i < 16; ++i) {
        float phi = 2.0f * PI * (float)i / 16.0f;
        planes.push_back(make_plane(V3<float>(::cosf(phi), 0.f, ::sinf(phi)), -1.0f));
    }
    ring(41.0f, {0, 12, 24, 36, 48, 60, 72, 84}, -0.67f, false);
    ring(42.5f, {95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85}, -0.68f, false);
    planes.push_back(make_plane(V3<float>(0.f, -1.f, 0.f), -0.88f));
    return planes;
}

struct BandSpec { float c, w, p; };

static inline void set_bands(gr_band *dst, uint32_t &count, const std::vector<BandSpec> &src) {
    for (uint32_t i = 0; i < GR_MAX_BANDS; ++i) { dst[i].center_nm = 0.f; dst[i].width_nm = 1.f; dst[i].peak = 0.f; }
    count = (uint32_t)src.size();
    for (size_t i = 0; i < src.size(); ++i) { dst[i].center_nm = src[i].c; dst[i].width_nm = src[i].w; dst[i].peak = src[i].p; }
}

static inline std::vector<BandSpec> legacy_rgb(float r, float g, float b) {  // absorption.rs legacy_rgb_bands
    return {{620.f, 55.f, r}, {540.f, 45.f, g}, {450.f, 45.f, b}};
}

enum { CUBIC = 0, TETRAGONAL = 1, HEXAGONAL = 2, TRIGONAL = 3, ORTHORHOMBIC = 4 };
enum { ISO = 0, UNI_POS = 1, UNI_NEG = 2, BI_POS = 3, BI_NEG = 4 };
enum { ABS_ISO = 0, ABS_UNI = 1, ABS_BI = 2 };

struct MatSpec {
    const char *name;
    uint32_t crystal, optical;
    uint32_t disp;
    float a[3], b[3];
    float bire;
    int abs_kind;
    std::vector<BandSpec> o, e, beta;
    float cx, cy, cz;
    bool has_biax;
    float biax;
};

static inline std::vector<MatSpec> material_specs() {
    std::vector<MatSpec> v;
    v.push_back({"Diamond", CUBIC, ISO, GR_DISP_SELLMEIER3, {4.3356f, 0.3306f, 0.0f}, {0.011236f, 0.030625f, 1.0f},
                 0.0f, ABS_ISO, {}, {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Sapphire", TRIGONAL, UNI_NEG, GR_DISP_SELLMEIER3, {1.431349f, 0.650547f, 5.341402f},
                 {0.00528f, 0.01424f, 325.015f}, -0.0081f, ABS_UNI, {{580.f, 90.f, 3.0f}}, {{700.f, 95.f, 2.1f}}, {},
                 0, 1, 0, false, 0});
    v.push_back({"Ruby", TRIGONAL, UNI_NEG, GR_DISP_SELLMEIER3, {1.431349f, 0.650547f, 5.341402f},
                 {0.00528f, 0.01424f, 325.015f}, -0.0081f, ABS_UNI, {{410.f, 30.f, 3.0f}, {556.f, 45.f, 2.5f}},
                 {{400.f, 30.f, 2.9f}, {550.f, 45.f, 1.4f}}, {}, 0, 1, 0, false, 0});
    v.push_back({"Emerald", HEXAGONAL, UNI_NEG, GR_DISP_CAUCHY, {1.566794f, 0.004273f, 0.0f}, {0, 0, 0}, -0.0060f,
                 ABS_ISO, {{430.f, 30.f, 2.8f}, {600.f, 40.f, 2.6f}}, {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Zircon", TETRAGONAL, UNI_POS, GR_DISP_CAUCHY, {1.890963f, 0.011820f, 0.0f}, {0, 0, 0}, 0.0590f,
                 ABS_ISO, legacy_rgb(0.2f, 0.6f, 1.8f), {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Alexandrite", ORTHORHOMBIC, BI_POS, GR_DISP_SELLMEIER3, {0.78522f, 1.21202f, 16.81f},
                 {0.0f, 0.01262f, 1000.0f}, 0.0076f, ABS_BI, {{565.f, 40.f, 1.9f}, {420.f, 32.f, 1.8f}},
                 {{595.f, 40.f, 3.1f}, {430.f, 32.f, 1.5f}}, {{560.f, 40.f, 0.65f}, {422.f, 32.f, 3.5f}}, 0, 1, 0,
                 true, 0.001951f});
    v.push_back({"Topaz", ORTHORHOMBIC, BI_POS, GR_DISP_CAUCHY, {1.614872f, 0.004273f, 0.0f}, {0, 0, 0}, 0.0080f,
                 ABS_ISO, legacy_rgb(1.2f, 0.4f, 0.1f), {}, {}, 0, 1, 0, true, 0.0024f});
    v.push_back({"Spinel", CUBIC, ISO, GR_DISP_SELLMEIER3, {1.8938f, 3.0755f, 0.0f}, {0.009884f, 250.462f, 1.0f}, 0.0f,
                 ABS_ISO, legacy_rgb(0.4f, 2.2f, 1.6f), {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Quartz", TRIGONAL, UNI_POS, GR_DISP_SELLMEIER3, {0.2860414f, 1.0704408f, 1.1020224f},
                 {0.0f, 0.0100586f, 100.0f}, 0.0091f, ABS_ISO, legacy_rgb(0.8f, 1.8f, 0.6f), {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Tourmaline", TRIGONAL, UNI_NEG, GR_DISP_CAUCHY, {1.624481f, 0.005183f, 0.0f}, {0, 0, 0}, -0.0210f,
                 ABS_UNI, {{720.f, 55.f, 3.0f}, {430.f, 45.f, 1.8f}}, {{720.f, 55.f, 1.0f}, {430.f, 45.f, 0.6f}}, {},
                 1, 0, 0, false, 0});
    v.push_back({"Tanzanite", ORTHORHOMBIC, BI_POS, GR_DISP_CAUCHY, {1.674589f, 0.009123f, 0.0f}, {0, 0, 0}, 0.0130f,
                 ABS_BI, {{595.f, 45.f, 1.3f}, {528.f, 35.f, 1.8f}},
                 {{595.f, 45.f, 1.6f}, {528.f, 35.f, 1.0f}, {455.f, 40.f, 2.6f}},
                 {{595.f, 45.f, 3.2f}, {528.f, 35.f, 2.8f}}, 0, 1, 0, true, 0.0070f});
    v.push_back({"Synthetic Moissanite", HEXAGONAL, UNI_POS, GR_DISP_SELLMEIER3, {1.163887f, 4.408433f, 21.53f},
                 {0.0f, 0.03178f, 1000.0f}, 0.0415f, ABS_ISO, {}, {}, {}, 0, 1, 0, false, 0});
    v.push_back({"Cubic Zirconia", CUBIC, ISO, GR_DISP_SELLMEIER3, {1.347091f, 2.117788f, 9.452943f},
                 {0.003912f, 0.027802f, 591.489f}, 0.0f, ABS_ISO, {}, {}, {}, 0, 1, 0, false, 0});
    return v;
}

// GpuGemMaterial::encode (renderer/buffers.rs:313-345) + DispersionParams::encode (:347-385).
static inline gr_material encode_material(const MatSpec &s) {
    gr_material m;
    std::memset(&m, 0, sizeof(m));
    m.dispersion.model_type = s.disp;
    if (s.disp == GR_DISP_CAUCHY) {
        m.dispersion.param_a[0] = s.a[0]; m.dispersion.param_a[1] = s.a[1]; m.dispersion.param_a[2] = s.a[2];
    } else {
        for (int i = 0; i < 3; ++i) { m.dispersion.param_a[i] = s.a[i]; m.dispersion.param_b[i] = s.b[i]; }
    }
    m.dispersion.c_axis_and_birefringence[0] = s.cx;
    m.dispersion.c_axis_and_birefringence[1] = s.cy;
    m.dispersion.c_axis_and_birefringence[2] = s.cz;
    m.dispersion.c_axis_and_birefringence[3] = s.bire;
    m.dispersion.is_anisotropic = (s.crystal != CUBIC && std::fabs(s.bire) > 1e-4f) ? 1u : 0u;
    m.dispersion.biaxial_delta_beta_alpha = s.has_biax ? s.biax : 0.0f;
    m.dispersion.has_biaxial_delta = s.has_biax ? 1u : 0u;
    m.crystal_system = s.crystal;
    m.optical_character = s.optical;
    m.is_pleochroic = s.abs_kind == ABS_ISO ? 0u : 1u;
    // AbsorptionTensor::{isotropic, uniaxial, biaxial}: biaxial stores alpha->o_ray,
    // gamma->e_ray, beta->beta_ray (optics/absorption.rs).
    if (s.abs_kind == ABS_ISO) {
        set_bands(m.o_ray_bands, m.o_ray_band_count, s.o);
        set_bands(m.e_ray_bands, m.e_ray_band_count, s.o);
        set_bands(m.beta_ray_bands, m.beta_ray_band_count, {});
    } else if (s.abs_kind == ABS_UNI) {
        set_bands(m.o_ray_bands, m.o_ray_band_count, s.o);
        set_bands(m.e_ray_bands, m.e_ray_band_count, s.e);
        set_bands(m.beta_ray_bands, m.beta_ray_band_count, {});
    } else {
        set_bands(m.o_ray_bands, m.o_ray_band_count, s.o);
        set_bands(m.e_ray_bands, m.e_ray_band_count, s.e);
        set_bands(m.beta_ray_bands, m.beta_ray_band_count, s.beta);
        m.has_beta_ray = 1;
    }
    m.scattering_sigma_s = 0.0f;
    m.scattering_g = 0.0f;
    m.edge_rounding_radius = 0.0f;
    m.absorption_path_scale = 1.0f;
    return m;
}

static inline bool builtin_material(const char *name, gr_material *out) {
    for (const MatSpec &s : material_specs())
        if (std::string(s.name) == name) { *out = encode_material(s); return true; }
    return false;
}

}  // namespace gro
