// gr_device.cuh -- device-side physics of the spectral transport path (sm_100a).
//
// One path-sample = one (pixel, absolute sample) tuple traced through a convex
// polyhedron with 8 hero-wavelength channels, each carrying a Stokes vector.  Every
// function states the reference item whose arithmetic it keeps (paths are inside the
// gemray-studio workspace, crates/gemray/src/...).  Floating-point contract:
//   * the file is compiled with --fmad=false: a*b+c is never contracted; fmaf()
//     appears exactly where the reference writes `f32::mul_add`;
//   * '/' and sqrtf are IEEE round-to-nearest (-prec-div/-prec-sqrt default);
//   * sinf/cosf/atan2f/atanf/acosf/expf are CUDA's accurate (non-intrinsic) forms;
//     `simd::exp_f32x8` is the reference's own polynomial, written out below, so it
//     is bit-identical to the reference on every input.
#pragma once

#include <cfloat>
#include <cstdint>

#include "gemray_cuda.h"

// Resident 128-thread blocks per SM the transport kernels' register allocation targets
// by default: 9 caps them at 56 registers, measured on B200 2-5% faster than the
// unconstrained 64-72 (more warps to hide the scalar physics code's latency outweigh a
// few spilled values).  The staged single-scene kernels are built for 9, 10, 12 and 16
// blocks (kScheduleBlocks), among which their per-stone schedule tuner chooses.
#ifndef GR_TRACE_MIN_BLOCKS
#define GR_TRACE_MIN_BLOCKS 9
#endif

namespace grd {

// ---------------------------------------------------------------------------------
// Scene constants (kernel parameter, uniform across the launch).
// ---------------------------------------------------------------------------------
struct SceneConst {
    float cam_o[3], cam_f[3], cam_r[3], cam_u[3];
    float fov_tan, width_f, height_f;
    uint32_t width, height, max_bounces, n_planes;
    // material (GpuGemMaterial fields the polished uniaxial path reads)
    uint32_t disp_model;
    float disp_a[3], disp_b[3];
    float bire;
    float c_axis[3];
    uint32_t anisotropic;
    uint32_t n_o_bands, n_e_bands;
    float o_bands[GR_MAX_BANDS][3], e_bands[GR_MAX_BANDS][3];
    uint32_t absorbing;  // any absorption data at all (bands or table)
    float path_scale, edge_radius;
    float ax0[3], ax1[3], ax2[3];  // AbsorptionTensor3::uniaxial frame, host-built
    // extension material data
    uint32_t ext_n;
    float ext_first, ext_step;
    uint32_t has_cauchy_e;
    float cauchy_e[3];
    // environment
    uint32_t env_mode;
    float uni_rgb[3];
    float temp_k, spot_mult, exposure;
    float denom560;  // max(exp(hck / (560 * T)) - 1, 1e-6), host-built
    float wb[3];     // von Kries LMS scale, host-built
    float key[3], fill[3], ring[16][3];  // StudioRig::new, host-built
    uint32_t map_w, map_h;
    uint32_t flags;
    // frosted facet finishes (bit i = plane i) and Henyey-Greenstein volume scattering
    uint32_t any_frosted;
    uint32_t frosted[GR_MAX_PLANES / 32];
    float sigma_s, hg_g;
    // biaxial indicatrix (optics/birefringence.rs:349-839): per channel n_beta = the
    // dispersion index, n_alpha = n_beta - d_beta_alpha, n_gamma = n_alpha + bire, in
    // the frame ax0/ax1/ax2; beta-ray absorption bands (trichroism, biaxial only)
    uint32_t biaxial;
    float d_beta_alpha;
    uint32_t has_beta, n_b_bands;
    float b_bands[GR_MAX_BANDS][3];
};

// Scenes that need the extension instantiation of the transport kernels (frosted
// facets, volume scattering, biaxial materials); every other scene runs the default
// instantiation, which contains none of that code.
__host__ __device__ inline bool needs_extras(const SceneConst &S) {
    return S.any_frosted || S.sigma_s > 0.0f || S.biaxial;
}

struct SceneBuffers {
    const float4 *planes;      // n_planes
    const float *map;          // map_w * map_h * 3
    const float *ext_alpha_o;  // ext_n
    const float *ext_alpha_e;  // ext_n
};

// ---------------------------------------------------------------------------------
// libm calls.  With GR_OUTLINE_MATH each CUDA math routine is emitted once and called,
// keeping the transport kernel's instruction footprint inside the SM instruction
// cache; the results are the same functions either way.
// ---------------------------------------------------------------------------------
#ifdef GR_OUTLINE_MATH
#define GR_MATH static __device__ __noinline__
#else
#define GR_MATH static __device__ __forceinline__
#endif
GR_MATH float2 m_sincos(float x) {
    float s, c;
    sincosf(x, &s, &c);
    return make_float2(s, c);
}
GR_MATH float m_atan2(float y, float x) { return atan2f(y, x); }
GR_MATH float m_atan(float x) { return atanf(x); }
GR_MATH float m_acos(float x) { return acosf(x); }
GR_MATH float m_exp(float x) { return expf(x); }
GR_MATH float m_log(float x) { return logf(x); }

// ---------------------------------------------------------------------------------
// Small vector helpers with glam's scalar semantics (no contraction).
// ---------------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 smul(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 cmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ V3 normalize(V3 a) { return mul(a, 1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ V3 normalize_or_zero(V3 a) {
    float r = 1.0f / sqrtf(dot(a, a));
    if (isfinite(r) && r > 0.0f) return mul(a, r);
    return v3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ V3 ld3(const float *p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
__device__ __forceinline__ float rem_euclid(float a, float b) {
    float r = fmodf(a, b);
    return r < 0.0f ? r + fabsf(b) : r;
}
// f32::powi: binary square-and-multiply (LLVM's powi expansion).
template <int N> __device__ __forceinline__ float powi(float x) {
    float r = 1.0f;
    bool have = false;
    float sq = x;
    int n = N;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (n) {
            if (n & 1) {
                r = have ? r * sq : sq;
                have = true;
            }
            n >>= 1;
            if (n) sq = sq * sq;
        }
    }
    return r;
}

// simd/exp_poly.rs:23-40 -- the reference's polynomial exponential, bit-exact.
__device__ __forceinline__ float exp_poly(float x) {
    const float LOG2E = 1.44269504088896340736f;
    const float C1 = __uint_as_float(0x3F318000u);
    const float C2 = -2.1219444e-4f;
    if (x < -87.33654f) x = -87.33654f;
    if (x > 88.02875f) x = 88.02875f;
    float n = floorf(fmaf(x, LOG2E, 0.5f));
    x = fmaf(n, -C1, x);
    x = fmaf(n, -C2, x);
    float z = x * x;
    float p = 1.9875691e-4f;
    p = fmaf(p, x, 1.3981999e-3f);
    p = fmaf(p, x, 8.333452e-3f);
    p = fmaf(p, x, 4.1665796e-2f);
    p = fmaf(p, x, 1.6666665e-1f);
    p = fmaf(p, x, 5.0000003e-1f);
    p = fmaf(p, z, x) + 1.0f;
    return p * __uint_as_float((uint32_t)(((int)n + 127) << 23));
}

// ---------------------------------------------------------------------------------
// a1. Sampler -- optics/raytracer/sampling.rs (integer-exact)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {  // sampling.rs:45-51
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float ld_base2(uint32_t n) {  // sampling.rs:139-147
    return (float)__brev(n) / 4294967296.0f;
}
template <uint32_t BASE> __device__ __forceinline__ float radical_inverse(uint32_t n) {  // sampling.rs:170-181
    float val = 0.0f;
    float inv_base = 1.0f / (float)BASE;
    while (n > 0) {
        uint32_t digit = n % BASE;
        val = fmaf((float)digit, inv_base, val);
        inv_base = inv_base / (float)BASE;
        n /= BASE;
    }
    return val;
}
__device__ __forceinline__ float cp_rotate(float x, float off) {  // sampling.rs:194-197
    float s = x + off;
    return s - floorf(s);
}
// Per-bounce draw: hash_u32(seed ^ hash_u32(bounce ^ SALT)) / 4294967295.0
__device__ __forceinline__ float rng_draw(uint32_t seed, uint32_t bounce, uint32_t salt) {
    return (float)hash_u32(seed ^ hash_u32(bounce ^ salt)) / 4294967295.0f;
}
constexpr uint32_t FRESNEL_BRANCH_STREAM = 0x9E3779B1u;
constexpr uint32_t RUSSIAN_ROULETTE_STREAM = 0x517CC1B7u;
constexpr uint32_t BIREFRINGENT_SPLIT_STREAM = 0x2545F491u;
constexpr uint32_t MODE_COUPLING_STREAM = 0xCC9E2D51u;
constexpr uint32_t PIXEL_JITTER_X_ROTATION_STREAM = 0xA511E9B3u;
constexpr uint32_t PIXEL_JITTER_Y_ROTATION_STREAM = 0x63D81B23u;
constexpr uint32_t HERO_WAVELENGTH_ROTATION_STREAM = 0x1B873593u;
constexpr uint32_t FROSTED_DIR_U_STREAM = 0x27D4EB2Fu;    // sampling.rs:28-41
constexpr uint32_t FROSTED_DIR_V_STREAM = 0x165667B1u;
constexpr uint32_t DISTANCE_SAMPLE_STREAM = 0xA24BAED4u;
constexpr uint32_t PHASE_DIR_U_STREAM = 0x9FB21C65u;
constexpr uint32_t PHASE_DIR_V_STREAM = 0x1CE4E5B9u;

struct Draws {
    uint32_t seed;
    float jx, jy, hero;
};
// sampling.rs:232-271 (pixel_rotations + sample_draws)
__device__ __forceinline__ Draws sample_draws(uint32_t pixel, uint32_t sample) {
    float rx = ld_base2(hash_u32(pixel ^ PIXEL_JITTER_X_ROTATION_STREAM));
    float ry = ld_base2(hash_u32(pixel ^ PIXEL_JITTER_Y_ROTATION_STREAM));
    float rh = ld_base2(hash_u32(pixel ^ HERO_WAVELENGTH_ROTATION_STREAM));
    Draws d;
    d.seed = hash_u32((pixel * 0x9e3779b9u) ^ (sample * 0x85ebca6bu));
    d.jx = cp_rotate(ld_base2(sample), rx) - 0.5f;
    d.jy = cp_rotate(radical_inverse<3>(sample), ry) - 0.5f;
    d.hero = cp_rotate(radical_inverse<5>(sample), rh);
    return d;
}

// ---------------------------------------------------------------------------------
// Material / spectrum helpers
// ---------------------------------------------------------------------------------
// transport.rs:45-53
__device__ __forceinline__ float lambda_k(float hero, int k) {
    float lh = fmaf(hero, 400.0f, 380.0f);
    float off = fmaf((float)k, 50.0f, lh - 380.0f);
    return 380.0f + rem_euclid(off, 400.0f);
}
// dispersion.rs:12-37
__device__ __forceinline__ float dispersion(const SceneConst &S, float lambda_nm) {
    float lum = lambda_nm * 1e-3f;
    float l2 = lum * lum;
    if (S.disp_model == GR_DISP_SELLMEIER1) {
        float n2 = 1.0f + (S.disp_a[0] * l2) / (l2 - S.disp_b[0]);
        return sqrtf(fmaxf(n2, 1.0f));
    } else if (S.disp_model == GR_DISP_SELLMEIER3) {
        float n2 = 1.0f;
        n2 = n2 + (S.disp_a[0] * l2) / (l2 - S.disp_b[0]);
        n2 = n2 + (S.disp_a[1] * l2) / (l2 - S.disp_b[1]);
        n2 = n2 + (S.disp_a[2] * l2) / (l2 - S.disp_b[2]);
        return sqrtf(fmaxf(n2, 1.0f));
    }
    float l4 = l2 * l2;
    return S.disp_a[0] + (S.disp_a[1] / l2) + (S.disp_a[2] / l4);
}
// optics/absorption.rs:30-33 summed as raytracer/absorption.rs:28-30 (fold from -0.0)
__device__ __forceinline__ float band_sum(const float (*bands)[3], uint32_t n, float lambda_nm) {
    float acc = -0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        float t = (lambda_nm - bands[i][0]) / bands[i][1];
        acc = acc + bands[i][2] * m_exp(-0.5f * t * t);
    }
    return acc;
}
__device__ __forceinline__ float table_lookup(const float *tab, uint32_t n, float first, float step, float lambda) {
    float f = (lambda - first) / step;
    if (!(f > 0.0f)) return tab[0];
    if (f >= (float)(n - 1)) return tab[n - 1];
    uint32_t i = (uint32_t)f;
    float t = f - (float)i;
    return tab[i] + t * (tab[i + 1] - tab[i]);
}

// ---------------------------------------------------------------------------------
// Stokes / Mueller -- optics/polarization.rs
// ---------------------------------------------------------------------------------
struct Stokes {
    float i, q, u, v;
};
__device__ __forceinline__ float intensity(const Stokes &s) { return fmaxf(s.i, 0.0f); }
__device__ __forceinline__ Stokes scale(const Stokes &s, float f) { return Stokes{s.i * f, s.q * f, s.u * f, s.v * f}; }
__device__ __forceinline__ float dop(const Stokes &s) {  // polarization.rs:38-48
    if (s.i <= 1e-7f) return 0.0f;
    return clampf(sqrtf(fmaf(s.v, s.v, fmaf(s.u, s.u, s.q * s.q))) / s.i, 0.0f, 1.0f);
}
// glam Mat4::mul_vec4 for the matrix families the transport uses.  Each row is the
// full left-to-right sum ((c0*x + c1*y) + c2*z) + c3*w including the zero entries,
// so signed zeros and non-finite values propagate exactly as on the CPU.
// frame_rotation(psi), polarization.rs:95-101 (cols: e0, (0,c2,-s2,0), (0,s2,c2,0), e3)
__device__ __forceinline__ Stokes apply_rotation(const Stokes &s, float c2, float s2) {
    Stokes o;
    o.i = ((1.0f * s.i + 0.0f * s.q) + 0.0f * s.u) + 0.0f * s.v;
    o.q = ((0.0f * s.i + c2 * s.q) + s2 * s.u) + 0.0f * s.v;
    o.u = ((0.0f * s.i + (-s2) * s.q) + c2 * s.u) + 0.0f * s.v;
    o.v = ((0.0f * s.i + 0.0f * s.q) + 0.0f * s.u) + 1.0f * s.v;
    return o;
}
// fresnel_reflection / fresnel_transmission layout (cols (a,b,0,0),(b,a,0,0),(0,0,c,0),(0,0,0,c))
__device__ __forceinline__ Stokes apply_fresnel(const Stokes &s, float a, float b, float c) {
    Stokes o;
    o.i = ((a * s.i + b * s.q) + 0.0f * s.u) + 0.0f * s.v;
    o.q = ((b * s.i + a * s.q) + 0.0f * s.u) + 0.0f * s.v;
    o.u = ((0.0f * s.i + 0.0f * s.q) + c * s.u) + 0.0f * s.v;
    o.v = ((0.0f * s.i + 0.0f * s.q) + 0.0f * s.u) + c * s.v;
    return o;
}
// tir_retardation(delta), polarization.rs:141-147 (cols e0, e1, (0,0,cd,-sd), (0,0,sd,cd))
__device__ __forceinline__ Stokes apply_tir(const Stokes &s, float cd, float sd) {
    Stokes o;
    o.i = ((1.0f * s.i + 0.0f * s.q) + 0.0f * s.u) + 0.0f * s.v;
    o.q = ((0.0f * s.i + 1.0f * s.q) + 0.0f * s.u) + 0.0f * s.v;
    o.u = ((0.0f * s.i + 0.0f * s.q) + cd * s.u) + sd * s.v;
    o.v = ((0.0f * s.i + 0.0f * s.q) + (-sd) * s.u) + cd * s.v;
    return o;
}
// Rust f32::midpoint on x86_64 == correctly rounded (a+b)/2 == (a+b)*0.5 in f32 for
// every non-subnormal sum.
__device__ __forceinline__ float midpoint(float a, float b) { return (a + b) * 0.5f; }

// Fresnel reflection matrix coefficients (polarization.rs:105-115)
__device__ __forceinline__ void fresnel_reflection_abc(float rs, float rp, float &a, float &b, float &c) {
    float rs2 = rs * rs, rp2 = rp * rp;
    a = midpoint(rs2, rp2);
    b = 0.5f * (rs2 - rp2);
    c = rs * rp;
}
// Fresnel transmission coefficients (polarization.rs:119-137)
__device__ __forceinline__ void fresnel_transmission_abc(float n1, float n2, float ci, float ct, float ts, float tp,
                                                         float &a, float &b, float &c) {
    float factor = (n2 * ct) / fmaxf(n1 * ci, 1e-6f);
    float ts2 = ts * ts * factor, tp2 = tp * tp * factor;
    a = midpoint(ts2, tp2);
    b = 0.5f * (ts2 - tp2);
    c = ts * tp * factor;
}
__device__ __forceinline__ void fresnel_rs_rp(float n1, float n2, float ci, float ct, float &rs, float &rp) {
    rs = fmaf(n2, -ct, n1 * ci) / fmaf(n2, ct, n1 * ci);
    rp = fmaf(n1, -ct, n2 * ci) / fmaf(n1, ct, n2 * ci);
}
__device__ __forceinline__ float r_unpol(float rs, float rp) {
    return clampf(0.5f * fmaf(rp, rp, rs * rs), 1e-4f, 1.0f - 1e-4f);
}
// refraction.rs:46-50
__device__ __forceinline__ float tir_phase_delta(float n1k, float ci, float si) {
    float num = ci * sqrtf(fmaxf(fmaf(n1k * n1k * si, si, -1.0f), 0.0f));
    float den = fmaxf(n1k * si * si, 1e-6f);
    return 2.0f * m_atan(num / den);
}

// polarization.rs:197-200 / birefringence.rs:126-131 (same construction)
__device__ __forceinline__ V3 perp_basis_t(V3 n) {
    V3 a = fabsf(n.x) > 0.9f ? v3(0.f, 1.f, 0.f) : v3(1.f, 0.f, 0.f);
    return normalize_or_zero(sub(a, mul(n, dot(n, a))));
}
// polarization.rs:172-192
__device__ __forceinline__ V3 electric_field_direction(const Stokes &st, V3 s_axis, V3 prop) {
    V3 k = normalize_or_zero(prop);
    V3 s_raw = sub(s_axis, mul(k, dot(k, s_axis)));
    V3 s_hat = dot(s_raw, s_raw) > 1e-8f ? normalize(s_raw) : perp_basis_t(k);
    V3 p_hat = cross(k, s_hat);
    float psi = 0.5f * m_atan2(st.u, st.q);
    float sp, cp;
    { float2 sc_ = m_sincos(psi); sp = sc_.x; cp = sc_.y; }
    V3 e = add(smul(cp, s_hat), smul(sp, p_hat));
    return dot(e, e) > 1e-8f ? normalize(e) : s_hat;
}

// ---------------------------------------------------------------------------------
// Uniaxial birefringence -- optics/birefringence.rs
// ---------------------------------------------------------------------------------
// :27-38 with sin/cos of theta supplied (same values the reference recomputes).
__device__ __forceinline__ float eff_e_index(float n_o, float n_e, float st, float ct) {
    if (fabsf(n_o - n_e) < 1e-5f) return n_o;
    float ns = n_o * st;
    float denom_sq = fmaf(n_e * ct, n_e * ct, ns * ns);
    if (denom_sq <= 1e-8f) return n_o;
    return (n_o * n_e) / sqrtf(denom_sq);
}
// :42-55
__device__ __forceinline__ float walk_off_angle(float n_o, float n_e, float theta) {
    if (fabsf(n_o - n_e) < 1e-5f) return 0.0f;
    float n_o2 = n_o * n_o, n_e2 = n_e * n_e;
    float s, c;
    { float2 sc_ = m_sincos(theta); s = sc_.x; c = sc_.y; }
    float num = (n_o2 - n_e2) * s * c;
    float den = fmaxf(fmaf(n_e2 * c, c, n_o2 * s * s), 1e-6f);
    return m_atan(num / den);
}
// :74-91 (outlined: rare, large)
static __device__ __noinline__ V3 extraordinary_poynting_dir(V3 wn, V3 c_axis, float n_o, float n_e) {
    float cos_theta = clampf(dot(wn, c_axis), -1.0f, 1.0f);
    float theta = m_acos(fabsf(cos_theta));
    float delta = walk_off_angle(n_o, n_e, theta);
    if (fabsf(delta) < 1e-5f) return wn;
    V3 c_proj = normalize_or_zero(sub(c_axis, smul(cos_theta, wn)));
    if (dot(c_proj, c_proj) < 1e-6f) return wn;
    float sign = cos_theta >= 0.0f ? 1.0f : -1.0f;
    float sd, cd;
    { float2 sc_ = m_sincos(delta); sd = sc_.x; cd = sc_.y; }
    return normalize(sub(mul(wn, cd), mul(smul(sign, c_proj), sd)));
}
// :101-118
__device__ __forceinline__ V3 ordinary_eigen(V3 wn, V3 c) {
    V3 cr = cross(wn, c);
    if (dot(cr, cr) > 1e-8f) return normalize(cr);
    return perp_basis_t(normalize_or_zero(wn));
}
__device__ __forceinline__ V3 extraordinary_eigen_from(V3 wn, V3 o) { return normalize_or_zero(cross(wn, o)); }

// AbsorptionTensor3::quadratic_form (:252-255) for alpha = (a_o, a_o, a_e).
__device__ __forceinline__ float quad_form(const SceneConst &S, float a_o, float a_e, V3 e) {
    float l0 = dot(ld3(S.ax0), e), l1 = dot(ld3(S.ax1), e), l2 = dot(ld3(S.ax2), e);
    return (a_o * (l0 * l0) + a_o * (l1 * l1)) + a_e * (l2 * l2);
}
// ... and for AbsorptionTensor3::biaxial (:238-245), alpha = (a_o, a_b, a_e).
__device__ __forceinline__ float quad_form3(const SceneConst &S, float a_o, float a_b, float a_e, V3 e) {
    float l0 = dot(ld3(S.ax0), e), l1 = dot(ld3(S.ax1), e), l2 = dot(ld3(S.ax2), e);
    return (a_o * (l0 * l0) + a_b * (l1 * l1)) + a_e * (l2 * l2);
}

// ---------------------------------------------------------------------------------
// Biaxial indicatrix -- optics/birefringence.rs:133-170,349-839.  The principal frame
// is the scene's tensor frame (ax0, ax1, ax2) = (stable_orthonormal_basis(c), c), the
// construction BiaxialIndicatrix::from_gamma_axis and AbsorptionTensor3 share.
// ---------------------------------------------------------------------------------
struct Ind {
    float na, nb, ng;
};
// GemMaterial::biaxial_indicatrix (materials.rs:1508-1519) at the channel whose
// dispersion index is n_beta.
__device__ __forceinline__ Ind make_ind(const SceneConst &S, float n_beta) {
    Ind I;
    I.nb = n_beta;
    I.na = n_beta - S.d_beta_alpha;
    I.ng = I.na + S.bire;
    return I;
}
// axes^T * v and axes * v (glam Mat3::mul_vec3: column sums left to right)
__device__ __forceinline__ V3 ind_local(const SceneConst &S, V3 v) {
    return v3(dot(ld3(S.ax0), v), dot(ld3(S.ax1), v), dot(ld3(S.ax2), v));
}
__device__ __forceinline__ V3 ind_world(const SceneConst &S, V3 v) {
    return add(add(mul(ld3(S.ax0), v.x), mul(ld3(S.ax1), v.y)), mul(ld3(S.ax2), v.z));
}
// indices_are_degenerate (:508-511)
__device__ __forceinline__ bool ind_degenerate(float a, float b) {
    const float scale = fmaxf(fmaxf(fabsf(a), fabsf(b)), 1.0f);
    return fabsf(a - b) <= sqrtf(FLT_EPSILON) * scale;
}
// wave_indices (:435-498): Fresnel's equation of wave normals -> (n_slow, n_fast);
// degenerate pairs take the uniaxial closed form.
__device__ __forceinline__ void wave_indices(const SceneConst &S, const Ind &I, V3 wave_normal, float &ns, float &nf) {
    const V3 k = normalize_or_zero(wave_normal);
    const bool ab = ind_degenerate(I.na, I.nb), bg = ind_degenerate(I.nb, I.ng);
    if (ab && bg) {
        const float n = ((I.na + I.nb) + I.ng) / 3.0f;
        ns = n;
        nf = n;
        return;
    }
    if (ab || bg) {
        const V3 c = ab ? ld3(S.ax2) : ld3(S.ax0);
        const float n_o = ab ? midpoint(I.na, I.nb) : midpoint(I.nb, I.ng);
        const float n_e = ab ? I.ng : I.na;
        const float theta = m_acos(fabsf(clampf(dot(k, c), -1.0f, 1.0f)));
        const float2 sc = m_sincos(theta);
        const float n_eff = eff_e_index(n_o, n_e, sc.x, sc.y);
        ns = fmaxf(n_o, n_eff);
        nf = fminf(n_o, n_eff);
        return;
    }
    const V3 l = ind_local(S, k);
    const float a2 = l.x * l.x, b2 = l.y * l.y, g2 = l.z * l.z;
    const float b1 = 1.0f / (I.na * I.na), b2c = 1.0f / (I.nb * I.nb), b3 = 1.0f / (I.ng * I.ng);
    const float big_b = fmaf(a2, b2c + b3, fmaf(b2, b1 + b3, g2 * (b1 + b2c)));
    const float big_c = fmaf(a2, b2c * b3, fmaf(b2, b1 * b3, (g2 * b1) * b2c));
    const float disc = sqrtf(fmaxf(fmaf(big_b, big_b, -4.0f * big_c), 0.0f));
    const float x_lo = 0.5f * (big_b - disc);
    const float x_hi = midpoint(big_b, disc);
    ns = 1.0f / sqrtf(fmaxf(x_lo, 1e-12f));
    nf = 1.0f / sqrtf(fmaxf(x_hi, 1e-12f));
}
__device__ __forceinline__ V3 cross_fma(V3 a, V3 b) {
    return v3(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
__device__ __forceinline__ float dot_fma(V3 a, V3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
// eigenvector_world (:659-702) with precise_root_near (:717-749): the D direction of
// the mode whose root is nearest x, in world space, its largest component positive.
static __device__ __noinline__ V3 eigenvector_world(const SceneConst &S, V3 l, float b0, float b1, float b2, float x_in,
                                                    V3 k_hat) {
    const float a = l.x * l.x, bb = l.y * l.y, cc = l.z * l.z;
    float x;
    {
        const float big_b = fmaf(a, b1 + b2, fmaf(bb, b0 + b2, cc * (b0 + b1)));
        const float xdiff = b0 - b1, ydiff = b2 - b0;
        const float a_plus_c = a + cc, a_plus_bb = a + bb;
        const float two_a_minus_bc = 2.0f * fmaf(bb, -cc, a);
        const float disc_sq = fmaf(a_plus_c * a_plus_c, xdiff * xdiff,
                                   fmaf(a_plus_bb * a_plus_bb, ydiff * ydiff, (two_a_minus_bc * xdiff) * ydiff));
        const float disc = sqrtf(fmaxf(disc_sq, 0.0f));
        const float x_lo = 0.5f * (big_b - disc);
        const float x_hi = midpoint(big_b, disc);
        x = fabsf(x_in - x_lo) <= fabsf(x_in - x_hi) ? x_lo : x_hi;
    }
    const float s = fmaf(b0, a, fmaf(b1, bb, (b2 * l.z) * l.z));
    const float m00 = fmaf(a, fmaf(2.0f, -b0, s), b0 - x);
    const float m11 = fmaf(bb, fmaf(2.0f, -b1, s), b1 - x);
    const float m22 = fmaf(cc, fmaf(2.0f, -b2, s), b2 - x);
    const float m01 = (l.x * l.y) * ((s - b0) - b1);
    const float m02 = (l.x * l.z) * ((s - b0) - b2);
    const float m12 = (l.y * l.z) * ((s - b1) - b2);
    const V3 r0 = v3(m00, m01, m02), r1 = v3(m01, m11, m12), r2 = v3(m02, m12, m22);
    const V3 c01 = cross_fma(r0, r1), c02 = cross_fma(r0, r2), c12 = cross_fma(r1, r2);
    const float s02 = dot_fma(c01, c02) < 0.0f ? -1.0f : 1.0f;
    const float s12 = dot_fma(c01, c12) < 0.0f ? -1.0f : 1.0f;
    const V3 vl = add(add(c01, mul(c02, s02)), mul(c12, s12));
    const V3 vw = ind_world(S, vl);
    if (dot(vw, vw) > 1e-12f) {
        const float ax = fabsf(vw.x), ay = fabsf(vw.y), az = fabsf(vw.z);
        const float largest = (ax >= ay && ax >= az) ? vw.x : (ay >= az ? vw.y : vw.z);
        return normalize(largest < 0.0f ? neg(vw) : vw);
    }
    return perp_basis_t(k_hat);
}
// eigen_polarizations (:542-554): the (slow, fast) D directions
__device__ __forceinline__ void eigen_pair(const SceneConst &S, const Ind &I, V3 wave_normal, V3 &d_slow, V3 &d_fast) {
    const V3 k = normalize_or_zero(wave_normal);
    const V3 l = ind_local(S, k);
    const float b0 = 1.0f / (I.na * I.na), b1 = 1.0f / (I.nb * I.nb), b2 = 1.0f / (I.ng * I.ng);
    float ns, nf;
    wave_indices(S, I, wave_normal, ns, nf);
    d_slow = eigenvector_world(S, l, b0, b1, b2, 1.0f / (ns * ns), k);
    d_fast = eigenvector_world(S, l, b0, b1, b2, 1.0f / (nf * nf), k);
}
// mode_poynting_dir (:831-836) = poynting_direction(k, d_to_e_direction(D of the mode))
// (:760-768, :860-870).  Only the requested mode's eigenvector is formed: the two are
// computed independently, so this is the reference's value.
static __device__ __noinline__ V3 mode_poynting_dir(const SceneConst &S, Ind I, V3 wave_normal, bool want_slow) {
    const V3 k = normalize_or_zero(wave_normal);
    const V3 l = ind_local(S, k);
    const float b0 = 1.0f / (I.na * I.na), b1 = 1.0f / (I.nb * I.nb), b2 = 1.0f / (I.ng * I.ng);
    float ns, nf;
    wave_indices(S, I, wave_normal, ns, nf);
    const float n = want_slow ? ns : nf;
    const V3 d = eigenvector_world(S, l, b0, b1, b2, 1.0f / (n * n), k);
    const V3 dl = ind_local(S, d);
    const V3 el = v3(dl.x / (I.na * I.na), dl.y / (I.nb * I.nb), dl.z / (I.ng * I.ng));
    // d_to_e_direction normalizes, and poynting_direction normalizes its input again
    const V3 e = normalize_or_zero(normalize_or_zero(ind_world(S, el)));
    const V3 perp = sub(k, mul(e, dot(e, k)));
    const float len2 = dot(perp, perp);
    if (len2 > 1e-10f) {
        const float len = sqrtf(len2);
        return v3(perp.x / len, perp.y / len, perp.z / len);
    }
    return k;
}
// resolve_entry_mode (:795-818): two fixed-point steps of the refracted wave normal
static __device__ __noinline__ V3 resolve_entry_mode(const SceneConst &S, Ind I, V3 incident, V3 normal, float cos_i,
                                                     float n_seed, bool want_slow) {
    float n_guess = n_seed;
    V3 wave_dir = incident;
    for (int it = 0; it < 2; ++it) {
        const float eta = 1.0f / n_guess;
        const float s2 = eta * eta * fmaf(cos_i, -cos_i, 1.0f);
        if (s2 > 1.0f) break;
        const float ct = sqrtf(fmaxf(1.0f - s2, 0.0f));
        wave_dir = normalize(add(smul(eta, incident), smul(fmaf(eta, cos_i, -ct), normal)));
        float ns, nf;
        wave_indices(S, I, wave_dir, ns, nf);
        n_guess = want_slow ? ns : nf;
    }
    return wave_dir;
}

// ---------------------------------------------------------------------------------
// a13. Environment radiance -- raytracer/environment.rs, env_map*.rs
// ---------------------------------------------------------------------------------
// environment.rs:12-21 with the lambda-independent 560 nm term host-built.
__device__ __forceinline__ float blackbody(const SceneConst &S, float lambda_nm) {
    float t_k = fmaxf(S.temp_k, 1000.0f);
    float e = m_exp(fminf(14388000.0f / (lambda_nm * t_k), 80.0f));
    float denom = fmaxf(e - 1.0f, 1e-6f);
    float ratio = S.denom560 / denom;
    return clampf(powi<5>(560.0f / lambda_nm) * ratio, 0.01f, 20.0f);
}
// environment.rs:280-321
__device__ __forceinline__ float studio_radiance(const SceneConst &S, V3 dn, float lambda_nm) {
    float spec = blackbody(S, lambda_nm);
    float bg = fmaxf(fmaf(0.012f, fmaf(dn.y, 0.5f, 0.5f), 0.015f), 0.005f) * S.exposure;
    float rad = bg * spec;
    float key_dot = fmaxf(dot(dn, ld3(S.key)), 0.0f);
    if (key_dot > 0.0f) rad = fmaf(powi<28>(key_dot) * 12.0f * S.spot_mult * S.exposure, spec, rad);
    float fill_dot = fmaxf(dot(dn, ld3(S.fill)), 0.0f);
    if (fill_dot > 0.0f) rad = fmaf(powi<18>(fill_dot) * 4.5f * S.exposure, spec, rad);
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
        float ring_dot = fmaxf(dot(dn, ld3(S.ring[i])), 0.0f);
        if (ring_dot > 0.96f) {
            float spark = (ring_dot - 0.96f) / 0.04f;
            rad = fmaf(powi<6>(spark) * 22.0f * S.spot_mult * S.exposure, spec, rad);
        }
    }
    return rad;
}
// env_map_spectrum.rs asymmetric_gaussian / rgb_to_spectral_radiance
__device__ __forceinline__ float asym_gauss(float x, float mu, float slo, float shi) {
    float sigma = x < mu ? slo : shi;
    float t = (x - mu) / sigma;
    return m_exp(-0.5f * t * t);
}
__device__ __forceinline__ float rgb_to_spectral(float r, float g, float b, float lambda_nm) {
    r = fmaxf(r, 0.0f); g = fmaxf(g, 0.0f); b = fmaxf(b, 0.0f);
    return fmaf(r, asym_gauss(lambda_nm, 615.0f, 45.0f, 65.0f),
                fmaf(g, asym_gauss(lambda_nm, 545.0f, 45.0f, 45.0f), b * asym_gauss(lambda_nm, 465.0f, 40.0f, 45.0f)));
}
// env_map.rs:231-239 + 287-323: bilinear lat-long lookup (wrap u, clamp v).
__device__ __forceinline__ void latlong_rgb(const SceneConst &S, const float *__restrict__ map, V3 dir, float rgb[3]) {
    const float PI = 3.14159265358979323846f;
    V3 d = normalize_or_zero(dir);
    float theta = m_acos(clampf(d.y, -1.0f, 1.0f));
    float phi = m_atan2(d.x, d.z);
    float v = theta / PI;
    float u = rem_euclid(phi / (2.0f * PI), 1.0f);
    uint32_t w = S.map_w, h = S.map_h;
    if (w == 1 && h == 1) {
        rgb[0] = map[0]; rgb[1] = map[1]; rgb[2] = map[2];
        return;
    }
    float fx = fmaf(rem_euclid(u, 1.0f), (float)w, -0.5f);
    float fy = fmaf(clampf(v, 0.0f, 1.0f), (float)h, -0.5f);
    float x0 = floorf(fx), y0 = floorf(fy);
    float tx = fx - x0, ty = fy - y0;
    long long xi = (long long)x0, yi = (long long)y0;
    long long x0w = xi % (long long)w; if (x0w < 0) x0w += w;
    long long x1w = (xi + 1) % (long long)w; if (x1w < 0) x1w += w;
    long long y0c = yi < 0 ? 0 : (yi > (long long)h - 1 ? (long long)h - 1 : yi);
    long long y1c = (yi + 1) < 0 ? 0 : ((yi + 1) > (long long)h - 1 ? (long long)h - 1 : (yi + 1));
    const float *p00 = map + 3 * ((size_t)y0c * w + x0w), *p10 = map + 3 * ((size_t)y0c * w + x1w);
    const float *p01 = map + 3 * ((size_t)y1c * w + x0w), *p11 = map + 3 * ((size_t)y1c * w + x1w);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float top = fmaf(__ldg(p10 + c), tx, __ldg(p00 + c) * (1.0f - tx));
        float bot = fmaf(__ldg(p11 + c), tx, __ldg(p01 + c) * (1.0f - tx));
        rgb[c] = fmaf(bot, ty, top * (1.0f - ty));
    }
}

// ---------------------------------------------------------------------------------
// a14. CIE 1931 via the reference polynomial exp (color/cie1931.rs:78-98)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float lobe(float l, float mu, float slo, float shi) {
    float sigma = l < mu ? slo : shi;
    float t = (l - mu) / sigma;
    return exp_poly(-0.5f * t * t);
}
__device__ __forceinline__ V3 cmf(float l) {
    float x = fmaf(0.065f, -lobe(l, 501.1f, 20.4f, 26.2f),
                   fmaf(1.056f, lobe(l, 599.8f, 37.9f, 31.0f), 0.362f * lobe(l, 442.0f, 16.0f, 26.7f)));
    float y = fmaf(0.286f, lobe(l, 530.9f, 16.3f, 31.1f), 0.821f * lobe(l, 568.8f, 46.9f, 40.5f));
    float z = fmaf(0.681f, lobe(l, 459.0f, 26.0f, 13.8f), 1.217f * lobe(l, 437.0f, 11.8f, 36.0f));
    return v3(fmaxf(x, 0.0f), fmaxf(y, 0.0f), fmaxf(z, 0.0f));
}
// raytracer/color.rs:215-251 (Bradford von Kries round trip)
__device__ __forceinline__ V3 von_kries(V3 xyz, const float wb[3]) {
    V3 lms = v3(fmaf(0.8951f, xyz.x, fmaf(0.2664f, xyz.y, -0.1614f * xyz.z)),
                fmaf(-0.7502f, xyz.x, fmaf(1.7135f, xyz.y, 0.0367f * xyz.z)),
                fmaf(0.0389f, xyz.x, fmaf(-0.0685f, xyz.y, 1.0296f * xyz.z)));
    lms = v3(lms.x * wb[0], lms.y * wb[1], lms.z * wb[2]);
    return v3(fmaf(0.986993f, lms.x, fmaf(-0.147054f, lms.y, 0.159963f * lms.z)),
              fmaf(0.432305f, lms.x, fmaf(0.518360f, lms.y, 0.049291f * lms.z)),
              fmaf(-0.008529f, lms.x, fmaf(0.040043f, lms.y, 0.968487f * lms.z)));
}

// ---------------------------------------------------------------------------------
// Frosted facets and Henyey-Greenstein scattering (raytracer/scattering.rs:337-443)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void frosted_basis(V3 n, V3 &t, V3 &b) {
    const V3 a = fabsf(n.x) > 0.9f ? v3(0.f, 1.f, 0.f) : v3(1.f, 0.f, 0.f);
    t = normalize_or_zero(sub(a, mul(n, dot(n, a))));
    b = cross(n, t);
}

__device__ __forceinline__ V3 cosine_weighted_hemisphere(float u1, float u2, V3 n) {
    const float r = sqrtf(u1);
    const float theta = (2.0f * 3.14159265358979323846f) * u2;
    const float2 sc = m_sincos(theta);
    V3 t, b;
    frosted_basis(n, t, b);
    return normalize_or_zero(add(add(mul(t, r * sc.y), mul(b, r * sc.x)), mul(n, sqrtf(fmaxf(1.0f - u1, 0.0f)))));
}

__device__ __forceinline__ V3 sample_hg_direction(float u1, float u2, float g, V3 fwd) {
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = fmaf(2.0f, -u1, 1.0f);
    } else {
        const float one_minus_g2 = fmaf(g, -g, 1.0f);
        const float denom = fmaf(2.0f * g, u1, 1.0f - g);
        const float sq = one_minus_g2 / denom;
        cos_theta = fmaf(sq, -sq, fmaf(g, g, 1.0f)) / (2.0f * g);
    }
    cos_theta = clampf(cos_theta, -1.0f, 1.0f);
    const float sin_theta = sqrtf(fmaxf(fmaf(cos_theta, -cos_theta, 1.0f), 0.0f));
    const float phi = (2.0f * 3.14159265358979323846f) * u2;
    const float2 sc = m_sincos(phi);
    V3 t, b;
    frosted_basis(fwd, t, b);
    return normalize_or_zero(add(add(mul(t, sin_theta * sc.y), mul(b, sin_theta * sc.x)), mul(fwd, cos_theta)));
}

__device__ __forceinline__ bool frosted_facet(const SceneConst &S, int idx) {
    return S.any_frosted && idx >= 0 && ((S.frosted[idx >> 5] >> (idx & 31)) & 1u);
}

}  // namespace grd
