// gr_oracle.hpp -- CPU restatement of gemray's spectral transport path.
//
// TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA engine is checked against:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
// The product (gemray_studio_b200/, libgemray_cuda.so) never links or calls it.
//
// It restates the reference Rust CPU tracer op for op:
//   * every `f32::mul_add` is `fma`, every other multiply/add is separate (the build
//     uses -ffp-contract=off), matching glam's scalar arithmetic
//     (crates/gemray/src/simd/mod.rs:13-17);
//   * Rust `f32::{sin,cos,tan,atan,atan2,acos,exp}` map to the platform libm;
//   * `simd::exp_f32x8` is the reference's own polynomial, restated bit-exactly.
// `Real` = float gives the FP32 oracle (pinned by the reference's to_bits goldens);
// `Real` = double gives the FP64 oracle: the same algorithm, every operation in
// double, sampler draws kept as their exact f32 values.
//
// glam 0.33.6 semantics used (third-party, not under the reference tree): Vec3::dot is
// (x*x' + y*y') + z*z'; cross is (y*z' - y'*z, z*x' - z'*x, x*y' - x'*y); normalize is
// v * (1/length); normalize_or_zero returns zero unless 1/length is finite and > 0;
// Mat4::mul_vec4 is ((c0*x + c1*y) + c2*z) + c3*w per row.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../include/gemray_cuda.h"

namespace gro {

// ---------------------------------------------------------------------------------
// Math policy: libm per precision, the reference's polynomial exp for FP32.
// ---------------------------------------------------------------------------------
template <class R> struct M;

template <> struct M<float> {
    static float sin(float x) { return ::sinf(x); }
    static float cos(float x) { return ::cosf(x); }
    static float tan(float x) { return ::tanf(x); }
    static float atan(float x) { return ::atanf(x); }
    static float atan2(float y, float x) { return ::atan2f(y, x); }
    static float acos(float x) { return ::acosf(x); }
    static float exp(float x) { return ::expf(x); }
    static float log(float x) { return ::logf(x); }
    static float sqrt(float x) { return ::sqrtf(x); }
    static float floor(float x) { return ::floorf(x); }
    static float fma(float a, float b, float c) { return ::fmaf(a, b, c); }
    static float fmod(float a, float b) { return ::fmodf(a, b); }
    // simd::exp_f32x8 lane (crates/gemray/src/simd/exp_poly.rs:8-40), Cephes/Moshier
    // constants with a Cody-Waite split of ln 2; bit-identical across dispatch levels.
    static float exp_poly(float xin) {
        const float LOG2E = 1.44269504088896340736f;
        float c1;
        const uint32_t c1_bits = 0x3F318000u;
        std::memcpy(&c1, &c1_bits, 4);
        const float C2 = -2.1219444e-4f;
        const float P0 = 1.9875691e-4f, P1 = 1.3981999e-3f, P2 = 8.333452e-3f;
        const float P3 = 4.1665796e-2f, P4 = 1.6666665e-1f, P5 = 5.0000003e-1f;
        const float HI = 88.02875f, LO = -87.33654f;
        float x = xin;
        if (x < LO) x = LO;
        if (x > HI) x = HI;
        float n = ::floorf(::fmaf(x, LOG2E, 0.5f));
        x = ::fmaf(n, -c1, x);
        x = ::fmaf(n, -C2, x);
        float z = x * x;
        float p = P0;
        p = ::fmaf(p, x, P1);
        p = ::fmaf(p, x, P2);
        p = ::fmaf(p, x, P3);
        p = ::fmaf(p, x, P4);
        p = ::fmaf(p, x, P5);
        p = ::fmaf(p, z, x) + 1.0f;
        uint32_t bits = (uint32_t)(((int32_t)n + 127) << 23);
        float pow2n;
        std::memcpy(&pow2n, &bits, 4);
        return p * pow2n;
    }
};

template <> struct M<double> {
    static double sin(double x) { return std::sin(x); }
    static double cos(double x) { return std::cos(x); }
    static double tan(double x) { return std::tan(x); }
    static double atan(double x) { return std::atan(x); }
    static double atan2(double y, double x) { return std::atan2(y, x); }
    static double acos(double x) { return std::acos(x); }
    static double exp(double x) { return std::exp(x); }
    static double log(double x) { return std::log(x); }
    static double sqrt(double x) { return std::sqrt(x); }
    static double floor(double x) { return std::floor(x); }
    static double fma(double a, double b, double c) { return std::fma(a, b, c); }
    static double fmod(double a, double b) { return std::fmod(a, b); }
    static double exp_poly(double x) { return std::exp(x); }
};

template <class R> static inline R rmax(R a, R b) { return a > b ? a : (b == b ? b : a); }
template <class R> static inline R rmin(R a, R b) { return a < b ? a : (b == b ? b : a); }
// Rust f32::clamp (NaN passes through).
template <class R> static inline R clampr(R x, R lo, R hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// Rust f32::rem_euclid.
template <class R> static inline R rem_euclid(R a, R b) {
    R r = M<R>::fmod(a, b);
    return r < R(0) ? r + std::fabs(b) : r;
}
// Rust f32::powi: binary square-and-multiply (LLVM powi expansion / __powisf2).
template <class R> static inline R powi(R x, int n) {
    R r = R(1);
    bool have = false;
    R sq = x;
    while (n) {
        if (n & 1) {
            r = have ? r * sq : sq;
            have = true;
        }
        n >>= 1;
        if (n) sq = sq * sq;
    }
    return have ? r : R(1);
}

// ---------------------------------------------------------------------------------
// glam::Vec3 with scalar glam semantics.
// ---------------------------------------------------------------------------------
template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    V3 operator+(const V3 &o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3 &o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
    V3 operator*(const V3 &o) const { return V3(x * o.x, y * o.y, z * o.z); }
    V3 operator-() const { return V3(-x, -y, -z); }
    R dot(const V3 &o) const { return (x * o.x + y * o.y) + z * o.z; }
    V3 cross(const V3 &o) const {
        return V3(y * o.z - o.y * z, z * o.x - o.z * x, x * o.y - o.x * y);
    }
    R length_squared() const { return dot(*this); }
    R length_recip() const { return R(1) / M<R>::sqrt(dot(*this)); }
    V3 normalize() const { return *this * length_recip(); }
    V3 normalize_or_zero() const {
        R rcp = length_recip();
        if (std::isfinite(rcp) && rcp > R(0)) return *this * rcp;
        return V3();
    }
};
template <class R> static inline V3<R> operator*(R s, const V3<R> &v) {
    return V3<R>(s * v.x, s * v.y, s * v.z);
}
template <class R> static inline V3<R> v3f(const float *p) { return V3<R>(R(p[0]), R(p[1]), R(p[2])); }

// ---------------------------------------------------------------------------------
// a1. Sampler -- crates/gemray/src/optics/raytracer/sampling.rs
// ---------------------------------------------------------------------------------
static const uint32_t FRESNEL_BRANCH_STREAM = 0x9E3779B1u;     // sampling.rs:12
static const uint32_t RUSSIAN_ROULETTE_STREAM = 0x517CC1B7u;   // sampling.rs:13
static const uint32_t BIREFRINGENT_SPLIT_STREAM = 0x2545F491u; // sampling.rs:17
static const uint32_t MODE_COUPLING_STREAM = 0xCC9E2D51u;      // sampling.rs:23
static const uint32_t PIXEL_JITTER_X_ROTATION_STREAM = 0xA511E9B3u; // sampling.rs:111
static const uint32_t PIXEL_JITTER_Y_ROTATION_STREAM = 0x63D81B23u; // sampling.rs:112
static const uint32_t HERO_WAVELENGTH_ROTATION_STREAM = 0x1B873593u; // sampling.rs:113
static const uint32_t FROSTED_DIR_U_STREAM = 0x27D4EB2Fu;    // sampling.rs:28
static const uint32_t FROSTED_DIR_V_STREAM = 0x165667B1u;    // sampling.rs:29
static const uint32_t DISTANCE_SAMPLE_STREAM = 0xA24BAED4u;  // sampling.rs:35
static const uint32_t PHASE_DIR_U_STREAM = 0x9FB21C65u;      // sampling.rs:40
static const uint32_t PHASE_DIR_V_STREAM = 0x1CE4E5B9u;      // sampling.rs:41

// sampling.rs:45-51
static inline uint32_t hash_u32(uint32_t x) {
    x = x * 0x85ebca6bu;
    x ^= x >> 13;
    x = x * 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

static inline uint32_t reverse_bits(uint32_t v) {
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
    v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
    return (v >> 16) | (v << 16);
}

// sampling.rs:139-147
static inline float low_discrepancy_base2(uint32_t n) {
    return (float)reverse_bits(n) / 4294967296.0f;
}

// sampling.rs:170-181 (digit * inv_base fused, inv_base /= base)
static inline float radical_inverse_base(uint32_t n, uint32_t base) {
    uint32_t remaining = n;
    float val = 0.0f;
    float inv_base = 1.0f / (float)base;
    while (remaining > 0) {
        uint32_t digit = remaining % base;
        val = ::fmaf((float)digit, inv_base, val);
        inv_base /= (float)base;
        remaining /= base;
    }
    return val;
}

// sampling.rs:194-197
static inline float cranley_patterson_rotate(float x, float offset) {
    float sum = x + offset;
    return sum - ::floorf(sum);
}

struct PixelRotations { float jitter_x, jitter_y, hero; };
struct SampleDraws { uint32_t seed; float jitter_x, jitter_y, hero_rand; };

// sampling.rs:232-238
static inline PixelRotations pixel_rotations(uint32_t pixel) {
    PixelRotations r;
    r.jitter_x = low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_X_ROTATION_STREAM));
    r.jitter_y = low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_Y_ROTATION_STREAM));
    r.hero = low_discrepancy_base2(hash_u32(pixel ^ HERO_WAVELENGTH_ROTATION_STREAM));
    return r;
}

// sampling.rs:259-271
static inline SampleDraws sample_draws(uint32_t pixel, uint32_t sample_num, const PixelRotations &rot) {
    SampleDraws d;
    d.seed = hash_u32((pixel * 0x9e3779b9u) ^ (sample_num * 0x85ebca6bu));
    d.jitter_x = cranley_patterson_rotate(low_discrepancy_base2(sample_num), rot.jitter_x) - 0.5f;
    d.jitter_y = cranley_patterson_rotate(radical_inverse_base(sample_num, 3), rot.jitter_y) - 0.5f;
    d.hero_rand = cranley_patterson_rotate(radical_inverse_base(sample_num, 5), rot.hero);
    return d;
}

// Per-bounce uniform draw: hash_u32(seed ^ hash_u32(bounce ^ SALT)) / 4294967295.0
// (transport.rs:211-212, refraction.rs:775-776,1057-1058, transport.rs:325-326).
static inline float rng_draw(uint32_t seed, uint32_t bounce, uint32_t stream) {
    return (float)hash_u32(seed ^ hash_u32(bounce ^ stream)) / 4294967295.0f;
}

// ---------------------------------------------------------------------------------
// a2. Camera -- optics/raytracer/camera.rs:62-114
// ---------------------------------------------------------------------------------
template <class R> struct Ray { V3<R> origin, dir; };

// camera.rs:62-93 (FP32 only: scene input built on the host).
static inline gr_camera camera_new(float yaw, float pitch, float distance, float fov_deg) {
    float cos_p = ::cosf(pitch), sin_p = ::sinf(pitch);
    float cos_y = ::cosf(yaw), sin_y = ::sinf(yaw);
    V3<float> origin(distance * cos_p * sin_y, distance * sin_p, distance * cos_p * cos_y);
    V3<float> forward = (-origin).normalize();
    V3<float> world_up = std::fabs(cos_p) < 1e-4f ? V3<float>(0.f, 0.f, -1.f) : V3<float>(0.f, 1.f, 0.f);
    V3<float> right = forward.cross(world_up).normalize();
    V3<float> up = right.cross(forward).normalize();
    // f32::to_radians = x * (PI / 180) with the constant folded in f32.
    const float deg2rad = 3.14159265358979323846f / 180.0f;
    float fov_tan = ::tanf(fov_deg * deg2rad * 0.5f);
    gr_camera c;
    c.origin[0] = origin.x; c.origin[1] = origin.y; c.origin[2] = origin.z;
    c.forward[0] = forward.x; c.forward[1] = forward.y; c.forward[2] = forward.z;
    c.right[0] = right.x; c.right[1] = right.y; c.right[2] = right.z;
    c.up[0] = up.x; c.up[1] = up.y; c.up[2] = up.z;
    c.fov_tan = fov_tan;
    return c;
}

// camera.rs:95-114 in precision R (the estimator always takes the FP32 ray; the FP64
// form is the camera case bank's reference).
template <class R>
static inline Ray<R> generate_ray_t(const gr_camera &cam, R sx, R sy, R w, R h, R jx, R jy) {
    R aspect = w / h;
    R u = ((sx + jx) / w - R(0.5f)) * R(2) * aspect * R(cam.fov_tan);
    R v = (R(0.5f) - (sy + jy) / h) * R(2) * R(cam.fov_tan);
    V3<R> f = v3f<R>(cam.forward), r = v3f<R>(cam.right), up = v3f<R>(cam.up);
    V3<R> dir = (f + r * u + up * v).normalize();
    Ray<R> ray;
    ray.origin = v3f<R>(cam.origin);
    ray.dir = dir;
    return ray;
}
// camera.rs:95-114 (always FP32: the camera ray is an input of the estimator).
static inline Ray<float> generate_ray(const gr_camera &cam, float sx, float sy, float w, float h,
                                      float jx, float jy) {
    return generate_ray_t<float>(cam, sx, sy, w, h, jx, jy);
}

// ---------------------------------------------------------------------------------
// a3. transport.rs:45-53 wrapped_hero_wavelengths (N = 8)
// ---------------------------------------------------------------------------------
template <class R> static inline void wrapped_hero_wavelengths(float hero_rand, R out[8]) {
    const R span = R(780) - R(380);
    const R width = span / R(8);
    R lambda_hero = M<R>::fma(R(hero_rand), span, R(380));
    for (int k = 0; k < 8; ++k) {
        R offset = M<R>::fma(R(k), width, lambda_hero - R(380));
        out[k] = R(380) + rem_euclid(offset, span);
    }
}

// ---------------------------------------------------------------------------------
// a4. Material model: dispersion.rs:12-37, optics/absorption.rs:30-33,
//     raytracer/absorption.rs:28-30.
// ---------------------------------------------------------------------------------
template <class R> static inline R dispersion_evaluate(const gr_dispersion &d, R lambda_nm) {
    R lum = lambda_nm * R(1e-3f);
    R l2 = lum * lum;
    if (d.model_type == GR_DISP_SELLMEIER1) {
        R n2 = R(1) + (R(d.param_a[0]) * l2) / (l2 - R(d.param_b[0]));
        return M<R>::sqrt(rmax(n2, R(1)));
    } else if (d.model_type == GR_DISP_SELLMEIER3) {
        R n2 = R(1);
        n2 = n2 + (R(d.param_a[0]) * l2) / (l2 - R(d.param_b[0]));
        n2 = n2 + (R(d.param_a[1]) * l2) / (l2 - R(d.param_b[1]));
        n2 = n2 + (R(d.param_a[2]) * l2) / (l2 - R(d.param_b[2]));
        return M<R>::sqrt(rmax(n2, R(1)));
    }
    R l4 = l2 * l2;
    return R(d.param_a[0]) + (R(d.param_a[1]) / l2) + (R(d.param_a[2]) / l4);
}

// Sum over bands, folded from -0.0 like Rust's `Sum for f32`.
template <class R> static inline R spectral_absorption(const gr_band *bands, uint32_t n, R lambda_nm) {
    R acc = R(-0.0);
    for (uint32_t i = 0; i < n; ++i) {
        R t = (lambda_nm - R(bands[i].center_nm)) / R(bands[i].width_nm);
        acc = acc + R(bands[i].peak) * M<R>::exp(R(-0.5f) * t * t);
    }
    return acc;
}

// Extension: linear interpolation of a tabulated coefficient (clamped at the ends).
template <class R> static inline R table_lookup(const float *tab, uint32_t n, float first, float step, R lambda) {
    if (n == 0) return R(0);
    R f = (lambda - R(first)) / R(step);
    if (!(f > R(0))) return R(tab[0]);
    if (f >= R(n - 1)) return R(tab[n - 1]);
    uint32_t i = (uint32_t)f;
    R t = f - R(i);
    return R(tab[i]) + t * (R(tab[i + 1]) - R(tab[i]));
}

// ---------------------------------------------------------------------------------
// Stokes / Mueller -- optics/polarization.rs
// ---------------------------------------------------------------------------------
template <class R> struct Stokes {
    R i, q, u, v;
    R intensity() const { return rmax(i, R(0)); }  // polarization.rs:33-35
    // polarization.rs:38-48
    R degree_of_polarization() const {
        if (i <= R(1e-7f)) return R(0);
        R s = M<R>::sqrt(M<R>::fma(v, v, M<R>::fma(u, u, q * q))) / i;
        return clampr(s, R(0), R(1));
    }
    R polarization_azimuth() const { return R(0.5f) * M<R>::atan2(u, q); }  // :58-60
    Stokes scale(R s) const { return Stokes{i * s, q * s, u * s, v * s}; }   // :69-71
};

// Column-major 4x4 (glam Mat4::from_cols_array); m[c][r].
template <class R> struct Mat4 { R m[4][4]; };

// glam Mat4::mul_vec4: ((c0*x + c1*y) + c2*z) + c3*w.
template <class R> static inline Stokes<R> apply_matrix(const Stokes<R> &s, const Mat4<R> &a) {
    R o[4];
    for (int r = 0; r < 4; ++r) {
        R acc = a.m[0][r] * s.i;
        acc = acc + a.m[1][r] * s.q;
        acc = acc + a.m[2][r] * s.u;
        acc = acc + a.m[3][r] * s.v;
        o[r] = acc;
    }
    return Stokes<R>{o[0], o[1], o[2], o[3]};
}

template <class R> static inline Mat4<R> from_cols(const R a[16]) {
    Mat4<R> m;
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) m.m[c][r] = a[c * 4 + r];
    return m;
}

// Rust f32::midpoint on x86_64: ((a as f64 + b as f64) / 2.0) as f32, which equals the
// correctly rounded (a + b) / 2 -- identical to (a + b) * 0.5 in f32 for every
// non-subnormal sum.
template <class R> static inline R midpoint(R a, R b) {
    return R(((double)a + (double)b) / 2.0);
}

// polarization.rs:95-101
template <class R> static inline Mat4<R> frame_rotation(R psi) {
    R c2 = M<R>::cos(R(2) * psi), s2 = M<R>::sin(R(2) * psi);
    const R a[16] = {1, 0, 0, 0, 0, c2, -s2, 0, 0, s2, c2, 0, 0, 0, 0, 1};
    return from_cols(a);
}
// polarization.rs:105-115
template <class R> static inline Mat4<R> fresnel_reflection(R rs, R rp) {
    R rs2 = rs * rs, rp2 = rp * rp;
    R a = midpoint(rs2, rp2), b = R(0.5f) * (rs2 - rp2), c = rs * rp;
    const R m[16] = {a, b, 0, 0, b, a, 0, 0, 0, 0, c, 0, 0, 0, 0, c};
    return from_cols(m);
}
// polarization.rs:119-137
template <class R> static inline Mat4<R> fresnel_transmission(R n1, R n2, R cos_i, R cos_t, R ts, R tp) {
    R factor = (n2 * cos_t) / rmax(n1 * cos_i, R(1e-6f));
    R ts2 = ts * ts * factor, tp2 = tp * tp * factor;
    R a = midpoint(ts2, tp2), b = R(0.5f) * (ts2 - tp2), c = ts * tp * factor;
    const R m[16] = {a, b, 0, 0, b, a, 0, 0, 0, 0, c, 0, 0, 0, 0, c};
    return from_cols(m);
}
// polarization.rs:141-147
template <class R> static inline Mat4<R> tir_retardation(R delta) {
    R cd = M<R>::cos(delta), sd = M<R>::sin(delta);
    const R m[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, cd, -sd, 0, 0, sd, cd};
    return from_cols(m);
}

// polarization.rs:197-200
template <class R> static inline V3<R> arbitrary_perpendicular(const V3<R> &n) {
    V3<R> a = std::fabs(n.x) > R(0.9f) ? V3<R>(0, 1, 0) : V3<R>(1, 0, 0);
    return (a - n * n.dot(a)).normalize_or_zero();
}

// polarization.rs:172-192
template <class R> static inline V3<R> electric_field_direction(const Stokes<R> &st, const V3<R> &s_axis,
                                                                 const V3<R> &prop) {
    V3<R> k = prop.normalize_or_zero();
    V3<R> s_raw = s_axis - k * k.dot(s_axis);
    V3<R> s_hat = s_raw.length_squared() > R(1e-8f) ? s_raw.normalize() : arbitrary_perpendicular(k);
    V3<R> p_hat = k.cross(s_hat);
    R psi = st.polarization_azimuth();
    V3<R> e = M<R>::cos(psi) * s_hat + M<R>::sin(psi) * p_hat;
    return e.length_squared() > R(1e-8f) ? e.normalize() : s_hat;
}

// ---------------------------------------------------------------------------------
// Uniaxial birefringence -- optics/birefringence.rs:27-131,202-286
// ---------------------------------------------------------------------------------
template <class R> static inline R effective_extraordinary_index(R n_o, R n_e, R theta) {  // :27-38
    if (std::fabs(n_o - n_e) < R(1e-5f)) return n_o;
    R s = M<R>::sin(theta), c = M<R>::cos(theta);
    R ns = n_o * s;
    R denom_sq = M<R>::fma(n_e * c, n_e * c, ns * ns);
    if (denom_sq <= R(1e-8f)) return n_o;
    return (n_o * n_e) / M<R>::sqrt(denom_sq);
}
template <class R> static inline R walk_off_angle(R n_o, R n_e, R theta) {  // :42-55
    if (std::fabs(n_o - n_e) < R(1e-5f)) return R(0);
    R n_o2 = n_o * n_o, n_e2 = n_e * n_e;
    R s = M<R>::sin(theta), c = M<R>::cos(theta);
    R num = (n_o2 - n_e2) * s * c;
    R den = rmax(M<R>::fma(n_e2 * c, c, n_o2 * s * s), R(1e-6f));
    return M<R>::atan(num / den);
}
template <class R>
static inline V3<R> extraordinary_poynting_dir(const V3<R> &wn, const V3<R> &c_axis, R n_o, R n_e) {  // :74-91
    R cos_theta = clampr(wn.dot(c_axis), R(-1), R(1));
    R theta = M<R>::acos(std::fabs(cos_theta));
    R delta = walk_off_angle(n_o, n_e, theta);
    if (std::fabs(delta) < R(1e-5f)) return wn;
    V3<R> c_proj = (c_axis - cos_theta * wn).normalize_or_zero();
    if (c_proj.length_squared() < R(1e-6f)) return wn;
    R sign = cos_theta >= R(0) ? R(1) : R(-1);
    return (wn * M<R>::cos(delta) - (sign * c_proj) * M<R>::sin(delta)).normalize();
}
template <class R> static inline void stable_orthonormal_basis(const V3<R> &n, V3<R> &t, V3<R> &b) {  // :126-131
    V3<R> a = std::fabs(n.x) > R(0.9f) ? V3<R>(0, 1, 0) : V3<R>(1, 0, 0);
    t = (a - n * n.dot(a)).normalize_or_zero();
    b = n.cross(t);
}
template <class R> static inline V3<R> ordinary_eigen_polarization(const V3<R> &wn, const V3<R> &c) {  // :101-108
    V3<R> cr = wn.cross(c);
    if (cr.length_squared() > R(1e-8f)) return cr.normalize();
    V3<R> t, b;
    stable_orthonormal_basis(wn.normalize_or_zero(), t, b);
    return t;
}
template <class R> static inline V3<R> extraordinary_eigen_polarization(const V3<R> &wn, const V3<R> &c) {  // :115-118
    V3<R> o = ordinary_eigen_polarization(wn, c);
    return wn.cross(o).normalize_or_zero();
}

// AbsorptionTensor3::uniaxial (:202-209): alpha = (a_o, a_o, a_e), axes = (a1, a2, c).
template <class R> struct Tensor3 { V3<R> alpha; V3<R> ax0, ax1, ax2; };
template <class R> static inline Tensor3<R> tensor_uniaxial(R a_o, R a_e, const V3<R> &c_axis) {
    Tensor3<R> t;
    V3<R> c = c_axis.normalize_or_zero();
    stable_orthonormal_basis(c, t.ax0, t.ax1);
    t.ax2 = c;
    t.alpha = V3<R>(a_o, a_o, a_e);
    return t;
}
// quadratic_form (:252-255): local = axes^T * e (glam Mat3 mul_vec3 order), alpha . local^2.
template <class R> static inline R quadratic_form(const Tensor3<R> &t, const V3<R> &e) {
    V3<R> local(t.ax0.dot(e), t.ax1.dot(e), t.ax2.dot(e));
    return t.alpha.dot(local * local);
}
// effective_pleochroic_alpha (:272-286)
template <class R>
static inline R effective_pleochroic_alpha(const Tensor3<R> &t, const V3<R> &e, const V3<R> &ea, const V3<R> &eb, R dop) {
    R p = clampr(dop, R(0), R(1));
    R a_pol = quadratic_form(t, e);
    R a_unpol = midpoint(quadratic_form(t, ea), quadratic_form(t, eb));
    return M<R>::fma(p, a_pol - a_unpol, a_unpol);
}

// ---------------------------------------------------------------------------------
// Biaxial indicatrix -- optics/birefringence.rs:133-170,349-839 (BiaxialIndicatrix),
// optics/materials.rs:1508-1519 (GemMaterial::biaxial_indicatrix)
// ---------------------------------------------------------------------------------
// Principal indices n_alpha <= n_beta <= n_gamma along the frame (ax0, ax1, ax2) =
// (stable_orthonormal_basis(c), c) -- the same frame as AbsorptionTensor3.
template <class R> struct Indicatrix { R na, nb, ng; V3<R> ax0, ax1, ax2; };

// biaxial_indicatrix (materials.rs:1508-1519) + from_gamma_axis (birefringence.rs:391-396):
// n_beta = dispersion(lambda), n_alpha = n_beta - delta_beta_alpha, n_gamma = n_alpha + birefringence.
template <class R> static inline Indicatrix<R> make_indicatrix(R n_beta, R d_beta_alpha, R bire, const V3<R> &c_axis) {
    Indicatrix<R> I;
    I.nb = n_beta;
    I.na = n_beta - d_beta_alpha;
    I.ng = I.na + bire;
    const V3<R> g = c_axis.normalize_or_zero();
    stable_orthonormal_basis(g, I.ax0, I.ax1);
    I.ax2 = g;
    return I;
}
// axes^T * v and axes * v (glam Mat3 mul_vec3: column sums, left to right)
template <class R> static inline V3<R> ind_local(const Indicatrix<R> &I, const V3<R> &v) {
    return V3<R>(I.ax0.dot(v), I.ax1.dot(v), I.ax2.dot(v));
}
template <class R> static inline V3<R> ind_world(const Indicatrix<R> &I, const V3<R> &v) {
    return (I.ax0 * v.x + I.ax1 * v.y) + I.ax2 * v.z;
}
// cross_fma / dot_fma / canonicalize_eigenvector_sign (birefringence.rs:139-170)
template <class R> static inline V3<R> cross_fma(const V3<R> &a, const V3<R> &b) {
    return V3<R>(M<R>::fma(a.y, b.z, -(a.z * b.y)), M<R>::fma(a.z, b.x, -(a.x * b.z)), M<R>::fma(a.x, b.y, -(a.y * b.x)));
}
template <class R> static inline R dot_fma(const V3<R> &a, const V3<R> &b) {
    return M<R>::fma(a.x, b.x, M<R>::fma(a.y, b.y, a.z * b.z));
}
template <class R> static inline V3<R> canonicalize_sign(const V3<R> &v) {
    const R ax = std::fabs(v.x), ay = std::fabs(v.y), az = std::fabs(v.z);
    const R largest = (ax >= ay && ax >= az) ? v.x : (ay >= az ? v.y : v.z);
    return largest < R(0) ? -v : v;
}
// indices_are_degenerate (:508-511): |a - b| <= sqrt(f32::EPSILON) * max(|a|, |b|, 1)
template <class R> static inline bool indices_degenerate(R a, R b) {
    const R scale = rmax(rmax(std::fabs(a), std::fabs(b)), R(1));
    return std::fabs(a - b) <= R(::sqrtf(FLT_EPSILON)) * scale;
}
// uniaxial_wave_indices (:494-498) -> (n_slow, n_fast)
template <class R> static inline void uniaxial_wave_indices(const V3<R> &k, const V3<R> &c, R n_o, R n_e, R &ns, R &nf) {
    const R theta = M<R>::acos(std::fabs(clampr(k.dot(c), R(-1), R(1))));
    const R n_eff = effective_extraordinary_index(n_o, n_e, theta);
    ns = rmax(n_o, n_eff);
    nf = rmin(n_o, n_eff);
}
// wave_indices (:435-484): Fresnel's equation of wave normals -> (n_slow, n_fast)
template <class R> static inline void wave_indices(const Indicatrix<R> &I, const V3<R> &wave_normal, R &ns, R &nf) {
    const V3<R> k = wave_normal.normalize_or_zero();
    const bool ab = indices_degenerate(I.na, I.nb);
    const bool bg = indices_degenerate(I.nb, I.ng);
    if (ab && bg) {
        const R n = ((I.na + I.nb) + I.ng) / R(3);
        ns = n;
        nf = n;
        return;
    }
    if (ab) { uniaxial_wave_indices(k, I.ax2, midpoint(I.na, I.nb), I.ng, ns, nf); return; }
    if (bg) { uniaxial_wave_indices(k, I.ax0, midpoint(I.nb, I.ng), I.na, ns, nf); return; }
    const V3<R> l = ind_local(I, k);
    const R a2 = l.x * l.x, b2 = l.y * l.y, g2 = l.z * l.z;
    const R b1 = R(1) / (I.na * I.na), b2c = R(1) / (I.nb * I.nb), b3 = R(1) / (I.ng * I.ng);
    const R big_b = M<R>::fma(a2, b2c + b3, M<R>::fma(b2, b1 + b3, g2 * (b1 + b2c)));
    const R big_c = M<R>::fma(a2, b2c * b3, M<R>::fma(b2, b1 * b3, g2 * b1 * b2c));
    const R disc = M<R>::sqrt(rmax(M<R>::fma(big_b, big_b, R(-4) * big_c), R(0)));
    const R x_lo = R(0.5f) * (big_b - disc);
    const R x_hi = midpoint(big_b, disc);
    ns = R(1) / M<R>::sqrt(rmax(x_lo, R(1e-12f)));
    nf = R(1) / M<R>::sqrt(rmax(x_hi, R(1e-12f)));
}
// precise_root_near (:717-749): the root of the same quadratic nearest x, its
// discriminant formed from direct differences of the principal 1/n^2
template <class R> static inline R precise_root_near(const V3<R> &l, const R b[3], R x) {
    const R a = l.x * l.x, bb = l.y * l.y, cc = l.z * l.z;
    const R big_b = M<R>::fma(a, b[1] + b[2], M<R>::fma(bb, b[0] + b[2], cc * (b[0] + b[1])));
    const R xdiff = b[0] - b[1];
    const R ydiff = b[2] - b[0];
    const R a_plus_c = a + cc;
    const R a_plus_bb = a + bb;
    const R two_a_minus_bc = R(2) * M<R>::fma(bb, -cc, a);
    const R disc_sq = M<R>::fma(a_plus_c * a_plus_c, xdiff * xdiff,
                                M<R>::fma(a_plus_bb * a_plus_bb, ydiff * ydiff, two_a_minus_bc * xdiff * ydiff));
    const R disc = M<R>::sqrt(rmax(disc_sq, R(0)));
    const R x_lo = R(0.5f) * (big_b - disc);
    const R x_hi = midpoint(big_b, disc);
    return std::fabs(x - x_lo) <= std::fabs(x - x_hi) ? x_lo : x_hi;
}
// eigenvector_world (:659-702): null vector of Gamma - x I (Gamma = P B P) as the
// sign-aligned sum of its three row-pair cross products, in world space
template <class R> static inline V3<R> eigenvector_world(const Indicatrix<R> &I, const V3<R> &l, const R b[3], R x_in,
                                                         const V3<R> &k_hat) {
    const R x = precise_root_near(l, b, x_in);
    const R s = M<R>::fma(b[0], l.x * l.x, M<R>::fma(b[1], l.y * l.y, b[2] * l.z * l.z));
    const R m00 = M<R>::fma(l.x * l.x, M<R>::fma(R(2), -b[0], s), b[0] - x);
    const R m11 = M<R>::fma(l.y * l.y, M<R>::fma(R(2), -b[1], s), b[1] - x);
    const R m22 = M<R>::fma(l.z * l.z, M<R>::fma(R(2), -b[2], s), b[2] - x);
    const R m01 = l.x * l.y * (s - b[0] - b[1]);
    const R m02 = l.x * l.z * (s - b[0] - b[2]);
    const R m12 = l.y * l.z * (s - b[1] - b[2]);
    const V3<R> row0(m00, m01, m02), row1(m01, m11, m12), row2(m02, m12, m22);
    const V3<R> c01 = cross_fma(row0, row1), c02 = cross_fma(row0, row2), c12 = cross_fma(row1, row2);
    const R sign02 = dot_fma(c01, c02) < R(0) ? R(-1) : R(1);
    const R sign12 = dot_fma(c01, c12) < R(0) ? R(-1) : R(1);
    const V3<R> v_local = (c01 + c02 * sign02) + c12 * sign12;
    const V3<R> v_world = ind_world(I, v_local);
    if (v_world.length_squared() > R(1e-12f)) return canonicalize_sign(v_world).normalize();
    V3<R> t, bt;
    stable_orthonormal_basis(k_hat, t, bt);
    return t;
}
// eigen_polarizations (:542-554): D directions of the (slow, fast) modes
template <class R> static inline void eigen_polarizations(const Indicatrix<R> &I, const V3<R> &wave_normal, V3<R> &d_slow,
                                                          V3<R> &d_fast) {
    const V3<R> k = wave_normal.normalize_or_zero();
    const V3<R> l = ind_local(I, k);
    const R b[3] = {R(1) / (I.na * I.na), R(1) / (I.nb * I.nb), R(1) / (I.ng * I.ng)};
    R ns, nf;
    wave_indices(I, wave_normal, ns, nf);
    const R x_slow = R(1) / (ns * ns);
    const R x_fast = R(1) / (nf * nf);
    d_slow = eigenvector_world(I, l, b, x_slow, k);
    d_fast = eigenvector_world(I, l, b, x_fast, k);
}
// d_to_e_direction (:760-768)
template <class R> static inline V3<R> d_to_e_direction(const Indicatrix<R> &I, const V3<R> &d_hat) {
    const V3<R> dl = ind_local(I, d_hat);
    const V3<R> el(dl.x / (I.na * I.na), dl.y / (I.nb * I.nb), dl.z / (I.ng * I.ng));
    return ind_world(I, el).normalize_or_zero();
}
// poynting_direction (:860-870): the component of k perpendicular to E
template <class R> static inline V3<R> poynting_direction(const V3<R> &wave_normal, const V3<R> &e_field) {
    const V3<R> k = wave_normal.normalize_or_zero();
    const V3<R> e = e_field.normalize_or_zero();
    const V3<R> perp = k - e * e.dot(k);
    const R len2 = perp.length_squared();
    if (len2 > R(1e-10f)) {
        const R l = M<R>::sqrt(len2);
        return V3<R>(perp.x / l, perp.y / l, perp.z / l);
    }
    return k;
}
// mode_poynting_dir (:831-836)
template <class R> static inline V3<R> mode_poynting_dir(const Indicatrix<R> &I, const V3<R> &wave_normal, bool want_slow) {
    V3<R> ds, df;
    eigen_polarizations(I, wave_normal, ds, df);
    return poynting_direction(wave_normal, d_to_e_direction(I, want_slow ? ds : df));
}
// resolve_entry_mode (:795-818): two fixed-point steps of the refracted wave normal
template <class R> static inline V3<R> resolve_entry_mode(const Indicatrix<R> &I, const V3<R> &incident, const V3<R> &normal,
                                                          R cos_i, R n_seed, bool want_slow) {
    R n_guess = n_seed;
    V3<R> wave_dir = incident;
    for (int it = 0; it < 2; ++it) {
        const R eta = R(1) / n_guess;
        const R s2 = eta * eta * M<R>::fma(cos_i, -cos_i, R(1));
        if (s2 > R(1)) break;
        const R ct = M<R>::sqrt(rmax(R(1) - s2, R(0)));
        wave_dir = (eta * incident + M<R>::fma(eta, cos_i, -ct) * normal).normalize();
        R ns, nf;
        wave_indices(I, wave_dir, ns, nf);
        n_guess = want_slow ? ns : nf;
    }
    return wave_dir;
}

// ---------------------------------------------------------------------------------
// a5. Polyhedron clip -- intersect.rs:93-132 + simd/slab.rs:101-152
// ---------------------------------------------------------------------------------
template <class R> struct Hit { bool hit; R t; V3<R> normal; int facet; };

// The reference scans planes with a vector pass computing every plane's (denom,
// side, t) lanes and a scalar replay of the per-plane decisions in ascending order
// (simd/slab.rs:186-382); both are written the same way here so the compiler can
// vectorise the first loop.  IEEE arithmetic per lane makes it bit-identical to the
// plain scalar scan.
template <class R> static inline Hit<R> intersect_polyhedron(const Ray<R> &ray, const gr_plane *planes, uint32_t n) {
    Hit<R> h;
    h.hit = false; h.t = 0; h.facet = 0;
    R t_near = R(-1e30f), t_far = R(1e30f);
    int near_idx = -1, far_idx = -1;
    constexpr uint32_t BLK = 64;
    R den[BLK], sid[BLK], tt[BLK];
    const R dx = ray.dir.x, dy = ray.dir.y, dz = ray.dir.z;
    const R ox = ray.origin.x, oy = ray.origin.y, oz = ray.origin.z;
    for (uint32_t b0 = 0; b0 < n; b0 += BLK) {
        const uint32_t cnt = n - b0 < BLK ? n - b0 : BLK;
        for (uint32_t j = 0; j < cnt; ++j) {
            const gr_plane &p = planes[b0 + j];
            R nx = R(p.normal[0]), ny = R(p.normal[1]), nz = R(p.normal[2]);
            R d = (nx * dx + ny * dy) + nz * dz;
            R sd = R(p.d) + ((nx * ox + ny * oy) + nz * oz);
            den[j] = d;
            sid[j] = sd;
            tt[j] = (-sd) / d;
        }
        for (uint32_t j = 0; j < cnt; ++j) {
            R denom = den[j], t = tt[j];
            if (std::fabs(denom) > R(1e-7f)) {
                if (denom < R(0)) {
                    if (t > t_near) { t_near = t; near_idx = (int)(b0 + j); }
                } else if (t < t_far) { t_far = t; far_idx = (int)(b0 + j); }
            } else if (sid[j] > R(0)) {
                return h;  // SlabScan::Outside
            }
        }
    }
    if (t_near > t_far) return h;
    if (t_near > R(1e-4f)) {
        h.hit = true; h.t = t_near;
        h.normal = near_idx >= 0 ? v3f<R>(planes[near_idx].normal) : V3<R>();
        h.facet = near_idx >= 0 ? near_idx : 0;
    } else if (t_far > R(1e-4f)) {
        h.hit = true; h.t = t_far;
        h.normal = far_idx >= 0 ? v3f<R>(planes[far_idx].normal) : V3<R>();
        h.facet = far_idx >= 0 ? far_idx : 0;
    }
    return h;
}

// a6. intersect.rs:196-229
template <class R>
static inline V3<R> shading_normal_near_edge(const gr_plane *planes, uint32_t n, const V3<R> &hp, int hit_idx,
                                             const V3<R> &hit_normal, R radius) {
    if (radius <= R(0)) return hit_normal;
    R nearest = R(INFINITY);
    V3<R> nearest_n = hit_normal;
    for (uint32_t i = 0; i < n; ++i) {
        if ((int)i == hit_idx) continue;
        V3<R> nn = v3f<R>(planes[i].normal);
        R dist = -(R(planes[i].d) + nn.dot(hp));
        if (dist < nearest) { nearest = dist; nearest_n = nn; }
    }
    if (nearest >= radius) return hit_normal;
    R t = clampr(R(1) - nearest / radius, R(0), R(1));
    R smooth_t = t * t * M<R>::fma(R(2), -t, R(3));
    V3<R> bis = (hit_normal + nearest_n).normalize_or_zero();
    return (hit_normal * (R(1) - smooth_t) + bis * smooth_t).normalize_or_zero();
}

// ---------------------------------------------------------------------------------
// a13. Environments -- raytracer/environment.rs, optics/studio_rig.rs,
//      renderer/env_map.rs, renderer/env_map_spectrum.rs
// ---------------------------------------------------------------------------------
// environment.rs:12-21
template <class R> static inline R blackbody_spectrum(R lambda_nm, R temp_k) {
    R t_k = rmax(temp_k, R(1000));
    const R hck = R(14388000.0f);
    R e = M<R>::exp(rmin(hck / (lambda_nm * t_k), R(80)));
    R e560 = M<R>::exp(rmin(hck / (R(560) * t_k), R(80)));
    R denom = rmax(e - R(1), R(1e-6f));
    R denom560 = rmax(e560 - R(1), R(1e-6f));
    R ratio = denom560 / denom;
    return clampr(powi(R(560) / lambda_nm, 5) * ratio, R(0.01f), R(20));
}

// studio_rig.rs:50-81
template <class R> struct StudioRig { V3<R> key, fill, ring[16]; R sin_lp; };
template <class R> static inline StudioRig<R> studio_rig_new(R yaw, R pitch) {
    StudioRig<R> rig;
    R cos_lp = M<R>::cos(pitch), sin_lp = M<R>::sin(pitch);
    R cos_ly = M<R>::cos(yaw), sin_ly = M<R>::sin(yaw);
    rig.key = V3<R>(cos_lp * sin_ly, sin_lp, cos_lp * cos_ly).normalize();
    const R PI = R(3.14159265358979323846f);
    R fill_yaw = M<R>::fma(PI, R(0.78f), yaw);
    R fill_pitch = clampr(pitch * R(0.65f), R(0.15f), R(1.2f));
    rig.fill = V3<R>(M<R>::cos(fill_pitch) * M<R>::sin(fill_yaw), M<R>::sin(fill_pitch),
                     M<R>::cos(fill_pitch) * M<R>::cos(fill_yaw)).normalize();
    const R step = R(3.14159265358979323846f * 2.0f / 16.0f);
    for (int i = 0; i < 16; ++i) {
        R angle = M<R>::fma(R(i), step, yaw);
        rig.ring[i] = V3<R>(M<R>::cos(angle) * R(0.75f), sin_lp * R(0.8f), M<R>::sin(angle) * R(0.75f)).normalize();
    }
    rig.sin_lp = sin_lp;
    return rig;
}

// environment.rs:280-321
template <class R>
static inline R studio_radiance(const V3<R> &dir, R lambda, R temp_k, R spot_mult, R exposure, const StudioRig<R> &rig) {
    V3<R> d = dir.normalize();
    R spec = blackbody_spectrum(lambda, temp_k);
    R bg = rmax(M<R>::fma(R(0.012f), M<R>::fma(d.y, R(0.5f), R(0.5f)), R(0.015f)), R(0.005f)) * exposure;
    R rad = bg * spec;
    R key_dot = rmax(d.dot(rig.key), R(0));
    if (key_dot > R(0)) {
        R softbox = powi(key_dot, 28) * R(12) * spot_mult * exposure;
        rad = M<R>::fma(softbox, spec, rad);
    }
    R fill_dot = rmax(d.dot(rig.fill), R(0));
    if (fill_dot > R(0)) {
        R fill = powi(fill_dot, 18) * R(4.5f) * exposure;
        rad = M<R>::fma(fill, spec, rad);
    }
    for (int i = 0; i < 16; ++i) {
        R ring_dot = rmax(d.dot(rig.ring[i]), R(0));
        if (ring_dot > R(0.96f)) {
            R spark = (ring_dot - R(0.96f)) / R(0.04f);
            R inten = powi(spark, 6) * R(22) * spot_mult * exposure;
            rad = M<R>::fma(inten, spec, rad);
        }
    }
    return rad;
}

// env_map_spectrum.rs (asymmetric_gaussian, rgb_to_spectral_radiance)
template <class R> static inline R asym_gauss(R x, R mu, R slo, R shi) {
    R sigma = x < mu ? slo : shi;
    R t = (x - mu) / sigma;
    return M<R>::exp(R(-0.5f) * t * t);
}
template <class R> static inline R rgb_to_spectral(R r0, R g0, R b0, R lambda) {
    R r = rmax(r0, R(0)), g = rmax(g0, R(0)), b = rmax(b0, R(0));
    return M<R>::fma(r, asym_gauss(lambda, R(615), R(45), R(65)),
                     M<R>::fma(g, asym_gauss(lambda, R(545), R(45), R(45)),
                               b * asym_gauss(lambda, R(465), R(40), R(45))));
}

// env_map.rs:231-239 direction_to_uv
template <class R> static inline void direction_to_uv(const V3<R> &dir, R &u, R &v) {
    const R PI = R(3.14159265358979323846f);
    V3<R> d = dir.normalize_or_zero();
    R theta = M<R>::acos(clampr(d.y, R(-1), R(1)));
    R phi = M<R>::atan2(d.x, d.z);
    v = theta / PI;
    u = rem_euclid(phi / R(2.0f * 3.14159265358979323846f), R(1));
}
// env_map.rs:287-323 sample_bilinear
template <class R> static inline void sample_bilinear(const float *px, uint32_t w, uint32_t h, R u, R v, R out[3]) {
    if (w == 1 && h == 1) { out[0] = px[0]; out[1] = px[1]; out[2] = px[2]; return; }
    R fx = M<R>::fma(rem_euclid(u, R(1)), R((float)w), R(-0.5f));
    R fy = M<R>::fma(clampr(v, R(0), R(1)), R((float)h), R(-0.5f));
    R x0 = M<R>::floor(fx), y0 = M<R>::floor(fy);
    R tx = fx - x0, ty = fy - y0;
    int64_t xi = (int64_t)x0, yi = (int64_t)y0;
    auto wrapx = [&](int64_t x) -> uint32_t { int64_t r = x % (int64_t)w; if (r < 0) r += w; return (uint32_t)r; };
    auto clampy = [&](int64_t y) -> uint32_t { if (y < 0) y = 0; if (y > (int64_t)h - 1) y = h - 1; return (uint32_t)y; };
    uint32_t x0i = wrapx(xi), x1i = wrapx(xi + 1), y0i = clampy(yi), y1i = clampy(yi + 1);
    const float *p00 = px + 3 * ((size_t)y0i * w + x0i), *p10 = px + 3 * ((size_t)y0i * w + x1i);
    const float *p01 = px + 3 * ((size_t)y1i * w + x0i), *p11 = px + 3 * ((size_t)y1i * w + x1i);
    for (int c = 0; c < 3; ++c) {
        R top = M<R>::fma(R(p10[c]), tx, R(p00[c]) * (R(1) - tx));
        R bot = M<R>::fma(R(p11[c]), tx, R(p01[c]) * (R(1) - tx));
        out[c] = M<R>::fma(bot, ty, top * (R(1) - ty));
    }
}

// ---------------------------------------------------------------------------------
// a14. Colour -- color/cie1931.rs:78-98, raytracer/color.rs:122-164,198-315
// ---------------------------------------------------------------------------------
template <class R> static inline R lobe_poly(R l, R mu, R slo, R shi) {
    R sigma = l < mu ? slo : shi;
    R t = (l - mu) / sigma;
    return M<R>::exp_poly(R(-0.5f) * t * t);
}
template <class R> static inline void cmf_x8(const R lam[8], R out[8][3]) {  // cie1931.rs:78-98
    for (int k = 0; k < 8; ++k) {
        R l = lam[k];
        R x0 = lobe_poly(l, R(501.1f), R(20.4f), R(26.2f));
        R x1 = lobe_poly(l, R(599.8f), R(37.9f), R(31.0f));
        R x2 = lobe_poly(l, R(442.0f), R(16.0f), R(26.7f));
        R y0 = lobe_poly(l, R(530.9f), R(16.3f), R(31.1f));
        R y1 = lobe_poly(l, R(568.8f), R(46.9f), R(40.5f));
        R z0 = lobe_poly(l, R(459.0f), R(26.0f), R(13.8f));
        R z1 = lobe_poly(l, R(437.0f), R(11.8f), R(36.0f));
        R x = M<R>::fma(R(0.065f), -x0, M<R>::fma(R(1.056f), x1, R(0.362f) * x2));
        R y = M<R>::fma(R(0.286f), y0, R(0.821f) * y1);
        R z = M<R>::fma(R(0.681f), z0, R(1.217f) * z1);
        out[k][0] = rmax(x, R(0)); out[k][1] = rmax(y, R(0)); out[k][2] = rmax(z, R(0));
    }
}
// Scalar libm CMF (cie1931.rs:13-42), used only by the host white-balance integral.
template <class R> static inline void cmf_scalar(R l, R out[3]) {
    R x = M<R>::fma(R(0.065f), -asym_gauss(l, R(501.1f), R(20.4f), R(26.2f)),
                    M<R>::fma(R(1.056f), asym_gauss(l, R(599.8f), R(37.9f), R(31.0f)),
                              R(0.362f) * asym_gauss(l, R(442.0f), R(16.0f), R(26.7f))));
    R y = M<R>::fma(R(0.286f), asym_gauss(l, R(530.9f), R(16.3f), R(31.1f)),
                    R(0.821f) * asym_gauss(l, R(568.8f), R(46.9f), R(40.5f)));
    R z = M<R>::fma(R(0.681f), asym_gauss(l, R(459.0f), R(26.0f), R(13.8f)),
                    R(1.217f) * asym_gauss(l, R(437.0f), R(11.8f), R(36.0f)));
    out[0] = rmax(x, R(0)); out[1] = rmax(y, R(0)); out[2] = rmax(z, R(0));
}

static const float BRADFORD_XYZ_TO_LMS[3][3] = {{0.8951f, 0.2664f, -0.1614f},
                                                {-0.7502f, 1.7135f, 0.0367f},
                                                {0.0389f, -0.0685f, 1.0296f}};
static const float BRADFORD_LMS_TO_XYZ[3][3] = {{0.986993f, -0.147054f, 0.159963f},
                                                {0.432305f, 0.518360f, 0.049291f},
                                                {-0.008529f, 0.040043f, 0.968487f}};
template <class R> static inline V3<R> mat3_fma(const float m[3][3], const V3<R> &v) {
    return V3<R>(M<R>::fma(R(m[0][0]), v.x, M<R>::fma(R(m[0][1]), v.y, R(m[0][2]) * v.z)),
                 M<R>::fma(R(m[1][0]), v.x, M<R>::fma(R(m[1][1]), v.y, R(m[1][2]) * v.z)),
                 M<R>::fma(R(m[2][0]), v.x, M<R>::fma(R(m[2][1]), v.y, R(m[2][2]) * v.z)));
}
// color.rs:249-251
template <class R> static inline V3<R> apply_von_kries(const V3<R> &xyz, const V3<R> &lms_scale) {
    return mat3_fma(BRADFORD_LMS_TO_XYZ, mat3_fma(BRADFORD_XYZ_TO_LMS, xyz) * lms_scale);
}
// color.rs:281-315 (401-point quadrature, scalar libm CMF)
template <class R> static inline V3<R> compute_illuminant_white_balance(R temp_k) {
    V3<R> w;
    for (int step = 0; step <= 400; ++step) {
        R lambda = R(380) + R(step);
        R c[3];
        cmf_scalar(lambda, c);
        R bb = blackbody_spectrum(lambda, temp_k);
        w = w + V3<R>(c[0], c[1], c[2]) * bb;
    }
    R ty = rmax(w.y, R(1e-6f));
    const float wx = 0.3127f, wy = 0.3290f;
    V3<R> target(R(wx / wy) * ty, ty, R((1.0f - wx - wy) / wy) * ty);
    V3<R> ls = mat3_fma(BRADFORD_XYZ_TO_LMS, w), lt = mat3_fma(BRADFORD_XYZ_TO_LMS, target);
    return V3<R>(ls.x > R(1e-6f) ? lt.x / ls.x : R(1), ls.y > R(1e-6f) ? lt.y / ls.y : R(1),
                 ls.z > R(1e-6f) ? lt.z / ls.z : R(1));
}

// Extension (no reference counterpart): the luminance-weighted Stokes vector of the
// escaping light, sum_k ybar(lambda_k) * ((S_k * env_k) * w) * norm in channel order,
// with the XYZ integral's weight w, normaliser and intensity clamp (stokes_env[k] =
// (fma(I_k clamped, env_k, 0), Q_k * env_k, U_k * env_k, V_k * env_k)), so its I is the
// XYZ integral's Y.
template <class R> static inline void integrate_channels_to_stokes(const R stokes_env[8][4], const R lam[8],
                                                                    const R pdf[8], R out[4]) {
    R sum = R(-0.0);
    for (int k = 0; k < 8; ++k) sum = sum + pdf[k];
    R w = sum <= R(1e-12f) ? R(1) : R(8) * pdf[0] / sum;
    const R norm = R((400.0f / 8.0f) / 106.856f);
    R c[8][3];
    cmf_x8(lam, c);
    for (int j = 0; j < 4; ++j) out[j] = R(0);
    for (int k = 0; k < 8; ++k)
        for (int j = 0; j < 4; ++j) out[j] = out[j] + c[k][1] * ((stokes_env[k][j] * w) * norm);
}

// color.rs:122-131 and 147-164
template <class R> static inline V3<R> integrate_channels_to_xyz(const R rad[8], const R lam[8], const R pdf[8]) {
    R sum = R(-0.0);
    for (int k = 0; k < 8; ++k) sum = sum + pdf[k];
    R w = sum <= R(1e-12f) ? R(1) : R(8) * pdf[0] / sum;
    const R norm = R((400.0f / 8.0f) / 106.856f);
    R c[8][3];
    cmf_x8(lam, c);
    V3<R> xyz;
    for (int k = 0; k < 8; ++k) {
        R wr = rad[k] * w;
        xyz = xyz + V3<R>(c[k][0], c[k][1], c[k][2]) * (wr * norm);
    }
    return xyz;
}

// ---------------------------------------------------------------------------------
// The transport loop -- transport.rs:684-940 and refraction.rs
// ---------------------------------------------------------------------------------
enum Termination : uint32_t { TERM_ESCAPED = 0, TERM_SCATTER_ABSORBED = 1, TERM_RUSSIAN_ROULETTE = 2, TERM_HIT_CAP = 3 };
enum EventKind : uint32_t { EV_TIR = 0, EV_REFLECT = 1, EV_REFRACT = 2, EV_SCATTER = 3 };

// Per-scene environment state prepared once (white balance, studio rig, map).
template <class R> struct EnvCtx {
    uint32_t mode;
    R uniform_rgb[3];
    R temp_k, spot_mult, exposure;
    StudioRig<R> rig;
    const float *map;
    uint32_t mw, mh;
    V3<R> white_balance;
};

template <class R> static inline EnvCtx<R> make_env(const gr_environment &e) {
    EnvCtx<R> c;
    c.mode = e.mode;
    for (int i = 0; i < 3; ++i) c.uniform_rgb[i] = R(e.uniform_rgb[i]);
    c.temp_k = R(e.temp_k); c.spot_mult = R(e.spot_mult); c.exposure = R(e.exposure);
    c.map = e.latlong_rgb; c.mw = e.latlong_w; c.mh = e.latlong_h;
    if (e.mode == GR_ENV_STUDIO) {
        c.rig = studio_rig_new(R(e.light_yaw), R(e.light_pitch));
        c.white_balance = compute_illuminant_white_balance(R(e.temp_k));  // environment.rs:238-243
    } else {
        c.white_balance = V3<R>(1, 1, 1);
    }
    return c;
}

// environment.rs:209-225 (+ env_map.rs:241-250 for the map variants)
template <class R> static inline R env_channel(const EnvCtx<R> &env, const V3<R> &dir, R lambda) {
    if (env.mode == GR_ENV_STUDIO)
        return studio_radiance(dir, lambda, env.temp_k, env.spot_mult, env.exposure, env.rig);
    R rgb[3];
    if (env.mode == GR_ENV_UNIFORM) {
        rgb[0] = env.uniform_rgb[0]; rgb[1] = env.uniform_rgb[1]; rgb[2] = env.uniform_rgb[2];
    } else {
        R u, v;
        direction_to_uv(dir, u, v);
        sample_bilinear(env.map, env.mw, env.mh, u, v, rgb);
    }
    return rgb_to_spectral(rgb[0], rgb[1], rgb[2], lambda);
}

template <class R> struct MaterialCtx {
    const gr_material *mat;
    const gr_material_ext *ext;
    bool anisotropic;
    bool biaxial;  // biaxial_delta_beta_alpha.is_some() (refraction.rs:459)
    V3<R> c_axis;
    R bire;
    R d_beta_alpha;
};

template <class R> static inline MaterialCtx<R> make_material(const gr_material *m, const gr_material_ext *ext) {
    MaterialCtx<R> c;
    c.mat = m;
    c.ext = ext;
    c.c_axis = V3<R>(R(m->dispersion.c_axis_and_birefringence[0]), R(m->dispersion.c_axis_and_birefringence[1]),
                     R(m->dispersion.c_axis_and_birefringence[2]));
    c.bire = R(m->dispersion.c_axis_and_birefringence[3]);
    c.biaxial = m->dispersion.has_biaxial_delta != 0;
    c.d_beta_alpha = R(m->dispersion.biaxial_delta_beta_alpha);
    // transport.rs:620-621
    c.anisotropic = m->crystal_system != GR_CRYSTAL_CUBIC && std::fabs(m->dispersion.c_axis_and_birefringence[3]) > 1e-4f;
    return c;
}

// Every material kind of the reference's render path is handled (isotropic, uniaxial,
// biaxial with or without a beta-ray band set; polished or frosted facets; volume
// scattering); the decline status stays for malformed materials only
// (renderer/gpu/frame.rs:680-693, GemMaterial::gpu_supported).
static inline bool material_supported(const gr_material *m, const uint32_t *finishes, uint32_t n_planes) {
    (void)finishes;
    (void)n_planes;
    return m->o_ray_band_count <= GR_MAX_BANDS && m->e_ray_band_count <= GR_MAX_BANDS &&
           m->beta_ray_band_count <= GR_MAX_BANDS;
}

// Per-sample wavelength cache (build_ray_wavelength_cache, refraction.rs:127-174).
template <class R> struct WaveCache {
    R n_o[8];
    R n_e_delta[8];  // n_e - n_o per channel (constant birefringence_delta unless extended)
    Tensor3<R> tensor[8];
    Indicatrix<R> ind[8];  // biaxial materials: per-channel indicatrix (hero = channel 0)
    bool any_absorption;
};

template <class R>
static inline WaveCache<R> build_cache(const MaterialCtx<R> &mc, const R lam[8]) {
    WaveCache<R> wc;
    const gr_material *m = mc.mat;
    wc.any_absorption = false;
    for (int k = 0; k < 8; ++k) {
        wc.n_o[k] = dispersion_evaluate(m->dispersion, lam[k]);
        if (mc.ext && mc.ext->has_cauchy_e) {
            R lum = lam[k] * R(1e-3f);
            R l2 = lum * lum, l4 = l2 * l2;
            R n_e = R(mc.ext->cauchy_e[0]) + R(mc.ext->cauchy_e[1]) / l2 + R(mc.ext->cauchy_e[2]) / l4;
            wc.n_e_delta[k] = n_e - wc.n_o[k];
        } else {
            wc.n_e_delta[k] = mc.bire;
        }
        R ao, ae;
        if (mc.ext && mc.ext->n_absorption > 0) {
            ao = table_lookup(mc.ext->alpha_o_table, mc.ext->n_absorption, mc.ext->absorption_nm_first,
                              mc.ext->absorption_nm_step, lam[k]);
            ae = table_lookup(mc.ext->alpha_e_table, mc.ext->n_absorption, mc.ext->absorption_nm_first,
                              mc.ext->absorption_nm_step, lam[k]);
        } else {
            ao = spectral_absorption(m->o_ray_bands, m->o_ray_band_count, lam[k]);
            ae = spectral_absorption(m->e_ray_bands, m->e_ray_band_count, lam[k]);
        }
        if (ao != R(0) || ae != R(0)) wc.any_absorption = true;
        wc.tensor[k] = tensor_uniaxial(ao, ae, mc.c_axis);
        if (mc.biaxial) {
            wc.ind[k] = make_indicatrix(wc.n_o[k], mc.d_beta_alpha, mc.bire, mc.c_axis);
            // AbsorptionTensor3::biaxial(alpha_o, beta, alpha_e, c) (birefringence.rs:238-245):
            // the uniaxial frame with the beta band set's coefficient on the second axis
            if (m->has_beta_ray) {
                const R ab = spectral_absorption(m->beta_ray_bands, m->beta_ray_band_count, lam[k]);
                wc.tensor[k].alpha = V3<R>(ao, ab, ae);
                if (ab != R(0)) wc.any_absorption = true;
            }
        }
    }
    return wc;
}

// signed_frame_rotation_psi (raytracer/absorption.rs:44-54): the signed angle from the
// previous plane-of-incidence normal to the current one about the wave normal.
template <class R> static inline R signed_frame_rotation_psi(const V3<R> &prev, const V3<R> &cur, const V3<R> &k) {
    R cos_psi = clampr(prev.dot(cur), R(-1), R(1));
    R sin_psi = prev.cross(cur).dot(k.normalize_or_zero());
    return M<R>::atan2(sin_psi, cos_psi);
}

// theta_c_for_bounce (refraction.rs:235-273): the angle between the c-axis and the
// wave normal the extraordinary index is taken at -- on entry (outside, uniaxial) the
// refracted wave normal after a two-step fixed point, otherwise the ray's own.
template <class R>
static inline R theta_c_for_bounce(const V3<R> &k_hat, const V3<R> &normal, R cos_i, R n_o_seed, R n_e_seed,
                                   const V3<R> &c_axis, bool entry) {
    R theta;
    if (entry) {
        R n_guess = n_o_seed;
        theta = R(0);
        for (int it = 0; it < 2; ++it) {
            R eta = R(1) / n_guess;
            R s2 = eta * eta * M<R>::fma(cos_i, -cos_i, R(1));
            if (s2 > R(1)) break;
            R ct = M<R>::sqrt(rmax(R(1) - s2, R(0)));
            V3<R> wd = (eta * k_hat + M<R>::fma(eta, cos_i, -ct) * normal).normalize();
            R ctw = std::fabs(clampr(wd.dot(c_axis), R(-1), R(1)));
            theta = M<R>::acos(ctw);
            n_guess = effective_extraordinary_index(n_o_seed, n_e_seed, theta);
        }
    } else {
        theta = M<R>::acos(std::fabs(clampr(k_hat.dot(c_axis), R(-1), R(1))));
    }
    return theta;
}

// refraction.rs:46-50
template <class R> static inline R tir_phase_delta(R n1k, R cos_i, R sin_i) {
    R num = cos_i * M<R>::sqrt(rmax(M<R>::fma(n1k * n1k * sin_i, sin_i, R(-1)), R(0)));
    R den = rmax(n1k * sin_i * sin_i, R(1e-6f));
    return R(2) * M<R>::atan(num / den);
}

template <class R> struct Geo {
    R cos_i, sin_i, n_o_hero, n_e_hero, n1, n2, sin2_t;
    R n_o_ch[8], n1_ch[8], n2_ch[8], sin2_t_ch[8];
    R n_biax_a_ch[8];  // biaxial: fast-mode index per channel at the hero's fast wave normal
};

// compute_bounce_refraction_geometry (refraction.rs:428-547)
template <class R>
static inline Geo<R> bounce_geometry(const MaterialCtx<R> &mc, const WaveCache<R> &wc, const V3<R> &normal,
                                     const V3<R> &k_hat, bool inside, bool is_e) {
    Geo<R> g;
    g.cos_i = clampr((-k_hat).dot(normal), R(0), R(1));
    g.sin_i = M<R>::sqrt(rmax(M<R>::fma(g.cos_i, -g.cos_i, R(1)), R(0)));
    R n_o_seed = wc.n_o[0];
    const R theta = theta_c_for_bounce(k_hat, normal, g.cos_i, n_o_seed, n_o_seed + wc.n_e_delta[0], mc.c_axis,
                                       !inside && mc.anisotropic && !mc.biaxial);
    R n_eff[8];
    for (int k = 0; k < 8; ++k) {
        R n_o_k = wc.n_o[k];
        R n_e_k = n_o_k + wc.n_e_delta[k];
        n_eff[k] = mc.anisotropic ? effective_extraordinary_index(n_o_k, n_e_k, theta) : n_o_k;
        g.n_o_ch[k] = n_o_k;
    }
    g.n_o_hero = wc.n_o[0];
    g.n_e_hero = g.n_o_hero + wc.n_e_delta[0];
    // hero_biaxial_wave_dirs + per_channel_biaxial_indices (refraction.rs:345-401): mode
    // A (fast) and mode B (slow) indices at the hero's two wave normals -- the ray's own
    // inside the stone, the refracted ones (resolve_entry_mode) on entry
    R n_biax_b[8];
    if (mc.biaxial) {
        V3<R> dir_a = k_hat, dir_b = k_hat;
        if (!inside) {
            dir_a = resolve_entry_mode(wc.ind[0], k_hat, normal, g.cos_i, n_o_seed, false);
            dir_b = resolve_entry_mode(wc.ind[0], k_hat, normal, g.cos_i, n_o_seed, true);
        }
        for (int k = 0; k < 8; ++k) {
            R ns, nf;
            wave_indices(wc.ind[k], dir_a, ns, nf);
            g.n_biax_a_ch[k] = nf;
            wave_indices(wc.ind[k], dir_b, ns, nf);
            n_biax_b[k] = ns;
        }
    } else {
        for (int k = 0; k < 8; ++k) { g.n_biax_a_ch[k] = R(0); n_biax_b[k] = R(0); }
    }
    const R *mode_a = mc.biaxial ? g.n_biax_a_ch : g.n_o_ch;
    const R *mode_b = mc.biaxial ? n_biax_b : n_eff;
    const R *n_med = (mc.anisotropic && inside && !is_e) ? mode_a : mode_b;
    R n_med_hero = n_med[0];
    g.n1 = inside ? n_med_hero : R(1);
    g.n2 = inside ? R(1) : n_med_hero;
    R eta = g.n1 / g.n2;
    g.sin2_t = eta * eta * M<R>::fma(g.cos_i, -g.cos_i, R(1));
    for (int k = 0; k < 8; ++k) {
        R n1k = inside ? n_med[k] : R(1);
        R n2k = inside ? R(1) : n_med[k];
        R etak = n1k / n2k;
        g.n1_ch[k] = n1k;
        g.n2_ch[k] = n2k;
        g.sin2_t_ch[k] = etak * etak * M<R>::fma(g.cos_i, -g.cos_i, R(1));
    }
    return g;
}

// poynting_dir_for_mode (refraction.rs:564-582): biaxial modes both walk off
template <class R>
static inline V3<R> poynting_dir_for_mode(const MaterialCtx<R> &mc, const WaveCache<R> &wc, const Geo<R> &g,
                                          const V3<R> &k, bool inside, bool is_e) {
    if (!inside || !mc.anisotropic) return k;
    if (mc.biaxial) return mode_poynting_dir(wc.ind[0], k, is_e);
    if (is_e) return extraordinary_poynting_dir(k, mc.c_axis, g.n_o_hero, g.n_e_hero);
    return k;
}

// channel_absorption_alphas' eigenmode pair (raytracer/absorption.rs:175-196): the hero
// indicatrix's (slow, fast) D directions for a biaxial material, else the uniaxial
// ordinary / extraordinary pair
template <class R>
static inline void absorption_eigenmodes(const MaterialCtx<R> &mc, const WaveCache<R> &wc, const V3<R> &k, V3<R> &ea,
                                         V3<R> &eb) {
    if (mc.biaxial) {
        eigen_polarizations(wc.ind[0], k, ea, eb);
    } else {
        ea = ordinary_eigen_polarization(k, mc.c_axis);
        eb = extraordinary_eigen_polarization(k, mc.c_axis);
    }
}

template <class R> static inline void fresnel_rs_rp(R n1k, R n2k, R cos_i, R cos_t, R &rs, R &rp) {
    rs = M<R>::fma(n2k, -cos_t, n1k * cos_i) / M<R>::fma(n2k, cos_t, n1k * cos_i);
    rp = M<R>::fma(n1k, -cos_t, n2k * cos_i) / M<R>::fma(n1k, cos_t, n2k * cos_i);
}
template <class R> static inline R r_unpol_clamped(R rs, R rp) {
    return clampr(R(0.5f) * M<R>::fma(rp, rp, rs * rs), R(1e-4f), R(1) - R(1e-4f));
}

// ---------------------------------------------------------------------------------
// Frosted facets and Henyey-Greenstein volume scattering -- raytracer/scattering.rs
// ---------------------------------------------------------------------------------
template <class R> static inline void frosted_orthonormal_basis(const V3<R> &n, V3<R> &t, V3<R> &b) {  // :337-342
    V3<R> a = std::fabs(n.x) > R(0.9f) ? V3<R>(R(0), R(1), R(0)) : V3<R>(R(1), R(0), R(0));
    t = (a - n * n.dot(a)).normalize_or_zero();
    b = n.cross(t);
}

template <class R> static inline V3<R> cosine_weighted_hemisphere(R u1, R u2, const V3<R> &n) {  // :356-362
    const R r = M<R>::sqrt(u1);
    const R theta = R(2.0f * 3.14159265358979323846f) * u2;
    const R sin_t = M<R>::sin(theta), cos_t = M<R>::cos(theta);
    V3<R> t, b;
    frosted_orthonormal_basis(n, t, b);
    return (t * (r * cos_t) + b * (r * sin_t) + n * M<R>::sqrt(rmax(R(1) - u1, R(0)))).normalize_or_zero();
}

template <class R> static inline V3<R> sample_hg_direction(R u1, R u2, R g, const V3<R> &fwd) {  // :428-443
    R cos_theta;
    if (std::fabs(g) < R(1e-3f)) {
        cos_theta = M<R>::fma(R(2), -u1, R(1));
    } else {
        const R one_minus_g2 = M<R>::fma(g, -g, R(1));
        const R denom = M<R>::fma(R(2) * g, u1, R(1) - g);
        const R sq = one_minus_g2 / denom;
        cos_theta = M<R>::fma(sq, -sq, M<R>::fma(g, g, R(1))) / (R(2) * g);
    }
    cos_theta = clampr(cos_theta, R(-1), R(1));
    const R sin_theta = M<R>::sqrt(rmax(M<R>::fma(cos_theta, -cos_theta, R(1)), R(0)));
    const R phi = R(2.0f * 3.14159265358979323846f) * u2;
    const R sin_p = M<R>::sin(phi), cos_p = M<R>::cos(phi);
    V3<R> t, b;
    frosted_orthonormal_basis(fwd, t, b);
    return (t * (sin_theta * cos_p) + b * (sin_theta * sin_p) + fwd * cos_theta).normalize_or_zero();
}

// Optional per-bounce event record (extends trace_spectral_ray_with_finish_instrumented,
// transport.rs:512-537).
struct EventLog {
    uint32_t bounces;
    uint32_t termination;
    uint32_t n_tir, n_reflect, n_refract, n_inside_abs, n_escape;
    uint32_t n_chan_tir;  // per-channel TIR-phase evaluations
    uint32_t n_scatter;   // Henyey-Greenstein volume events
    int32_t facets[64];
    uint8_t events[64];
    float ts[64];  // hit distance of each logged bounce (the tie rule's t)
};

struct TraceOpts {
    uint32_t max_bounces;
    bool internal_mode_coupling;
};

// transport.rs:684-940 for one sample.  Returns XYZ after white balance.
template <class R>
static inline V3<R> trace_spectral_ray(const Ray<float> &initial, const gr_plane *planes, uint32_t n_planes,
                                       const MaterialCtx<R> &mc, const EnvCtx<R> &env, uint32_t max_bounces,
                                       uint32_t rng_seed, float hero_rand, EventLog *log,
                                       const uint32_t *finishes = nullptr, R *stokes_out = nullptr) {
    R lam[8];
    wrapped_hero_wavelengths<R>(hero_rand, lam);
    Stokes<R> st[8];
    R rad[8], pdf[8], stokes_env[8][4];
    for (int k = 0; k < 8; ++k) {
        st[k] = Stokes<R>{R(1), R(0), R(0), R(0)}; rad[k] = R(0); pdf[k] = R(1);
        for (int j = 0; j < 4; ++j) stokes_env[k][j] = R(0);
    }
    Ray<R> ray;
    ray.origin = V3<R>(initial.origin.x, initial.origin.y, initial.origin.z);
    ray.dir = V3<R>(initial.dir.x, initial.dir.y, initial.dir.z);
    V3<R> cur_k = ray.dir;
    bool inside = false, have_prev = false, is_e = false;
    V3<R> prev_plane;
    WaveCache<R> wc = build_cache(mc, lam);
    const gr_material *mat = mc.mat;
    if (log) { log->bounces = max_bounces; log->termination = TERM_HIT_CAP; }

    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        Hit<R> hit = intersect_polyhedron(ray, planes, n_planes);
        if (!hit.hit) {
            // accumulate_miss_radiance (transport.rs:67-90)
            for (int k = 0; k < 8; ++k) {
                R e = env_channel(env, ray.dir, lam[k]);
                rad[k] = M<R>::fma(st[k].intensity(), e, rad[k]);
                stokes_env[k][0] = rad[k];
                stokes_env[k][1] = st[k].q * e;
                stokes_env[k][2] = st[k].u * e;
                stokes_env[k][3] = st[k].v * e;
            }
            if (log) { log->bounces = bounce; log->termination = TERM_ESCAPED; log->n_escape++; }
            break;
        }
        if (log && bounce < 64) { log->facets[bounce] = hit.facet; log->ts[bounce] = (float)hit.t; }
        // try_scatter_step (raytracer/scattering.rs:246-315, maybe_scatter_or_extinguish
        // :132-212): a Henyey-Greenstein event somewhere along this interior segment,
        // drawn before the facet is processed; on no event, the segment's extinction
        // (which then replaces apply_absorption below).
        if (inside && mat->scattering_sigma_s > 0.0f) {
            const V3<R> s_axis = have_prev ? prev_plane : V3<R>();
            V3<R> ea, eb;
            absorption_eigenmodes(mc, wc, cur_k, ea, eb);
            R alphas[8];
            for (int k = 0; k < 8; ++k) {
                V3<R> e_hat = electric_field_direction(st[k], s_axis, cur_k);
                alphas[k] = effective_pleochroic_alpha(wc.tensor[k], e_hat, ea, eb, st[k].degree_of_polarization());
            }
            const R sigma_s = R(mat->scattering_sigma_s);
            const R sigma_t_hero = alphas[0] + sigma_s;  // the hero is channel 0
            const R dist_rand = R(rng_draw(rng_seed, bounce, DISTANCE_SAMPLE_STREAM));
            const R omu = rmax(R(1) - dist_rand, R(1e-7f));
            const R t_free = -(M<R>::log(omu)) / sigma_t_hero;
            const R hit_scaled = hit.t * R(mat->absorption_path_scale);
            if (t_free < hit_scaled) {
                const R pdf_hero = sigma_t_hero * omu;
                for (int k = 0; k < 8; ++k) {
                    const R sigma_t_k = alphas[k] + sigma_s;
                    const R tr = M<R>::exp_poly(-(alphas[k] + sigma_s) * t_free);
                    const R w = tr * sigma_s / pdf_hero;
                    st[k] = Stokes<R>{st[k].intensity() * w, R(0), R(0), R(0)};
                    pdf[k] = pdf[k] * (sigma_t_k * tr);
                }
                const R u1 = R(rng_draw(rng_seed, bounce, PHASE_DIR_U_STREAM));
                const R u2 = R(rng_draw(rng_seed, bounce, PHASE_DIR_V_STREAM));
                const V3<R> new_dir = sample_hg_direction(u1, u2, R(mat->scattering_g), ray.dir);
                ray.origin = ray.origin + (t_free / R(mat->absorption_path_scale)) * ray.dir;
                ray.dir = new_dir;
                cur_k = new_dir;
                have_prev = false;  // depolarized: no previous plane of incidence
                if (log) { log->n_scatter++; if (bounce < 64) log->events[bounce] = EV_SCATTER; }
                if (bounce > 4) {   // apply_russian_roulette (transport.rs:204-220)
                    R mx = R(0);
                    for (int k = 0; k < 8; ++k) mx = rmax(mx, st[k].intensity());
                    R q = clampr(mx, R(0.05f), R(1));
                    R rr = R(rng_draw(rng_seed, bounce, RUSSIAN_ROULETTE_STREAM));
                    if (rr > q) {
                        if (log) { log->bounces = bounce; log->termination = TERM_RUSSIAN_ROULETTE; }
                        break;
                    }
                    for (int k = 0; k < 8; ++k) st[k] = st[k].scale(R(1) / q);
                }
                continue;
            }
            R sv[8];
            for (int k = 0; k < 8; ++k) sv[k] = M<R>::exp_poly(-(alphas[k] + sigma_s) * hit_scaled);
            const R sh = rmax(sv[0], R(1e-30f));
            for (int k = 0; k < 8; ++k) {
                st[k] = st[k].scale(sv[k] / sh);
                pdf[k] = pdf[k] * sv[k];
            }
        }
        V3<R> hp = ray.origin + hit.t * ray.dir;
        V3<R> normal = shading_normal_near_edge(planes, n_planes, hp, hit.facet, hit.normal, R(mat->edge_rounding_radius));

        // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:71-89)
        V3<R> cur_plane = cur_k.cross(normal).normalize_or_zero();
        if (have_prev && cur_plane.length_squared() > R(1e-6f) && prev_plane.length_squared() > R(1e-6f)) {
            R psi = signed_frame_rotation_psi(prev_plane, cur_plane, cur_k);
            Mat4<R> rot = frame_rotation(psi);
            for (int k = 0; k < 8; ++k) st[k] = apply_matrix(st[k], rot);
        }
        prev_plane = cur_plane;
        have_prev = true;

        // apply_interior_segment (transport.rs:586-605) -> apply_absorption (absorption.rs:115-141)
        if (inside) {
            normal = -normal;
            if (mat->scattering_sigma_s <= 0.0f) {
                V3<R> ea, eb;
                absorption_eigenmodes(mc, wc, cur_k, ea, eb);
                R scaled = hit.t * R(mat->absorption_path_scale);
                R alphas[8];
                for (int k = 0; k < 8; ++k) {
                    V3<R> e_hat = electric_field_direction(st[k], cur_plane, cur_k);
                    alphas[k] = effective_pleochroic_alpha(wc.tensor[k], e_hat, ea, eb, st[k].degree_of_polarization());
                }
                for (int k = 0; k < 8; ++k) {
                    R arg = -alphas[k] * scaled;
                    st[k] = st[k].scale(M<R>::exp_poly(arg));
                }
                if (log) log->n_inside_abs++;
            }
        }

        Geo<R> g = bounce_geometry(mc, wc, normal, cur_k, inside, is_e);

        // dispatch_bounce (transport.rs:128-193)
        V3<R> new_k, new_s;
        bool new_inside = inside;
        bool has_update = false, update_val = false;
        if (finishes && finishes[hit.facet] != 0) {
            // apply_frosted_bounce (raytracer/scattering.rs:522-602): a Lambertian lobe
            // on either side, depolarizing, no pdf division on the forced (TIR) branch
            const R u1 = R(rng_draw(rng_seed, bounce, FROSTED_DIR_U_STREAM));
            const R u2 = R(rng_draw(rng_seed, bounce, FROSTED_DIR_V_STREAM));
            V3<R> nd;
            if (g.sin2_t > R(1)) {
                nd = cosine_weighted_hemisphere(u1, u2, normal);
                for (int k = 0; k < 8; ++k) st[k] = Stokes<R>{st[k].intensity(), R(0), R(0), R(0)};
                if (log) { log->n_tir++; if (bounce < 64) log->events[bounce] = EV_TIR; }
            } else {
                const R ct = M<R>::sqrt(rmax(R(1) - g.sin2_t, R(0)));
                const R r_s = M<R>::fma(g.n2, -ct, g.n1 * g.cos_i) / M<R>::fma(g.n2, ct, g.n1 * g.cos_i);
                const R r_p = M<R>::fma(g.n1, -ct, g.n2 * g.cos_i) / M<R>::fma(g.n1, ct, g.n2 * g.cos_i);
                const R ru = clampr(R(0.5f) * M<R>::fma(r_p, r_p, r_s * r_s), R(1e-4f), R(1) - R(1e-4f));
                const R rng_b = R(rng_draw(rng_seed, bounce, FRESNEL_BRANCH_STREAM));
                if (rng_b < ru) {
                    nd = cosine_weighted_hemisphere(u1, u2, normal);
                    for (int k = 0; k < 8; ++k) {
                        st[k] = Stokes<R>{st[k].intensity() / ru, R(0), R(0), R(0)};
                        pdf[k] = pdf[k] * ru;
                    }
                    if (log) { log->n_reflect++; if (bounce < 64) log->events[bounce] = EV_REFLECT; }
                } else {
                    nd = cosine_weighted_hemisphere(u1, u2, -normal);
                    const bool entering_aniso = !inside && mc.anisotropic;
                    const bool use_e = entering_aniso ? rng_draw(rng_seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f : is_e;
                    const R tu = R(1) - ru;
                    for (int k = 0; k < 8; ++k) {
                        st[k] = Stokes<R>{st[k].intensity() / tu, R(0), R(0), R(0)};
                        pdf[k] = pdf[k] * tu;
                    }
                    new_inside = !inside;
                    if (entering_aniso) { has_update = true; update_val = use_e; }
                    if (log) { log->n_refract++; if (bounce < 64) log->events[bounce] = EV_REFRACT; }
                }
            }
            new_k = nd;
            new_s = nd;
        } else if (g.sin2_t > R(1)) {
            // apply_tir_bounce (refraction.rs:599-637)
            for (int k = 0; k < 8; ++k) {
                R n1k = g.n1_ch[k], n2k = g.n2_ch[k];
                if (g.sin2_t_ch[k] > R(1)) {
                    R dk = tir_phase_delta(n1k, g.cos_i, g.sin_i);
                    st[k] = apply_matrix(st[k], tir_retardation(dk));
                    if (log) log->n_chan_tir++;
                } else {
                    R ct = M<R>::sqrt(rmax(R(1) - g.sin2_t_ch[k], R(0)));
                    R rs, rp;
                    fresnel_rs_rp(n1k, n2k, g.cos_i, ct, rs, rp);
                    st[k] = apply_matrix(st[k], fresnel_reflection(rs, rp));
                    pdf[k] = pdf[k] * r_unpol_clamped(rs, rp);
                }
            }
            new_k = cur_k - (R(2) * cur_k.dot(normal)) * normal;
            new_s = poynting_dir_for_mode(mc, wc, g, new_k, inside, is_e);
            if (log) { log->n_tir++; if (bounce < 64) log->events[bounce] = EV_TIR; }
        } else {
            // apply_partial_fresnel_bounce (refraction.rs:1036-1086)
            R cos_t = M<R>::sqrt(R(1) - g.sin2_t);
            R rs, rp;
            fresnel_rs_rp(g.n1, g.n2, g.cos_i, cos_t, rs, rp);
            R r_unpol = r_unpol_clamped(rs, rp);
            R rng_b = R(rng_draw(rng_seed, bounce, FRESNEL_BRANCH_STREAM));
            if (rng_b < r_unpol) {
                // apply_partial_reflect_bounce (refraction.rs:650-690)
                for (int k = 0; k < 8; ++k) {
                    R n1k = g.n1_ch[k], n2k = g.n2_ch[k];
                    Mat4<R> mm;
                    if (g.sin2_t_ch[k] > R(1)) {
                        mm = tir_retardation(tir_phase_delta(n1k, g.cos_i, g.sin_i));
                        if (log) log->n_chan_tir++;
                    } else {
                        R ct = M<R>::sqrt(rmax(R(1) - g.sin2_t_ch[k], R(0)));
                        R rsk, rpk;
                        fresnel_rs_rp(n1k, n2k, g.cos_i, ct, rsk, rpk);
                        pdf[k] = pdf[k] * r_unpol_clamped(rsk, rpk);
                        mm = fresnel_reflection(rsk, rpk);
                    }
                    st[k] = apply_matrix(st[k], mm).scale(R(1) / r_unpol);
                }
                new_k = cur_k - (R(2) * cur_k.dot(normal)) * normal;
                new_s = poynting_dir_for_mode(mc, wc, g, new_k, inside, is_e);
                if (log) { log->n_reflect++; if (bounce < 64) log->events[bounce] = EV_REFLECT; }
            } else {
                // apply_refract_bounce (refraction.rs:748-867)
                bool entering_aniso = !inside && mc.anisotropic;
                bool use_e = is_e;
                if (entering_aniso) use_e = rng_draw(rng_seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f;
                // biaxial entry: the selected mode's hero index, both modes walk off
                const bool biax_entry = entering_aniso && mc.biaxial;
                R n2_dir;
                if (biax_entry) n2_dir = use_e ? g.n2 : g.n_biax_a_ch[0];
                else n2_dir = (entering_aniso && !use_e) ? g.n_o_hero : g.n2;
                R eta_dir = g.n1 / n2_dir;
                R s2d = rmin(eta_dir * eta_dir * M<R>::fma(g.cos_i, -g.cos_i, R(1)), R(1));
                R ctd = M<R>::sqrt(rmax(R(1) - s2d, R(0)));
                V3<R> refr = (eta_dir * cur_k + M<R>::fma(eta_dir, g.cos_i, -ctd) * normal).normalize();
                V3<R> final_dir;
                if (biax_entry) final_dir = mode_poynting_dir(wc.ind[0], refr, use_e);
                else final_dir = (entering_aniso && use_e)
                                     ? extraordinary_poynting_dir(refr, mc.c_axis, g.n_o_hero, g.n_e_hero)
                                     : refr;
                // apply_refract_channel (refraction.rs:883-1011)
                const R TOL = R(1) - R(1e-6f);
                for (int k = 0; k < 8; ++k) {
                    R n1k = g.n1_ch[k];
                    R n2k = (entering_aniso && !use_e) ? (mc.biaxial ? g.n_biax_a_ch[k] : g.n_o_ch[k]) : g.n2_ch[k];
                    R ratio = n1k / n2k;
                    R s2k = (ratio * ratio) * M<R>::fma(g.cos_i, -g.cos_i, R(1));
                    if (s2k > R(1)) { st[k] = st[k].scale(R(0)); pdf[k] = R(0); continue; }
                    R ctk = M<R>::sqrt(rmax(R(1) - s2k, R(0)));
                    R eta_k = n1k / n2k;
                    V3<R> rk = (eta_k * cur_k + M<R>::fma(eta_k, g.cos_i, -ctk) * normal).normalize();
                    V3<R> fk = rk;
                    if (biax_entry) {
                        fk = mode_poynting_dir(wc.ind[k], rk, use_e);
                    } else if (entering_aniso && use_e) {
                        R n_e_k = g.n_o_ch[k] + wc.n_e_delta[k];
                        fk = extraordinary_poynting_dir(rk, mc.c_axis, g.n_o_ch[k], n_e_k);
                    }
                    if (fk.dot(final_dir) >= TOL) {
                        R ts = (R(2) * n1k * g.cos_i) / M<R>::fma(n2k, ctk, n1k * g.cos_i);
                        R tp = (R(2) * n1k * g.cos_i) / M<R>::fma(n1k, ctk, n2k * g.cos_i);
                        Mat4<R> tm = fresnel_transmission(n1k, n2k, g.cos_i, ctk, ts, tp);
                        st[k] = apply_matrix(st[k], tm).scale(R(1) / (R(1) - r_unpol));
                        R rsk, rpk;
                        fresnel_rs_rp(n1k, n2k, g.cos_i, ctk, rsk, rpk);
                        pdf[k] = pdf[k] * (R(1) - r_unpol_clamped(rsk, rpk));
                    } else {
                        st[k] = st[k].scale(R(0));
                        pdf[k] = R(0);
                    }
                }
                new_k = refr;
                new_s = final_dir;
                new_inside = !inside;
                if (entering_aniso) { has_update = true; update_val = use_e; }
                if (log) { log->n_refract++; if (bounce < 64) log->events[bounce] = EV_REFRACT; }
            }
        }
        bool was_internal_reflection = inside && !has_update && new_inside == inside;
        ray.dir = new_s;
        ray.origin = hp + new_s * R(1e-4f);
        cur_k = new_k;
        inside = new_inside;
        if (has_update) is_e = update_val;
        // maybe_apply_internal_mode_coupling (transport.rs:343-353)
        if (mc.anisotropic && was_internal_reflection)
            is_e = rng_draw(rng_seed, bounce, MODE_COUPLING_STREAM) < 0.5f;

        // apply_russian_roulette (transport.rs:204-220)
        if (bounce > 4) {
            R mx = R(0);
            for (int k = 0; k < 8; ++k) mx = rmax(mx, st[k].intensity());
            R q = clampr(mx, R(0.05f), R(1));
            R rr = R(rng_draw(rng_seed, bounce, RUSSIAN_ROULETTE_STREAM));
            if (rr > q) {
                if (log) { log->bounces = bounce; log->termination = TERM_RUSSIAN_ROULETTE; }
                break;
            }
            for (int k = 0; k < 8; ++k) st[k] = st[k].scale(R(1) / q);
        }
    }
    V3<R> xyz = integrate_channels_to_xyz(rad, lam, pdf);
    if (stokes_out) integrate_channels_to_stokes(stokes_env, lam, pdf, stokes_out);
    return apply_von_kries(xyz, env.white_balance);
}

// ---------------------------------------------------------------------------------
// a16. Tone map -- renderer/tonemap.rs:52-108, color/space.rs:20-30,256-334,
//      color/gamut.rs:38-118, optics/raytracer/color.rs:365-417 (FP32)
// ---------------------------------------------------------------------------------
static const float SRGB_FROM_XYZ[3][3] = {{3.2404542f, -1.5371385f, -0.4985314f},
                                          {-0.969266f, 1.8760108f, 0.0415560f},
                                          {0.0556434f, -0.2040259f, 1.0572252f}};
static inline bool srgb_in_range(const V3<float> &v, float mx) {
    return v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f && v.x <= mx && v.y <= mx && v.z <= mx;
}
static inline V3<float> project_to_gamut_bounded(const V3<float> &xyz, float mx) {
    float sum = xyz.x + xyz.y + xyz.z;
    if (!std::isfinite(sum) || sum <= 1e-6f) return V3<float>();
    float x = xyz.x / sum, y = xyz.y / sum;
    float lum = rmax(xyz.y, 0.0f);
    V3<float> lin = mat3_fma(SRGB_FROM_XYZ, xyz);
    if (srgb_in_range(lin, mx)) return lin;
    const float wx = 0.3127f, wy = 0.3290f;
    auto mapped = [&](float t) {
        float xp = ::fmaf(wx - x, t, x), yp = ::fmaf(wy - y, t, y);
        if (yp > 1e-6f) return V3<float>((xp / yp) * lum, lum, ((1.0f - xp - yp) / yp) * lum);
        return V3<float>((wx / wy) * lum, lum, ((1.0f - wx - wy) / wy) * lum);
    };
    V3<float> r = mat3_fma(SRGB_FROM_XYZ, mapped(1.0f));
    V3<float> resolved(rmax(r.x, 0.0f), rmax(r.y, 0.0f), rmax(r.z, 0.0f));
    for (uint32_t i = 0; i <= 32; ++i) {
        float t = (float)i / 32.0f;
        V3<float> c = mat3_fma(SRGB_FROM_XYZ, mapped(t));
        if (srgb_in_range(c, mx)) { resolved = c; break; }
    }
    return resolved;
}
static inline float aces_tonemap(float y) {
    return (y * ::fmaf(2.51f, y, 0.03f)) / ::fmaf(y, ::fmaf(2.43f, y, 0.59f), 0.14f);
}
static inline uint8_t encode_channel(float c) {
    float lin = std::isfinite(c) ? clampr(c, 0.0f, 1.0f) : 0.0f;
    float enc = lin <= 0.0031308f ? lin * 12.92f : ::fmaf(1.055f, ::powf(lin, 1.0f / 2.4f), -0.055f);
    enc = clampr(enc, 0.0f, 1.0f);
    float v = enc * 255.0f;
    return (uint8_t)(v >= 255.0f ? 255 : (v > 0.0f ? (int)v : 0));
}
static inline void srgb_encode(const V3<float> &xyz, uint8_t out[4]) {
    out[0] = out[1] = out[2] = 0; out[3] = 255;
    float sum = xyz.x + xyz.y + xyz.z;
    if (!std::isfinite(sum) || sum <= 1e-6f) return;
    float lum = rmax(xyz.y, 0.0f);
    float el = rmax(lum * 1.0f, 0.0f);
    float ytm = aces_tonemap(el);
    float ls = (ytm / rmax(el, 1e-5f)) * 1.0f;
    V3<float> toned = project_to_gamut_bounded(xyz * ls, 1.0f);
    out[0] = encode_channel(toned.x); out[1] = encode_channel(toned.y); out[2] = encode_channel(toned.z);
}

// ---------------------------------------------------------------------------------
// a17. Optical metrics -- color/metrics.rs:16-30,118-227,230-284,383-448,504,568-676,
//      899-975,1082-1237 (FP32, libm, the reference's sequential reduction order)
// ---------------------------------------------------------------------------------
static inline void camera_view_basis(float yaw, float pitch, V3<float> &f, V3<float> &r, V3<float> &u) {
    float cp = ::cosf(pitch), sp = ::sinf(pitch), cy = ::cosf(yaw), sy = ::sinf(yaw);
    f = V3<float>(-cp * sy, -sp, -cp * cy).normalize();
    V3<float> up = std::fabs(cp) < 1e-4f ? V3<float>(0.f, 0.f, -1.f) : V3<float>(0.f, 1.f, 0.f);
    r = f.cross(up).normalize();
    u = r.cross(f).normalize();
}

static inline float metric_fresnel_t(float n1, float n2, float ci, float ct) {
    float ds = ::fmaf(n2, ct, n1 * ci), dp = ::fmaf(n2, ci, n1 * ct);
    if (std::fabs(ds) < 1e-6f || std::fabs(dp) < 1e-6f) return 0.0f;
    float a = ::fmaf(n2, -ct, n1 * ci) / ds, b = ::fmaf(n2, -ci, n1 * ct) / dp;
    float r = midpoint(a * a, b * b);
    return clampr(1.0f - r, 0.0f, 1.0f);
}

enum Fate { FATE_ENTRY_BLOCKED = 0, FATE_LEAKED = 1, FATE_EXITED = 2, FATE_ABSORBED = 3 };
struct ExitPath { V3<float> dir; float transmittance, exit_cos; int facet; uint32_t bounces; };

static inline int trace_wavelength(const V3<float> &entry, const V3<float> &in_dir, const V3<float> &n_entry,
                                   float cos_i, const gr_plane *planes, uint32_t n, float index, ExitPath &ex) {
    float sin2_t = (1.0f / (index * index)) * ::fmaf(cos_i, -cos_i, 1.0f);
    if (sin2_t > 1.0f) return FATE_ENTRY_BLOCKED;
    float cos_t = ::sqrtf(1.0f - sin2_t);
    V3<float> dir = ((1.0f / index) * in_dir + ::fmaf(1.0f / index, cos_i, -cos_t) * n_entry).normalize();
    V3<float> hp = entry + dir * 1e-4f;
    float sin_crit = 1.0f / index;
    float entry_t = metric_fresnel_t(1.0f, index, cos_i, cos_t);
    bool leaked = false, up = false;
    for (uint32_t bounce = 0; bounce < 10; ++bounce) {
        Ray<float> r;
        r.origin = hp;
        r.dir = dir;
        Hit<float> h = intersect_polyhedron(r, planes, n);
        if (!h.hit) break;
        V3<float> np = r.origin + h.t * r.dir;
        V3<float> n_out = h.normal;
        float ct = clampr(dir.dot(n_out), 0.0f, 1.0f);
        float st = ::sqrtf(rmax(::fmaf(ct, -ct, 1.0f), 0.0f));
        if (st < sin_crit) {
            float s2o = (index * index) * ::fmaf(ct, -ct, 1.0f);
            if (s2o <= 1.0f) {
                float co = ::sqrtf(1.0f - s2o);
                V3<float> od = (index * dir + ::fmaf(index, -ct, co) * n_out).normalize();
                if (n_out.y < -0.05f) {
                    leaked = true;
                } else if (od.y > 0.05f) {
                    up = true;
                    ex.dir = od;
                    ex.transmittance = metric_fresnel_t(index, 1.0f, ct, co);
                    ex.exit_cos = co;
                    ex.facet = h.facet;
                    ex.bounces = bounce;
                }
                break;
            }
        }
        dir = (dir - (2.0f * ct) * n_out).normalize();
        hp = np + dir * 1e-4f;
    }
    if (leaked) return FATE_LEAKED;
    if (up) { ex.transmittance = entry_t * ex.transmittance; return FATE_EXITED; }
    return FATE_ABSORBED;
}

static inline bool visibly_returned(const V3<float> &d, const V3<float> &fwd, const StudioRig<float> &rig) {
    bool head = (-d).dot(fwd) > 0.96f;
    float kd = rmax(d.dot(rig.key), 0.0f), fd = rmax(d.dot(rig.fill), 0.0f);
    bool ring = std::fabs(::fmaf(rig.sin_lp, -0.8f, d.y)) < 0.35f;
    bool lit = (kd > 0.70f) || (fd > 0.75f) || (ring && d.y > 0.2f);
    return !head && lit;
}

struct MetricsOut { float brilliance, fire, scintillation, windowing, extinction; };

static inline MetricsOut evaluate_gem_optical_metrics(const gr_plane *planes, uint32_t n, const gr_material *m,
                                                      float cam_yaw, float cam_pitch, float light_yaw, float light_pitch) {
    if (n == 0) return MetricsOut{85.0f, 25.0f, 75.0f, 5.0f, 5.0f};
    float nd = rmax(dispersion_evaluate<float>(m->dispersion, 589.3f), 1.1f);
    float nf = rmax(dispersion_evaluate<float>(m->dispersion, 486.1f), 1.001f);
    float nc = rmax(dispersion_evaluate<float>(m->dispersion, 656.3f), 1.001f);
    V3<float> fwd, right, upv;
    camera_view_basis(cam_yaw, cam_pitch, fwd, right, upv);
    StudioRig<float> rig = studio_rig_new<float>(light_yaw, light_pitch);
    const float ap[5][2] = {{0.f, 0.f}, {0.08f, 0.f}, {-0.08f, 0.f}, {0.f, 0.08f}, {0.f, -0.08f}};
    const float yaw_off[5] = {-3.0f, -1.5f, 0.0f, 1.5f, 3.0f};
    const float deg2rad = 3.14159265358979323846f / 180.0f;
    const float rad2deg = 57.2957795130823208767981548141051703f;
    uint32_t total = 0, windowed = 0, extinct = 0, returned = 0, cell_count = 0;
    float fire_sum = 0.f, cf_sum = 0.f, cf_sq = 0.f, tv_sum = 0.f;
    const int grid = 18;
    for (int ix = 0; ix < grid; ++ix) {
        for (int iz = 0; iz < grid; ++iz) {
            float u = ::fmaf(((float)ix + 0.5f) / (float)grid, 2.0f, -1.0f);
            float v = ::fmaf(((float)iz + 0.5f) / (float)grid, 2.0f, -1.0f);
            if (::fmaf(v, v, u * u) > 0.70f) continue;
            uint32_t ct_total = 0, ct_ret = 0;
            for (int a = 0; a < 5; ++a) {
                V3<float> rd = (fwd + ap[a][0] * right + ap[a][1] * upv).normalize();
                V3<float> ro = (-fwd) * 2.5f + (u * 0.95f) * right + (v * 0.95f) * upv;
                Ray<float> ray;
                ray.origin = ro;
                ray.dir = rd;
                Hit<float> h = intersect_polyhedron(ray, planes, n);
                if (!h.hit) continue;
                total++;
                ct_total++;
                V3<float> hp = ray.origin + h.t * ray.dir;
                float ci = clampr((-ray.dir).dot(h.normal), 0.0f, 1.0f);
                ExitPath e;
                int fate = trace_wavelength(hp, ray.dir, h.normal, ci, planes, n, nd, e);
                if (fate == FATE_ENTRY_BLOCKED) continue;
                if (fate == FATE_LEAKED) { windowed++; continue; }
                if (fate == FATE_ABSORBED) { extinct++; continue; }
                if (!visibly_returned(e.dir, fwd, rig)) { extinct++; continue; }
                returned++;
                ct_ret++;
                ExitPath ef, ec;
                int ff = trace_wavelength(hp, ray.dir, h.normal, ci, planes, n, nf, ef);
                int fc = trace_wavelength(hp, ray.dir, h.normal, ci, planes, n, nc, ec);
                if (ff == FATE_EXITED && fc == FATE_EXITED && ef.facet == ec.facet && ef.bounces == ec.bounces) {
                    float cs = clampr(ef.dir.dot(ec.dir), -1.0f, 1.0f);
                    float ang = ::acosf(cs) * rad2deg;
                    float w = (e.transmittance * ef.transmittance * ec.transmittance) *
                              (rmax(ef.exit_cos, 0.0f) * rmax(ec.exit_cos, 0.0f));
                    fire_sum = ::fmaf(ang, w, fire_sum);
                }
            }
            if (ct_total > 0) {
                float frac = (float)ct_ret / (float)ct_total;
                cf_sum += frac;
                cf_sq = ::fmaf(frac, frac, cf_sq);
                cell_count++;
                uint32_t tr = 0;
                for (int k = 0; k < 5; ++k) {
                    V3<float> f2, r2, u2;
                    camera_view_basis(cam_yaw + yaw_off[k] * deg2rad, cam_pitch, f2, r2, u2);
                    Ray<float> ray;
                    ray.origin = (-f2) * 2.5f + (u * 0.95f) * r2 + (v * 0.95f) * u2;
                    ray.dir = f2;
                    Hit<float> h = intersect_polyhedron(ray, planes, n);
                    if (!h.hit) continue;
                    V3<float> hp = ray.origin + h.t * ray.dir;
                    float ci = clampr((-ray.dir).dot(h.normal), 0.0f, 1.0f);
                    ExitPath e;
                    if (trace_wavelength(hp, ray.dir, h.normal, ci, planes, n, nd, e) == FATE_EXITED &&
                        visibly_returned(e.dir, f2, rig))
                        tr++;
                }
                float tp = (float)tr / 5.0f;
                tv_sum += ::fmaf(tp, -tp, tp);
            }
        }
    }
    float nt = (float)(total > 1 ? total : 1);
    MetricsOut o;
    o.windowing = clampr((float)windowed / nt * 100.0f, 0.0f, 100.0f);
    o.extinction = clampr((float)extinct / nt * 100.0f, 0.0f, 100.0f);
    o.brilliance = clampr((float)returned / nt * 100.0f, 0.0f, 100.0f);
    o.fire = rmax(fire_sum / nt * 275.0f, 0.1f);
    float spatial = 0.0f;
    if (cell_count > 0) {
        float mean = cf_sum / (float)cell_count;
        if (mean > 1e-4f) {
            float var = rmax(::fmaf(mean, -mean, cf_sq / (float)cell_count), 0.0f);
            float cv = ::sqrtf(var) / mean;
            spatial = clampr(cv / (1.0f + cv) * 100.0f, 0.0f, 100.0f);
        }
    }
    float temporal = cell_count > 0 ? clampr((tv_sum / (float)cell_count) / 0.24f * 100.0f, 0.0f, 100.0f) : 0.0f;
    o.scintillation = clampr(::fmaf(0.4f, temporal, 0.6f * spatial), 0.0f, 100.0f);
    return o;
}

}  // namespace gro
