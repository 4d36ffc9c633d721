// gr_trace.cuh -- the per-path transport loop (optics/raytracer/transport.rs:684-940)
// for polished facets of isotropic and uniaxial materials, split into resumable
// stages over a path record:
//
//   path_init    sampler draws, camera ray, per-sample wavelength cache
//   step_hit     one intersection; on a hit: Stokes frame rotation, interior
//                Beer-Lambert absorption, refraction geometry and the hero's event
//                decision (TIR / partial reflect / refract) -> Event
//   step_reflect the TIR and partial-reflect channel updates (one loop: a TIR event
//                is the reflect update with scale factor exactly 1.0)
//   step_refract the refract channel updates (chromatic termination, walk-off)
//   path_finish  escape radiance, spectral MIS, CIE integration, white balance
//
// The plain and staged kernels run the stages back to back in one thread; the sorted
// kernel (gr_sorted.cuh) keeps records in shared-memory slots and lets any thread of
// the block run any slot's next stage, grouped by event kind.  `Path` is a record of
// float4 rows: in the plain kernel it lives in the thread's local memory, in the
// sorted kernel in shared memory, in the staged kernels' park buffers in global
// memory -- the same code serves all of them.
#pragma once

#include <cstddef>

#include "gr_device.cuh"

namespace grd {

constexpr int NCH = 8;

// Unroll factors of the per-channel loops on the bounce path (code size vs. issue).
#ifndef GR_ROT_UNROLL
#define GR_ROT_UNROLL 8
#endif
#ifndef GR_RR_UNROLL
#define GR_RR_UNROLL 4  // measured on the c2 frame: 4 beats 8 / 2 / 1 by 1-3% (code layout)
#endif
// The rotation loop of the general (absorbing or birefringent) scene classes: measured
// at 16 blocks per SM, unrolled by 2 / 4 / 8, the c3 emerald 585.5 / 580.7 / 563.6 M
// path-samples/s and the c4 random stones one at a time at full size 571 / 583 / 577 M;
// the clear brilliant wants 8 (1,032.6 against 1,017.2 at 4 and 1,009.6 at 2).  The best
// factor follows the kernel's code layout; 4 is the best for both general workloads.
#ifndef GR_ROT_UNROLL_GENERAL
#define GR_ROT_UNROLL_GENERAL 4
#endif
constexpr int ROT_UNROLL = GR_ROT_UNROLL;
constexpr int RR_UNROLL = GR_RR_UNROLL;

// Per-path record (352 B).  Flag bits live in k_state.w's integer view.
struct __align__(16) Path {
    float4 o_hero;      // ray origin, hero_rand
    float4 d_seed;      // ray (Poynting) direction S, rng seed bits
    float4 k_state;     // wave normal k, state bits (bounce | flags)
    float4 prev_tuple;  // previous plane-of-incidence normal (zero = none), tuple bits
    float4 st[NCH];     // Stokes (I, Q, U, V) per channel
    float4 pdf4[2];     // spectral-MIS path pdf per channel
    float4 n_o4[2];     // ordinary index per channel
    float4 ne_d4[2];    // n_e - n_o per channel (biaxial materials: beta-ray absorption coefficient)
    float4 a_o4[2];     // ordinary absorption coefficient per channel
    float4 a_e4[2];     // extraordinary absorption coefficient per channel
};
static_assert(sizeof(Path) == 352, "path record size");
static_assert(offsetof(Path, ne_d4) == 256, "the tables a clear isotropic stone never touches come last");

// Event scratch between step_hit and the event stage (64 B).
struct __align__(16) Event {
    float4 hp_cos;   // hit point, cos_i (against the wave normal, normal facing the ray)
    float4 n_ru;     // normal (flipped to face the interior ray), hero r_unpol (0 for TIR)
    float4 n_med4[2];
};

constexpr uint32_t F_INSIDE = 1u << 0;
constexpr uint32_t F_IS_E = 1u << 1;
constexpr uint32_t F_ABSORBING = 1u << 2;
constexpr uint32_t F_ESCAPED = 1u << 3;
constexpr uint32_t F_ALIVE = 1u << 4;
constexpr uint32_t F_TIR = 1u << 5;  // the pending event is a hero TIR
constexpr uint32_t BOUNCE_SHIFT = 8;

// Scene class known at compile time (template parameter K of the single-scene kernels):
// the run-time material and environment checks it settles are folded away, so a clear
// isotropic stone's kernel carries none of the birefringence, walk-off, absorption or
// other-environment code.  K = K_ANY keeps every check at run time (batched launches,
// the instrumented variants).
constexpr int K_ANY = 0;
constexpr int K_ISO = 1;        // S.anisotropic == 0 (and not biaxial)
constexpr int K_CLEAR = 2;      // S.absorbing == 0: no absorption data at all
constexpr int K_ENV_SHIFT = 2;  // bits 2-3: 0 = the environment kind at run time, else GR_ENV_* + 1
__host__ __device__ constexpr int k_env(uint32_t env) { return (int)(env + 1) << K_ENV_SHIFT; }
// The rotation loop's unroll factor in the kernels of scene class K.
__host__ __device__ constexpr int rot_unroll(int K) {
    return (K != K_ANY && !(K & K_CLEAR)) ? GR_ROT_UNROLL_GENERAL : GR_ROT_UNROLL;
}
template <int K> __device__ __forceinline__ bool aniso_k(const SceneConst &S) {
    return (K & K_ISO) ? false : (S.anisotropic != 0);
}
template <int K> __device__ __forceinline__ bool absorbing_k(uint32_t bits) {
    return (K & K_CLEAR) ? false : ((bits & F_ABSORBING) != 0);
}
template <int K> __device__ __forceinline__ uint32_t env_k(const SceneConst &S) {
    return (K >> K_ENV_SHIFT) ? (uint32_t)((K >> K_ENV_SHIFT) - 1) : S.env_mode;
}

// EV_HANDLED: the bounce was completed inside step_hit (a frosted facet or a volume
// scattering event); the path continues with the next intersection if still alive.
enum EventKind : uint32_t { EV_DONE = 0, EV_REFLECT = 1, EV_REFRACT = 2, EV_HANDLED = 3 };

__device__ __forceinline__ float &arr(float4 (&a)[2], int k) { return reinterpret_cast<float *>(a)[k]; }
__device__ __forceinline__ float arr(const float4 (&a)[2], int k) { return reinterpret_cast<const float *>(a)[k]; }
// Bytes of Path an isotropic stone's kernels touch: the per-channel tables after n_o4
// (n_e - n_o and the absorption coefficients) are neither written nor read for K_ISO |
// K_CLEAR, and an isotropic stone's Event carries no medium indices (they are n_o4):
// the shared-memory slots of the sorted kernel hold only these leading bytes.
constexpr size_t PATH_CLEAR_BYTES = 256;
constexpr size_t EVENT_ISO_BYTES = 32;
// The medium index of channel k at the pending event: the ordinary index of an
// isotropic stone, else what step_hit left in the event record.
template <int K> __device__ __forceinline__ float n_med(const Path &P, const Event &E, int k) {
    return (K & K_ISO) ? arr(P.n_o4, k) : arr(E.n_med4, k);
}
__device__ __forceinline__ V3 xyz(const float4 &v) { return v3(v.x, v.y, v.z); }
__device__ __forceinline__ void set_xyz(float4 &v, V3 a) { v.x = a.x; v.y = a.y; v.z = a.z; }
__device__ __forceinline__ uint32_t state_bits(const Path &P) { return __float_as_uint(P.k_state.w); }
__device__ __forceinline__ void set_state_bits(Path &P, uint32_t s) { P.k_state.w = __uint_as_float(s); }
__device__ __forceinline__ uint32_t p_bounce(const Path &P) { return state_bits(P) >> BOUNCE_SHIFT; }
__device__ __forceinline__ uint32_t p_flags(const Path &P) { return state_bits(P) & ((1u << BOUNCE_SHIFT) - 1u); }
__device__ __forceinline__ uint32_t p_seed(const Path &P) { return __float_as_uint(P.d_seed.w); }
__device__ __forceinline__ uint32_t p_tuple(const Path &P) { return __float_as_uint(P.prev_tuple.w); }
__device__ __forceinline__ float p_hero(const Path &P) { return P.o_hero.w; }

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

// Per-tuple event-sequence recorder of the instrumented variant (gr_trace_events): the
// facet, hit distance and event of each bounce b < kmax, and how the path ended.  The
// other hook types record nothing, so their instantiations carry no recording code.
struct EventRec {
    int32_t *facets;
    float *ts;
    uint8_t *events;
    uint32_t *bounces, *term;
    uint32_t kmax;
    uint64_t t;
};
template <class CT> __device__ __forceinline__ void note_hit(CT &, uint32_t, int, float) {}
template <class CT> __device__ __forceinline__ void note_event(CT &, uint32_t, uint32_t) {}
template <class CT> __device__ __forceinline__ void note_end(CT &, uint32_t, uint32_t) {}
template <> __device__ __forceinline__ void note_hit<EventRec>(EventRec &r, uint32_t b, int f, float t) {
    if (b < r.kmax) {
        r.facets[r.t * r.kmax + b] = f;
        r.ts[r.t * r.kmax + b] = t;
    }
}
template <> __device__ __forceinline__ void note_event<EventRec>(EventRec &r, uint32_t b, uint32_t ev) {
    if (b < r.kmax) r.events[r.t * r.kmax + b] = (uint8_t)ev;
}
template <> __device__ __forceinline__ void note_end<EventRec>(EventRec &r, uint32_t b, uint32_t term) {
    r.bounces[r.t] = b;
    r.term[r.t] = term;
}

// Build the path of tuple (pixel, sample): sampler draws (sampling.rs:232-271),
// camera ray (camera.rs:95-114), per-sample wavelength cache (refraction.rs:127-174).
// X: the extension instantiation (biaxial materials keep their beta-ray coefficient,
// or the ordinary one when the material has no third band set, where uniaxial ones
// keep n_e - n_o, which no biaxial step reads).
// Camera::generate_ray (camera.rs:95-114): the primary direction through pixel (x, y)
// with jitter (jx, jy).
__device__ __forceinline__ V3 camera_dir(const SceneConst &S, float x, float y, float jx, float jy) {
    float aspect = S.width_f / S.height_f;
    float u = ((x + jx) / S.width_f - 0.5f) * 2.0f * aspect * S.fov_tan;
    float v = (0.5f - (y + jy) / S.height_f) * 2.0f * S.fov_tan;
    return normalize(add(add(ld3(S.cam_f), mul(ld3(S.cam_r), u)), mul(ld3(S.cam_u), v)));
}

template <int U = 1, bool X = false, int K = K_ANY>
__device__ __forceinline__ void path_init(Path &P, const SceneConst &S, const SceneBuffers &B, uint32_t pixel,
                                          uint32_t sample, uint32_t tuple) {
    Draws dr = sample_draws(pixel, sample);
    uint32_t x = pixel % S.width, y = pixel / S.width;
    V3 dir = camera_dir(S, (float)x, (float)y, dr.jx, dr.jy);
    P.o_hero = make_float4(S.cam_o[0], S.cam_o[1], S.cam_o[2], dr.hero);
    P.d_seed = make_float4(dir.x, dir.y, dir.z, __uint_as_float(dr.seed));
    P.prev_tuple = make_float4(0.f, 0.f, 0.f, __uint_as_float(tuple));
    bool any = false;
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        P.st[k] = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        arr(P.pdf4, k) = 1.0f;
        float lam = lambda_k(dr.hero, k);
        float n_o = dispersion(S, lam);
        arr(P.n_o4, k) = n_o;
        if (K & K_ISO) {
            // no birefringence: n_e - n_o is never read
        } else if (S.has_cauchy_e) {
            float lum = lam * 1e-3f;
            float l2 = lum * lum, l4 = l2 * l2;
            float n_e = S.cauchy_e[0] + S.cauchy_e[1] / l2 + S.cauchy_e[2] / l4;
            arr(P.ne_d4, k) = n_e - n_o;
        } else {
            arr(P.ne_d4, k) = S.bire;
        }
        float ao = 0.0f, ae = 0.0f;
        if (!(K & K_CLEAR) && S.absorbing) {
            if (S.ext_n > 0) {
                ao = table_lookup(B.ext_alpha_o, S.ext_n, S.ext_first, S.ext_step, lam);
                ae = table_lookup(B.ext_alpha_e, S.ext_n, S.ext_first, S.ext_step, lam);
            } else {
                ao = band_sum(S.o_bands, S.n_o_bands, lam);
                ae = band_sum(S.e_bands, S.n_e_bands, lam);
            }
        }
        if (!(K & K_CLEAR)) {  // a clear stone's kernel never reads them
            arr(P.a_o4, k) = ao;
            arr(P.a_e4, k) = ae;
        }
        any = any || (ao != 0.0f) || (ae != 0.0f);
        if (X && S.biaxial) {
            const float ab = (S.absorbing && S.has_beta) ? band_sum(S.b_bands, S.n_b_bands, lam) : ao;
            arr(P.ne_d4, k) = ab;
            any = any || (ab != 0.0f);
        }
    }
    // Every alpha exactly zero makes the Beer-Lambert factor exp_poly(-0) == 1.0 for
    // every channel, so skipping the absorption step is bit-identical.
    uint32_t flags = F_ALIVE | (any ? F_ABSORBING : 0u);
    if (S.max_bounces == 0) flags &= ~F_ALIVE;
    P.k_state = make_float4(dir.x, dir.y, dir.z, __uint_as_float(flags));
}

// Convex clip against planes staged in shared memory (intersect.rs:93-132,
// simd/slab.rs:101-152).  Returns false on a miss.
//
// The reference divides t = -side/denom for every plane, but a plane's t only
// matters if it can raise the running near maximum (denom < 0) or lower the running
// far minimum (denom > 0).  q' = (-side) * rcp.approx(denom) is within 2^-21 relative
// of the exact quotient q; if q' + |q'| 2^-19 < t_near then q < t_near, so the
// correctly rounded fl(q) <= t_near and the plane cannot update (rounding is
// monotone) -- likewise for the far side.  Only the remaining planes take the IEEE
// division, so every t that is compared or kept is the reference's own bits.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ bool intersect(const float4 *__restrict__ planes, uint32_t n, V3 o, V3 d, float &t_hit,
                                          int &idx_hit) {
    float t_near = -1e30f, t_far = 1e30f;
    int near_idx = -1, far_idx = -1;
    bool outside = false;
#pragma unroll 2
    for (uint32_t i = 0; i < n; ++i) {
        float4 p = planes[i];
        float denom = (p.x * d.x + p.y * d.y) + p.z * d.z;
        float side = p.w + ((p.x * o.x + p.y * o.y) + p.z * o.z);
        if (fabsf(denom) > 1e-7f) {
            const float num = -side;
            const float qa = num * rcp_approx(denom);
            const float margin = fabsf(qa) * 1.9073486e-6f;  // 2^-19
            if (denom < 0.0f) {
                if (!(qa + margin < t_near)) {
                    float t = num / denom;
                    if (t > t_near) { t_near = t; near_idx = (int)i; }
                }
            } else if (!(qa - margin > t_far)) {
                float t = num / denom;
                if (t < t_far) { t_far = t; far_idx = (int)i; }
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

// ---------------------------------------------------------------------------------
// Paired plane scan for the transport kernels.
//
// Planes are staged twice in shared memory: as float4 (n.xyz, d) for lookups by
// index, and pair-interleaved as {nx0, nx1, ny0, ny1}, {nz0, nz1, d0, d1}, so that
// one packed mul.rn.f32x2 (sm_100: two IEEE round-to-nearest products) forms the
// same product for two planes.  The sums stay scalar: a fully packed evaluation
// (packed sums as well) did not reproduce the scalar scan's results on B200, while
// packed products with scalar sums are bit-identical to it.  An odd tail is padded
// with the plane n = 0, d = -1 (denom = 0, side = -1), which never acts.
//
// The per-plane decisions are those of the reference loop, reduced by two exact
// rules (intersect.rs:93-132):
//   * an entering plane (denom < -1e-7) with side <= 0 has t = -side/denom <= 0.
//     Such t can only matter through t_near > t_far or t_near > 1e-4; the second is
//     false for t <= 0, and if t_far < t <= 0 the far test (t_far > 1e-4) fails as
//     well, so the outcome is a miss either way -- the plane is skipped;
//   * a plane with side > 0 that the ray does not enter (denom >= -1e-7) is either
//     parallel and outside (SlabScan::Outside) or gives t < 0 as a far candidate,
//     forcing t_far < 0 and hence a miss -- the scan returns a miss at once.
// Every t that is compared or kept is still the IEEE quotient -side / denom.
// ---------------------------------------------------------------------------------
struct Planes {
    const float4 *aos;    // n x (n.xyz, d)
    const float4 *pairs;  // ceil(n / 2) x 2 float4, interleaved as above
    uint32_t n;
};

__host__ __device__ constexpr size_t planes_smem_bytes(uint32_t n) {
    return (size_t)(n + 2u * ((n + 1u) / 2u)) * 16u;
}

typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(f32x2 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// One plane's contribution; returns false when the scan ends in a miss.  With R
// (FP64 re-solve) the division-skip margin widens to 2^-15 and the runner-up t of
// each side is tracked: every plane whose t lies within ~2.9e-5 (relative) of the
// running extremum is divided exactly, so a runner-up within 1e-5 is never missed.
template <bool R>
__device__ __forceinline__ bool scan_plane(float denom, float side, int i, float &t_near, int &near_idx, float &t_far,
                                           int &far_idx, float &t_near2, float &t_far2) {
    constexpr float M = R ? 3.0517578e-5f : 1.9073486e-6f;  // 2^-15 : 2^-19
    if (denom < -1e-7f) {
        if (side > 0.0f) {
            const float num = -side;
            const float qa = num * rcp_approx(denom);
            if (!(qa + fabsf(qa) * M < t_near)) {
                const float t = num / denom;
                if (t > t_near) {
                    if (R) t_near2 = t_near;
                    t_near = t;
                    near_idx = i;
                } else if (R && t > t_near2) {
                    t_near2 = t;
                }
            }
        }
    } else if (side > 0.0f) {
        return false;
    } else if (denom > 1e-7f) {
        const float num = -side;
        const float qa = num * rcp_approx(denom);
        if (!(qa - fabsf(qa) * M > t_far)) {
            const float t = num / denom;
            if (t < t_far) {
                if (R) t_far2 = t_far;
                t_far = t;
                far_idx = i;
            } else if (R && t < t_far2) {
                t_far2 = t;
            }
        }
    }
    return true;
}

// The reference clip (intersect.rs:93-132) in FP64, t rounded back to f32: the
// re-solve for rays whose f32 exit facet is ambiguous.  Out of line: it runs for
// only a tiny fraction of rays.
static __device__ __noinline__ bool intersect_fp64(const float4 *__restrict__ planes, uint32_t n, V3 o, V3 d,
                                                   float &t_hit, int &idx_hit) {
    double tn = -1e30, tf = 1e30;
    int ni = -1, fi = -1;
    for (uint32_t i = 0; i < n; ++i) {
        const float4 p = planes[i];
        const double denom = ((double)p.x * d.x + (double)p.y * d.y) + (double)p.z * d.z;
        const double side = (double)p.w + (((double)p.x * o.x + (double)p.y * o.y) + (double)p.z * o.z);
        if (fabs(denom) > 1e-7) {
            const double t = -side / denom;
            if (denom < 0.0) {
                if (t > tn) { tn = t; ni = (int)i; }
            } else if (t < tf) {
                tf = t;
                fi = (int)i;
            }
        } else if (side > 0.0) {
            return false;
        }
    }
    if (tn > tf) return false;
    if (tn > 1e-4) { t_hit = (float)tn; idx_hit = ni; return true; }
    if (tf > 1e-4) { t_hit = (float)tf; idx_hit = fi; return true; }
    return false;
}

// R: re-solve in FP64 when the chosen exit is within 1e-5 (relative) of the
// runner-up plane or of the other side's extremum (a ray grazing an edge).
template <bool R = false>
__device__ __forceinline__ bool intersect(const Planes &PL, V3 o, V3 d, float &t_hit, int &idx_hit) {
    float t_near = -1e30f, t_far = 1e30f, t_near2 = -1e30f, t_far2 = 1e30f;
    int near_idx = -1, far_idx = -1;
    const f32x2 dx = pk2(d.x, d.x), dy = pk2(d.y, d.y), dz = pk2(d.z, d.z);
    const f32x2 ox = pk2(o.x, o.x), oy = pk2(o.y, o.y), oz = pk2(o.z, o.z);
    const uint32_t np = (PL.n + 1u) >> 1;
    // not unrolled: unrolling the pair loop by 2 / 4 was measured 4% / 18% slower on the
    // c2 frame (the kernels are instruction-fetch bound)
#pragma unroll 1
    for (uint32_t j = 0; j < np; ++j) {
        const float4 a = PL.pairs[2 * j], b = PL.pairs[2 * j + 1];
        const f32x2 nx = pk2(a.x, a.y), ny = pk2(a.z, a.w), nz = pk2(b.x, b.y);
        float xd0, xd1, yd0, yd1, zd0, zd1, xo0, xo1, yo0, yo1, zo0, zo1;
        upk2(mul2(nx, dx), xd0, xd1);
        upk2(mul2(ny, dy), yd0, yd1);
        upk2(mul2(nz, dz), zd0, zd1);
        upk2(mul2(nx, ox), xo0, xo1);
        upk2(mul2(ny, oy), yo0, yo1);
        upk2(mul2(nz, oz), zo0, zo1);
        // denom = (nx*dx + ny*dy) + nz*dz;  side = d + ((nx*ox + ny*oy) + nz*oz)
        const float den0 = (xd0 + yd0) + zd0, den1 = (xd1 + yd1) + zd1;
        const float sid0 = b.z + ((xo0 + yo0) + zo0), sid1 = b.w + ((xo1 + yo1) + zo1);
        if (!scan_plane<R>(den0, sid0, (int)(2 * j), t_near, near_idx, t_far, far_idx, t_near2, t_far2)) return false;
        if (!scan_plane<R>(den1, sid1, (int)(2 * j + 1), t_near, near_idx, t_far, far_idx, t_near2, t_far2))
            return false;
    }
    if (R) {
        const float tol = 1e-5f;
        bool amb = fabsf(t_near - t_far) <= tol * fmaxf(fabsf(t_near), fabsf(t_far));
        if (t_near > 1e-4f) amb = amb || (t_near - t_near2 <= tol * t_near);
        else if (t_far > 1e-4f) amb = amb || (t_far2 - t_far <= tol * t_far);
        if (amb) return intersect_fp64(PL.aos, PL.n, o, d, t_hit, idx_hit);
    }
    if (t_near > t_far) return false;
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

// Per-channel pleochroic alpha of the current segment (channel_absorption_alphas,
// raytracer/absorption.rs:175-216) against plane-of-incidence normal `s_axis`.
// The eigenmode pair of channel_absorption_alphas (raytracer/absorption.rs:175-196):
// the hero indicatrix's (slow, fast) D directions for a biaxial material (X only),
// else the uniaxial ordinary / extraordinary pair.
template <bool X>
__device__ __forceinline__ void absorption_eigenmodes(const Path &P, const SceneConst &S, V3 kk, V3 &ea, V3 &eb) {
    if (X && S.biaxial) {
        eigen_pair(S, make_ind(S, arr(P.n_o4, 0)), kk, ea, eb);
    } else {
        ea = ordinary_eigen(kk, ld3(S.c_axis));
        eb = extraordinary_eigen_from(kk, ea);
    }
}
// effective_pleochroic_alpha (optics/birefringence.rs:272-286) of channel k against the
// tensor the wavelength cache built for it (uniaxial, or biaxial with a beta band set).
// effective_pleochroic_alpha for the uniaxial tensor (a_o, a_o, a_e) of the scene frame.
__device__ __forceinline__ float pleochroic_alpha(const SceneConst &S, float a_o, float a_e, const Stokes &st, V3 e_hat,
                                                  V3 ea, V3 eb) {
    const float p = clampf(dop(st), 0.0f, 1.0f);
    const float a_pol = quad_form(S, a_o, a_e, e_hat);
    const float a_unp = midpoint(quad_form(S, a_o, a_e, ea), quad_form(S, a_o, a_e, eb));
    return fmaf(p, a_pol - a_unp, a_unp);
}
template <bool X>
__device__ __forceinline__ float channel_alpha(const Path &P, const SceneConst &S, int k, const Stokes &st, V3 e_hat,
                                               V3 ea, V3 eb) {
    const float a_o = arr(P.a_o4, k), a_e = arr(P.a_e4, k);
    if (X && S.biaxial) {
        const float p = clampf(dop(st), 0.0f, 1.0f);
        const float a_b = arr(P.ne_d4, k);
        const float a_pol = quad_form3(S, a_o, a_b, a_e, e_hat);
        const float a_unp = midpoint(quad_form3(S, a_o, a_b, a_e, ea), quad_form3(S, a_o, a_b, a_e, eb));
        return fmaf(p, a_pol - a_unp, a_unp);
    }
    return pleochroic_alpha(S, a_o, a_e, st, e_hat, ea, eb);
}

template <int U, bool X = false>
__device__ __forceinline__ void segment_alphas(const Path &P, const SceneConst &S, V3 s_axis, V3 kk, float alpha[NCH]) {
    if (!(state_bits(P) & F_ABSORBING)) {
#pragma unroll
        for (int k = 0; k < NCH; ++k) alpha[k] = 0.0f;
        return;
    }
    V3 ea, eb;
    absorption_eigenmodes<X>(P, S, kk, ea, eb);
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        const float4 s4 = P.st[k];
        const Stokes st{s4.x, s4.y, s4.z, s4.w};
        const V3 e_hat = electric_field_direction(st, s_axis, kk);
        alpha[k] = channel_alpha<X>(P, S, k, st, e_hat, ea, eb);
    }
}

// Roulette and the bounce count after a step that does not go through step_post
// (apply_russian_roulette, transport.rs:204-220, then the loop's next bounce).
template <class CT>
__device__ __forceinline__ void advance_bounce(Path &P, const SceneConst &S, CT &ct) {
    uint32_t bits = state_bits(P);
    const uint32_t bounce = bits >> BOUNCE_SHIFT;
    if (bounce > 4) {
        float mx = 0.0f;
#pragma unroll RR_UNROLL
        for (int k = 0; k < NCH; ++k) mx = fmaxf(mx, fmaxf(P.st[k].x, 0.0f));
        const float q = clampf(mx, 0.05f, 1.0f);
        if (rng_draw(p_seed(P), bounce, RUSSIAN_ROULETTE_STREAM) > q) {
            note_end(ct, bounce, GR_TERM_ROULETTE);
            set_state_bits(P, bits & ~F_ALIVE);
            return;
        }
        const float iq = 1.0f / q;
#pragma unroll RR_UNROLL
        for (int k = 0; k < NCH; ++k) {
            const float4 s4 = P.st[k];
            P.st[k] = make_float4(s4.x * iq, s4.y * iq, s4.z * iq, s4.w * iq);
        }
    }
    const uint32_t nb = bounce + 1;
    bits = (bits & ((1u << BOUNCE_SHIFT) - 1u)) | (nb << BOUNCE_SHIFT);
    if (nb >= S.max_bounces) bits &= ~F_ALIVE;
    set_state_bits(P, bits);
}

// maybe_scatter_or_extinguish (raytracer/scattering.rs:132-212) for the interior
// segment of length t_hit from the path's origin (out of line, like frosted_bounce:
// rare paths kept out of the transport loop's registers).  Returns true when a scattering
// event happened (the path moved to the event point with a new direction, and the
// bounce is complete); false when the segment was crossed, its extinction applied.
template <int U, class CT>
__device__ __noinline__ bool scatter_step(Path &P, const SceneConst &S, float t_hit, CT &ct) {
    const uint32_t bounce = p_bounce(P);
    const uint32_t seed = p_seed(P);
    const V3 kk = xyz(P.k_state);
    float alpha[NCH];
    segment_alphas<U, true>(P, S, xyz(P.prev_tuple), kk, alpha);
    const float sigma_s = S.sigma_s;
    const float sigma_t_hero = alpha[0] + sigma_s;  // the hero is channel 0
    const float omu = fmaxf(1.0f - rng_draw(seed, bounce, DISTANCE_SAMPLE_STREAM), 1e-7f);
    const float t_free = -(m_log(omu)) / sigma_t_hero;
    const float hit_scaled = t_hit * S.path_scale;
    if (t_free < hit_scaled) {
        const float pdf_hero = sigma_t_hero * omu;
#pragma unroll U
        for (int k = 0; k < NCH; ++k) {
            const float sigma_t_k = alpha[k] + sigma_s;
            const float tr = exp_poly(-(alpha[k] + sigma_s) * t_free);
            const float w = tr * sigma_s / pdf_hero;
            P.st[k] = make_float4(fmaxf(P.st[k].x, 0.0f) * w, 0.0f, 0.0f, 0.0f);
            arr(P.pdf4, k) = arr(P.pdf4, k) * (sigma_t_k * tr);
        }
        const float u1 = rng_draw(seed, bounce, PHASE_DIR_U_STREAM);
        const float u2 = rng_draw(seed, bounce, PHASE_DIR_V_STREAM);
        const V3 d = xyz(P.d_seed);
        const V3 nd = sample_hg_direction(u1, u2, S.hg_g, d);
        set_xyz(P.o_hero, add(xyz(P.o_hero), smul(t_free / S.path_scale, d)));
        set_xyz(P.d_seed, nd);
        set_xyz(P.k_state, nd);
        set_xyz(P.prev_tuple, v3(0.f, 0.f, 0.f));  // depolarized: no previous plane of incidence
        note_event(ct, bounce, GR_SEQ_SCATTER);
        advance_bounce(P, S, ct);
        return true;
    }
    float sv[NCH];
#pragma unroll U
    for (int k = 0; k < NCH; ++k) sv[k] = exp_poly(-(alpha[k] + sigma_s) * hit_scaled);
    const float sh = fmaxf(sv[0], 1e-30f);
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        const float f = sv[k] / sh;
        const float4 s4 = P.st[k];
        P.st[k] = make_float4(s4.x * f, s4.y * f, s4.z * f, s4.w * f);
        arr(P.pdf4, k) = arr(P.pdf4, k) * sv[k];
    }
    return false;
}

// hero_biaxial_wave_dirs + per_channel_biaxial_indices (refraction.rs:345-401) with the
// medium choice of compute_bounce_refraction_geometry (:509-520): each channel's slow
// (mode B) index at the hero's slow wave normal -- the ray's own inside the stone, the
// resolved refracted one (resolve_entry_mode) outside -- or, for the fast mode inside
// (use_a), its fast (mode A) index.
static __device__ __noinline__ void biaxial_media(const Path &P, const SceneConst &S, V3 kk, V3 normal, float cos_i,
                                                  bool inside, bool use_a, Event &E) {
    const float n0 = arr(P.n_o4, 0);
    const V3 dir = inside ? kk : resolve_entry_mode(S, make_ind(S, n0), kk, normal, cos_i, n0, true);
#pragma unroll 1
    for (int k = 0; k < NCH; ++k) {
        float ns, nf;
        wave_indices(S, make_ind(S, arr(P.n_o4, k)), dir, ns, nf);
        arr(E.n_med4, k) = use_a ? nf : ns;
    }
}
// The mode-A (fast) indices at the hero's resolved fast wave normal, for a fast-mode
// biaxial entry (n_biax_a_ch, refraction.rs:381-401).
static __device__ __noinline__ void biaxial_fast_entry(const Path &P, const SceneConst &S, V3 kk, V3 normal,
                                                       float cos_i, Event &E) {
    const float n0 = arr(P.n_o4, 0);
    const V3 dir = resolve_entry_mode(S, make_ind(S, n0), kk, normal, cos_i, n0, false);
#pragma unroll 1
    for (int k = 0; k < NCH; ++k) {
        float ns, nf;
        wave_indices(S, make_ind(S, arr(P.n_o4, k)), dir, ns, nf);
        arr(E.n_med4, k) = nf;
    }
}

// signed_frame_rotation_psi (raytracer/absorption.rs:44-54)
__device__ __forceinline__ float signed_psi(V3 prev, V3 cur, V3 kk) {
    float cos_psi = clampf(dot(prev, cur), -1.0f, 1.0f);
    float sin_psi = dot(cross(prev, cur), normalize_or_zero(kk));
    return m_atan2(sin_psi, cos_psi);
}

// theta_c_for_bounce (refraction.rs:235-273): on entry the refracted wave normal's
// angle to the c-axis after a two-step fixed point (refraction.rs:248-269), otherwise
// the ray's own.
template <int U>
__device__ __forceinline__ float theta_c(V3 kk, V3 normal, float cos_i, float one_m_c2, float n_o_hero, float n_e_hero,
                                         V3 c_axis, bool entry) {
    float theta;
    if (entry) {
        float n_guess = n_o_hero;
        theta = 0.0f;
#pragma unroll U
        for (int it = 0; it < 2; ++it) {
            float eta = 1.0f / n_guess;
            float s2 = eta * eta * one_m_c2;
            if (s2 > 1.0f) break;
            float ctg = sqrtf(fmaxf(1.0f - s2, 0.0f));
            V3 wd = normalize(add(smul(eta, kk), smul(fmaf(eta, cos_i, -ctg), normal)));
            theta = m_acos(fabsf(clampf(dot(wd, c_axis), -1.0f, 1.0f)));
            float2 sc = m_sincos(theta);
            n_guess = eff_e_index(n_o_hero, n_e_hero, sc.x, sc.y);
        }
    } else {
        theta = m_acos(fabsf(clampf(dot(kk, c_axis), -1.0f, 1.0f)));
    }
    return theta;
}

// One intersection and everything of the bounce up to the hero's event decision
// (transport.rs:781-895, raytracer/absorption.rs:71-141, refraction.rs:428-547,
// 1036-1060).  Returns EV_DONE on an escape (F_ESCAPED set, F_ALIVE cleared).
// X: the instantiation that handles frosted facets, volume scattering and biaxial
// materials (scenes without any of them run the X = false code, which has none of
// those branches).
template <int U, class CT, bool R = false, bool X = false, int K = K_ANY>
__device__ __forceinline__ uint32_t step_hit(Path &P, const SceneConst &S, const Planes &PL, Event &E, CT &ct) {
    const uint32_t bits = state_bits(P);
    const uint32_t bounce = bits >> BOUNCE_SHIFT;
    const bool inside = (bits & F_INSIDE) != 0;
    const V3 o = xyz(P.o_hero), d = xyz(P.d_seed), kk = xyz(P.k_state);
    float t_hit = 0.0f;
    int fidx = 0;
    tally(ct, C_BOUNCES);
    if (!intersect<R>(PL, o, d, t_hit, fidx)) {
        // accumulate_miss_radiance (transport.rs:67-90) runs in path_finish
        tally(ct, C_ESCAPES);
        note_end(ct, bounce, GR_TERM_ESCAPED);
        set_state_bits(P, (bits | F_ESCAPED) & ~F_ALIVE);
        return EV_DONE;
    }
    note_hit(ct, bounce, fidx, t_hit);
    bool extinguished = false;  // the segment's extinction was applied by the scattering step
    if (X && inside && S.sigma_s > 0.0f) {
        // try_scatter_step / maybe_scatter_or_extinguish (raytracer/scattering.rs:132-315):
        // a Henyey-Greenstein event along this interior segment, drawn before the facet
        if (scatter_step<U>(P, S, t_hit, ct)) return EV_HANDLED;
        extinguished = true;
    }
    V3 hp = add(o, smul(t_hit, d));
    V3 normal = shading_normal(PL.aos, PL.n, hp, fidx, plane_normal(PL.aos, fidx), S.edge_radius);

    // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:71-89)
    V3 cur_plane = normalize_or_zero(cross(kk, normal));
    const V3 prev = xyz(P.prev_tuple);
    if (dot(cur_plane, cur_plane) > 1e-6f && dot(prev, prev) > 1e-6f) {
        float psi = signed_psi(prev, cur_plane, kk);
        float2 sc = m_sincos(2.0f * psi);
#pragma unroll (rot_unroll(K))
        for (int k = 0; k < NCH; ++k) {
            float4 s = P.st[k];
            Stokes r = apply_rotation(Stokes{s.x, s.y, s.z, s.w}, sc.y, sc.x);
            P.st[k] = make_float4(r.i, r.q, r.u, r.v);
        }
        tally(ct, C_ROTATIONS);
    }
    set_xyz(P.prev_tuple, cur_plane);

    // apply_interior_segment (transport.rs:586-605) -> apply_absorption (absorption.rs:115-141)
    if (inside) {
        normal = neg(normal);
        if (absorbing_k<K>(bits) && !extinguished) {
            tally(ct, C_ABSORB);
            V3 ea, eb;
            absorption_eigenmodes<X>(P, S, kk, ea, eb);
            float scaled = t_hit * S.path_scale;
            // Every channel's alpha reads that channel's Stokes vector before it is
            // scaled, so computing and applying per channel is the reference's
            // two-pass loop (absorption.rs:123-140) in one pass.
#pragma unroll U
            for (int k = 0; k < NCH; ++k) {
                float4 s4 = P.st[k];
                Stokes s{s4.x, s4.y, s4.z, s4.w};
                V3 e_hat = electric_field_direction(s, cur_plane, kk);
                float alpha = channel_alpha<X>(P, S, k, s, e_hat, ea, eb);
                Stokes r = scale(s, exp_poly(-alpha * scaled));
                P.st[k] = make_float4(r.i, r.q, r.u, r.v);
            }
        }
    }

    // compute_bounce_refraction_geometry (refraction.rs:428-547), uniaxial branch
    const bool aniso = aniso_k<K>(S);
    float cos_i = clampf(dot(neg(kk), normal), 0.0f, 1.0f);
    float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    float n_o_hero = arr(P.n_o4, 0);
    if (X && S.biaxial) {
        if (aniso) tally(ct, C_ANISO_BOUNCES);
        biaxial_media(P, S, kk, normal, cos_i, inside, aniso && inside && !(bits & F_IS_E), E);
    } else if (aniso) {
        tally(ct, C_ANISO_BOUNCES);
        float n_e_hero = n_o_hero + arr(P.ne_d4, 0);
        const float theta = theta_c<U>(kk, normal, cos_i, one_m_c2, n_o_hero, n_e_hero, ld3(S.c_axis), !inside);
        float2 sc = m_sincos(theta);
        const bool use_o = inside && !(bits & F_IS_E);
#pragma unroll U
        for (int k = 0; k < NCH; ++k) {
            float n_o = arr(P.n_o4, k);
            arr(E.n_med4, k) = use_o ? n_o : eff_e_index(n_o, n_o + arr(P.ne_d4, k), sc.x, sc.y);
        }
    } else if (!(K & K_ISO)) {
        E.n_med4[0] = P.n_o4[0];
        E.n_med4[1] = P.n_o4[1];
    }
    const float n_med0 = n_med<K>(P, E, 0);
    const float n1 = inside ? n_med0 : 1.0f;
    const float n2 = inside ? 1.0f : n_med0;
    const float eta0 = n1 / n2;
    const float sin2_t = eta0 * eta0 * one_m_c2;
    E.hp_cos = make_float4(hp.x, hp.y, hp.z, cos_i);

    // dispatch_bounce (transport.rs:158-176): hero TIR, or the Fresnel draw of
    // apply_partial_fresnel_bounce (refraction.rs:1049-1060)
    if (X && frosted_facet(S, fidx)) {
        frosted_bounce(P, S, hp, normal, inside, n1, n2, cos_i, sin2_t, ct);
        return EV_HANDLED;
    }
    bool tir = sin2_t > 1.0f;
    if (R && fabsf(sin2_t - 1.0f) < 1e-5f) {
        // near the critical angle: decide TIR in FP64 (refraction.rs:428-547 in double)
        const double ci = fmin(fmax(-((double)kk.x * normal.x + (double)kk.y * normal.y) - (double)kk.z * normal.z, 0.0), 1.0);
        const double eta = (double)n1 / (double)n2;
        tir = eta * eta * (1.0 - ci * ci) > 1.0;
    }
    if (tir) {
        E.n_ru = make_float4(normal.x, normal.y, normal.z, 0.0f);
        set_state_bits(P, bits | F_TIR);
        return EV_REFLECT;
    }
    float cos_t = sqrtf(R ? fmaxf(1.0f - sin2_t, 0.0f) : 1.0f - sin2_t);
    float rs, rp;
    fresnel_rs_rp(n1, n2, cos_i, cos_t, rs, rp);
    float ru = r_unpol(rs, rp);
    E.n_ru = make_float4(normal.x, normal.y, normal.z, ru);
    set_state_bits(P, bits & ~F_TIR);
    const bool refract = !(rng_draw(p_seed(P), bounce, FRESNEL_BRANCH_STREAM) < ru);
    // a biaxial entry in the fast mode (the split draw of apply_refract_bounce,
    // refraction.rs:781-789) refracts with the mode-A indices
    if (X && S.biaxial && refract && !inside && aniso &&
        !(rng_draw(p_seed(P), bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f))
        biaxial_fast_entry(P, S, kk, normal, cos_i, E);
    return refract ? EV_REFRACT : EV_REFLECT;
}

// Direction / state update after an event, internal mode coupling and Russian
// roulette (transport.rs:177-193,204-220,343-353,919-928).
template <class CT, int K = K_ANY>
__device__ __forceinline__ void step_post(Path &P, const SceneConst &S, V3 hp, V3 new_k, V3 new_s, bool new_inside,
                                          bool has_update, bool update_val, CT &ct) {
    uint32_t bits = state_bits(P);
    const uint32_t bounce = bits >> BOUNCE_SHIFT;
    const bool inside = (bits & F_INSIDE) != 0;
    const bool was_internal_reflection = inside && !has_update && new_inside == inside;
    set_xyz(P.d_seed, new_s);
    set_xyz(P.o_hero, add(hp, mul(new_s, 1e-4f)));
    set_xyz(P.k_state, new_k);
    bits = new_inside ? (bits | F_INSIDE) : (bits & ~F_INSIDE);
    if (has_update) bits = update_val ? (bits | F_IS_E) : (bits & ~F_IS_E);
    const uint32_t seed = p_seed(P);
    if (aniso_k<K>(S) && was_internal_reflection)
        bits = rng_draw(seed, bounce, MODE_COUPLING_STREAM) < 0.5f ? (bits | F_IS_E) : (bits & ~F_IS_E);
    if (bounce > 4) {
        tally(ct, C_ROULETTE);
        float mx = 0.0f;
#pragma unroll RR_UNROLL
        for (int k = 0; k < NCH; ++k) mx = fmaxf(mx, fmaxf(P.st[k].x, 0.0f));
        float q = clampf(mx, 0.05f, 1.0f);
        if (rng_draw(seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) {
            tally(ct, C_ROULETTE_KILLS);
            note_end(ct, bounce, GR_TERM_ROULETTE);
            set_state_bits(P, bits & ~F_ALIVE);
            return;
        }
        const float iq = 1.0f / q;
#pragma unroll RR_UNROLL
        for (int k = 0; k < NCH; ++k) {
            float4 s = P.st[k];
            P.st[k] = make_float4(s.x * iq, s.y * iq, s.z * iq, s.w * iq);
        }
    }
    const uint32_t nb = bounce + 1;
    bits = (bits & ((1u << BOUNCE_SHIFT) - 1u)) | (nb << BOUNCE_SHIFT);
    if (nb >= S.max_bounces) bits &= ~F_ALIVE;
    set_state_bits(P, bits);
}

// apply_frosted_bounce (raytracer/scattering.rs:522-602): a Lambertian lobe on either
// side of the facet, every channel depolarized; the forced (TIR) branch takes no pdf.
template <class CT>
__device__ __noinline__ void frosted_bounce(Path &P, const SceneConst &S, V3 hp, V3 normal, bool inside, float n1,
                                               float n2, float cos_i, float sin2_t, CT &ct) {
    const uint32_t bits = state_bits(P);
    const uint32_t bounce = bits >> BOUNCE_SHIFT;
    const uint32_t seed = p_seed(P);
    const float u1 = rng_draw(seed, bounce, FROSTED_DIR_U_STREAM);
    const float u2 = rng_draw(seed, bounce, FROSTED_DIR_V_STREAM);
    V3 nd;
    bool new_inside = inside, has_update = false, use_e = false;
    if (sin2_t > 1.0f) {
        note_event(ct, bounce, GR_SEQ_TIR);
        nd = cosine_weighted_hemisphere(u1, u2, normal);
#pragma unroll
        for (int k = 0; k < NCH; ++k) P.st[k] = make_float4(fmaxf(P.st[k].x, 0.0f), 0.0f, 0.0f, 0.0f);
    } else {
        const float c_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
        const float r_s = fmaf(n2, -c_t, n1 * cos_i) / fmaf(n2, c_t, n1 * cos_i);
        const float r_p = fmaf(n1, -c_t, n2 * cos_i) / fmaf(n1, c_t, n2 * cos_i);
        const float ru = clampf(0.5f * fmaf(r_p, r_p, r_s * r_s), 1e-4f, 1.0f - 1e-4f);
        if (rng_draw(seed, bounce, FRESNEL_BRANCH_STREAM) < ru) {
            note_event(ct, bounce, GR_SEQ_REFLECT);
            nd = cosine_weighted_hemisphere(u1, u2, normal);
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                P.st[k] = make_float4(fmaxf(P.st[k].x, 0.0f) / ru, 0.0f, 0.0f, 0.0f);
                arr(P.pdf4, k) = arr(P.pdf4, k) * ru;
            }
        } else {
            note_event(ct, bounce, GR_SEQ_REFRACT);
            nd = cosine_weighted_hemisphere(u1, u2, neg(normal));
            const bool entering_aniso = !inside && S.anisotropic;
            use_e = entering_aniso ? rng_draw(seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f : (bits & F_IS_E) != 0;
            has_update = entering_aniso;
            const float tu = 1.0f - ru;
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                P.st[k] = make_float4(fmaxf(P.st[k].x, 0.0f) / tu, 0.0f, 0.0f, 0.0f);
                arr(P.pdf4, k) = arr(P.pdf4, k) * tu;
            }
            new_inside = !inside;
        }
    }
    step_post(P, S, hp, nd, nd, new_inside, has_update, use_e, ct);
}

// apply_tir_bounce (refraction.rs:599-637) and apply_partial_reflect_bounce
// (refraction.rs:650-690) in one channel loop.
template <int U, class CT, bool X = false, int K = K_ANY>
__device__ __forceinline__ void step_reflect(Path &P, const SceneConst &S, const Event &E, CT &ct) {
    const uint32_t bits = state_bits(P);
    const bool inside = (bits & F_INSIDE) != 0;
    const bool hero_tir = (bits & F_TIR) != 0;
    const V3 hp = xyz(E.hp_cos), normal = xyz(E.n_ru), kk = xyz(P.k_state);
    const float cos_i = E.hp_cos.w;
    const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    const float sin_i = sqrtf(fmaxf(one_m_c2, 0.0f));
    if (hero_tir) tally(ct, C_TIR); else tally(ct, C_REFLECT);
    note_event(ct, bits >> BOUNCE_SHIFT, hero_tir ? GR_SEQ_TIR : GR_SEQ_REFLECT);
    // A TIR event applies each channel's matrix unscaled: the reflect branch's
    // `.scale(1 / r_unpol)` with factor 1.0 (x * 1.0f == x exactly).
    const float inv = hero_tir ? 1.0f : 1.0f / E.n_ru.w;
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        const float nm = n_med<K>(P, E, k);
        const float n1k = inside ? nm : 1.0f, n2k = inside ? 1.0f : nm;
        const float etak = n1k / n2k;
        const float s2k = etak * etak * one_m_c2;
        float4 s4 = P.st[k];
        Stokes s{s4.x, s4.y, s4.z, s4.w};
        if (s2k > 1.0f) {
            tally(ct, C_CH_TIR);
            float2 sc = m_sincos(tir_phase_delta(n1k, cos_i, sin_i));
            s = scale(apply_tir(s, sc.y, sc.x), inv);
        } else {
            float ctk = sqrtf(fmaxf(1.0f - s2k, 0.0f));
            float rsk, rpk, a, b, c;
            fresnel_rs_rp(n1k, n2k, cos_i, ctk, rsk, rpk);
            arr(P.pdf4, k) = arr(P.pdf4, k) * r_unpol(rsk, rpk);
            fresnel_reflection_abc(rsk, rpk, a, b, c);
            s = scale(apply_fresnel(s, a, b, c), inv);
        }
        P.st[k] = make_float4(s.i, s.q, s.u, s.v);
    }
    V3 new_k = sub(kk, smul(2.0f * dot(kk, normal), normal));
    // poynting_dir_for_mode (refraction.rs:564-582): both biaxial modes walk off
    V3 new_s = new_k;
    if (X && S.biaxial) {
        if (inside && S.anisotropic) new_s = mode_poynting_dir(S, make_ind(S, arr(P.n_o4, 0)), new_k, (bits & F_IS_E) != 0);
    } else if (inside && aniso_k<K>(S) && (bits & F_IS_E)) {
        float n_o_hero = arr(P.n_o4, 0);
        new_s = extraordinary_poynting_dir(new_k, ld3(S.c_axis), n_o_hero, n_o_hero + arr(P.ne_d4, 0));
    }
    step_post<CT, K>(P, S, hp, new_k, new_s, inside, false, false, ct);
}

// apply_refract_bounce (refraction.rs:748-867) + apply_refract_channel (:883-1011)
template <int U, class CT, bool X = false, int K = K_ANY>
__device__ __forceinline__ void step_refract(Path &P, const SceneConst &S, const Event &E, CT &ct) {
    const uint32_t bits = state_bits(P);
    const uint32_t bounce = bits >> BOUNCE_SHIFT;
    const bool inside = (bits & F_INSIDE) != 0;
    const bool aniso = aniso_k<K>(S);
    const V3 hp = xyz(E.hp_cos), normal = xyz(E.n_ru), kk = xyz(P.k_state);
    const float cos_i = E.hp_cos.w, ru = E.n_ru.w;
    const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    tally(ct, C_REFRACT);
    note_event(ct, bounce, GR_SEQ_REFRACT);
    const float n_med0 = n_med<K>(P, E, 0);
    const float n1 = inside ? n_med0 : 1.0f;
    const float n2 = inside ? 1.0f : n_med0;
    const float n_o_hero = arr(P.n_o4, 0);
    const float n_e_hero = (K & K_ISO) ? n_o_hero : n_o_hero + arr(P.ne_d4, 0);
    const bool entering_aniso = !inside && aniso;
    bool use_e = (bits & F_IS_E) != 0;
    if (entering_aniso) use_e = rng_draw(p_seed(P), bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f;
    // A biaxial entry (X only) refracts with the selected mode's indices, which step_hit
    // left in n_med4, and both of its modes walk off (refraction.rs:791-806,929-950).
    const bool biax_entry = X && S.biaxial && entering_aniso;
    const bool ordinary_entry = entering_aniso && !use_e && !biax_entry;
    const bool extra_entry = entering_aniso && use_e && !biax_entry;
    const float n2_dir = ordinary_entry ? n_o_hero : n2;
    const float eta_dir = n1 / n2_dir;
    const float s2d = fminf(eta_dir * eta_dir * one_m_c2, 1.0f);
    const float ctd = sqrtf(fmaxf(1.0f - s2d, 0.0f));
    const V3 refr = normalize(add(smul(eta_dir, kk), smul(fmaf(eta_dir, cos_i, -ctd), normal)));
    const V3 c_axis = ld3(S.c_axis);
    V3 final_dir = extra_entry ? extraordinary_poynting_dir(refr, c_axis, n_o_hero, n_e_hero) : refr;
    if (biax_entry) final_dir = mode_poynting_dir(S, make_ind(S, n_o_hero), refr, use_e);
    if (extra_entry) tally(ct, C_WALKOFF, 9);
    const float tinv = 1.0f / (1.0f - ru);
    const float TOL = 1.0f - 1e-6f;
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        const float n_o_k = arr(P.n_o4, k);
        const float n1k = inside ? n_med<K>(P, E, k) : 1.0f;
        const float n2k = ordinary_entry ? n_o_k : (inside ? 1.0f : n_med<K>(P, E, k));
        const float ratio = n1k / n2k;
        const float s2k = (ratio * ratio) * one_m_c2;
        float4 s4 = P.st[k];
        Stokes s{s4.x, s4.y, s4.z, s4.w};
        bool keep = false;
        float ctk = 0.0f;
        if (!(s2k > 1.0f)) {
            tally(ct, C_CH_REFR);
            ctk = sqrtf(fmaxf(1.0f - s2k, 0.0f));
            V3 rk = normalize(add(smul(ratio, kk), smul(fmaf(ratio, cos_i, -ctk), normal)));
            V3 fk = extra_entry ? extraordinary_poynting_dir(rk, c_axis, n_o_k, n_o_k + arr(P.ne_d4, k)) : rk;
            if (biax_entry) fk = mode_poynting_dir(S, make_ind(S, n_o_k), rk, use_e);
            keep = dot(fk, final_dir) >= TOL;
        }
        if (keep) {
            float ts = (2.0f * n1k * cos_i) / fmaf(n2k, ctk, n1k * cos_i);
            float tp = (2.0f * n1k * cos_i) / fmaf(n1k, ctk, n2k * cos_i);
            float a, b, c;
            fresnel_transmission_abc(n1k, n2k, cos_i, ctk, ts, tp, a, b, c);
            s = scale(apply_fresnel(s, a, b, c), tinv);
            float rsk, rpk;
            fresnel_rs_rp(n1k, n2k, cos_i, ctk, rsk, rpk);
            arr(P.pdf4, k) = arr(P.pdf4, k) * (1.0f - r_unpol(rsk, rpk));
        } else {
            // chromatic termination / channel cannot transmit (refraction.rs:919-927,1006-1009)
            s = scale(s, 0.0f);
            arr(P.pdf4, k) = 0.0f;
        }
        P.st[k] = make_float4(s.i, s.q, s.u, s.v);
    }
    step_post<CT, K>(P, S, hp, refr, final_dir, !inside, entering_aniso, use_e, ct);
}

// Escape radiance, spectral MIS and CIE integration (transport.rs:67-90,931-939,
// raytracer/color.rs:122-164) for a finished path.  STOKES: also the luminance-weighted
// Stokes vector of the escaping light, iquv = sum_k ybar(lambda_k) * (S_k * env_k * w)
// * norm in channel order (I with the intensity clamp of the XYZ sum, so iquv.x equals
// the XYZ sum's Y before white balance bit for bit; Q, U, V in the frame of the last
// plane of incidence).
template <int U = 1, bool STOKES = false, int K = K_ANY>
__device__ __forceinline__ V3 path_finish(const Path &P, const SceneConst &S, const SceneBuffers &B,
                                          float4 *iquv = nullptr) {
    const uint32_t env_mode = env_k<K>(S);
    float sum = -0.0f;
#pragma unroll
    for (int k = 0; k < NCH; ++k) sum = sum + arr(P.pdf4, k);
    const float w = sum <= 1e-12f ? 1.0f : 8.0f * arr(P.pdf4, 0) / sum;
    const float norm = (400.0f / 8.0f) / 106.856f;
    const bool escaped = (p_flags(P) & F_ESCAPED) != 0;
    const float hero = p_hero(P);
    const V3 dir = xyz(P.d_seed);
    float rgb[3] = {0.0f, 0.0f, 0.0f};
    V3 dn = v3(0.f, 0.f, 0.f);
    if (escaped) {
        if (env_mode == GR_ENV_STUDIO) {
            dn = normalize(dir);
        } else if (env_mode == GR_ENV_UNIFORM) {
            rgb[0] = S.uni_rgb[0]; rgb[1] = S.uni_rgb[1]; rgb[2] = S.uni_rgb[2];
        } else {
            latlong_rgb(S, B.map, dir, rgb);
        }
    }
    V3 acc = v3(0.f, 0.f, 0.f);
    float4 sk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll U
    for (int k = 0; k < NCH; ++k) {
        const float lam = lambda_k(hero, k);
        float rad = 0.0f, q = 0.0f, u = 0.0f, v = 0.0f;
        if (escaped) {
            float env = env_mode == GR_ENV_STUDIO ? studio_radiance(S, dn, lam)
                                                     : rgb_to_spectral(rgb[0], rgb[1], rgb[2], lam);
            rad = fmaf(fmaxf(P.st[k].x, 0.0f), env, 0.0f);
            if (STOKES) {
                q = P.st[k].y * env;
                u = P.st[k].z * env;
                v = P.st[k].w * env;
            }
        }
        float wr = rad * w;
        const V3 c = cmf(lam);
        acc = add(acc, mul(c, wr * norm));
        if (STOKES) {
            sk.x = sk.x + c.y * (wr * norm);
            sk.y = sk.y + c.y * ((q * w) * norm);
            sk.z = sk.z + c.y * ((u * w) * norm);
            sk.w = sk.w + c.y * ((v * w) * norm);
        }
    }
    if (STOKES) *iquv = sk;
    return von_kries(acc, S.wb);
}

// One whole path in the calling thread (the plain kernel's body).
template <class CT, bool R = false, bool X = false, int K = K_ANY>
__device__ __forceinline__ V3 trace_path(Path &P, const SceneConst &S, const SceneBuffers &B, const Planes &PL,
                                         CT &ct) {
    while (state_bits(P) & F_ALIVE) {
        Event E;
        uint32_t ev = step_hit<1, CT, R, X, K>(P, S, PL, E, ct);
        if (ev == EV_REFLECT) step_reflect<1, CT, X, K>(P, S, E, ct);
        else if (ev == EV_REFRACT) step_refract<1, CT, X, K>(P, S, E, ct);
    }
    return path_finish<1, false, K>(P, S, B);
}

}  // namespace grd
