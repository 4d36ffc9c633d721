/*
 * gemray_cuda.h -- C ABI of the B200 spectral-transport engine.
 *
 * This is the drop-in boundary for gemray's `gpu`-feature render path.  Every entry
 * point below replaces one item of the reference's Rust GPU backend; the comment
 * above each declaration names the reference item (path:line inside the
 * gemray-studio workspace) whose contract it keeps.
 *
 * Conventions
 *   - Plain C: fixed-width integers, float, pointers and sizes.  No CUDA or torch
 *     types appear in any signature; streams are passed as `void*` (a cudaStream_t).
 *   - Every call returns a gr_status.  Nothing aborts the process; a failing call
 *     leaves caller buffers untouched and records a message readable through
 *     gr_last_error_string().
 *   - Struct layouts are frozen (see the static asserts at the end of this file).
 *     gr_plane, gr_band and gr_material are byte-identical to the reference's
 *     `GpuFacetPlane`, `GpuAbsorptionBand` and `GpuGemMaterial`
 *     (crates/gemray/src/geometry/plane.rs:6-9, renderer/buffers.rs:148-165,236-299),
 *     so a Rust caller can pass `bytemuck::bytes_of(&GpuGemMaterial::encode(m))`.
 *   - Calls on one context are serialised by its mutex, and its device scratch (the
 *     per-tuple XYZ chunk, the staged kernels' park records, batch tables) is reused
 *     call after call in stream order.  Work a caller queues on its own streams must
 *     therefore be ordered with the context's other work on the device (one stream,
 *     or events).  The request loop queues on the context stream; frame streams own
 *     their scratch and streams.
 */
#ifndef GEMRAY_CUDA_H
#define GEMRAY_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GR_ABI_VERSION 1u
/* Per-band-set limit, = MAX_ABSORPTION_BANDS (renderer/buffers.rs:148). */
#define GR_MAX_BANDS 8u
/* Largest facet-plane count a scene may carry (planes are staged in shared memory). */
#define GR_MAX_PLANES 512u
/* Largest bounce cap accepted (= worker MAX_BOUNCES, apps/gemray-worker/src/validate/mod.rs). */
#define GR_MAX_BOUNCES 4096u

/* Status codes.  GR_DECLINED_* mirror GpuFrameError (renderer/gpu/frame.rs:196-210):
 * they mean "render this on the CPU tracer instead", exactly like a `false` from
 * GpuBackend::try_accumulate (renderer/gpu_backend.rs:160-193).  Every environment
 * kind and material kind of the reference's render path is handled on the device, so
 * neither is returned at present; they stay part of the contract. */
typedef enum gr_status {
    GR_OK = 0,
    GR_DECLINED_ENV = 1,      /* environment kind not handled on the device */
    GR_DECLINED_MATERIAL = 2, /* material kind not handled on the device */
    GR_NO_DEVICE = 3,         /* no usable CUDA device (GpuAcquireError) */
    GR_EINVAL = 4,            /* bad argument (length mismatch, null pointer, limits) */
    GR_ENOMEM = 5,            /* device or pinned-host allocation failed */
    GR_ETIMEOUT = 6,          /* a bounded wait ran out */
    GR_ECANCELLED = 7,        /* request cancelled before completion */
    GR_ECUDA = 8,             /* CUDA runtime error; see gr_last_error_string() */
    GR_EBUSY = 9,             /* admission refused: device-memory budget exhausted */
    GR_ENOTFOUND = 10         /* unknown scene or request id */
} gr_status;

/* One half-space: inside <=> dot(normal, x) + d <= 0.  = GpuFacetPlane. */
typedef struct gr_plane {
    float normal[3];
    float d;
} gr_plane;

/* One Gaussian absorption band.  = GpuAbsorptionBand. */
typedef struct gr_band {
    float center_nm;
    float width_nm;
    float peak;
} gr_band;

/* Dispersion model ids, = dispersion_model_type (renderer/buffers.rs:117-121). */
#define GR_DISP_SELLMEIER1 0u
#define GR_DISP_SELLMEIER3 1u
#define GR_DISP_CAUCHY 2u

/* = DispersionParams (renderer/buffers.rs:84-99).  Sellmeier1: a=[b1], b=[c1];
 * Sellmeier3: a=b[0..3], b=c[0..3]; Cauchy: a=[A, B, C].  c_axis_and_birefringence
 * = (c_axis.xyz, n_e - n_o). */
typedef struct gr_dispersion {
    uint32_t model_type;
    uint32_t pad0[3];
    float param_a[4];
    float param_b[4];
    float param_c[4];
    float c_axis_and_birefringence[4];
    uint32_t is_anisotropic;
    float biaxial_delta_beta_alpha;
    uint32_t has_biaxial_delta;
    float pad_tail;
} gr_dispersion;

/* Crystal-system ids, = crystal_system (renderer/buffers.rs:170-178). */
#define GR_CRYSTAL_CUBIC 0u

/* = GpuGemMaterial (renderer/buffers.rs:236-299), 432 bytes. */
typedef struct gr_material {
    gr_dispersion dispersion;
    uint32_t crystal_system;
    uint32_t optical_character;
    uint32_t is_pleochroic;
    uint32_t o_ray_band_count;
    uint32_t e_ray_band_count;
    gr_band o_ray_bands[GR_MAX_BANDS];
    gr_band e_ray_bands[GR_MAX_BANDS];
    float scattering_sigma_s;  /* > 0: Henyey-Greenstein volume scattering inside the stone
                                  (maybe_scatter_or_extinguish, optics/raytracer/scattering.rs:132) */
    float scattering_g;        /* HG asymmetry, > 0 forward */
    float edge_rounding_radius;
    uint32_t has_beta_ray;
    uint32_t beta_ray_band_count;
    gr_band beta_ray_bands[GR_MAX_BANDS];
    float absorption_path_scale;
    uint32_t pad_trailing;
} gr_material;

/* Pinhole camera, = optics::raytracer::Camera (optics/raytracer/camera.rs:53-59).
 * The host builds it (Camera::new uses libm sin/cos/tan); the device only reads it. */
typedef struct gr_camera {
    float origin[3];
    float forward[3];
    float right[3];
    float up[3];
    float fov_tan;
} gr_camera;

/* Environment kinds.  UNIFORM is EnvironmentMap::uniform (renderer/env_map.rs:163-168),
 * STUDIO is EnvironmentSource::Studio (optics/raytracer/environment.rs:187-196),
 * LATLONG is EnvironmentSource::HdrMap over an RGB f32 lat-long map. */
#define GR_ENV_UNIFORM 0u
#define GR_ENV_STUDIO 1u
#define GR_ENV_LATLONG 2u

typedef struct gr_environment {
    uint32_t mode;
    /* GR_ENV_UNIFORM: the map's single RGB radiance. */
    float uniform_rgb[3];
    /* GR_ENV_STUDIO: LightingPreset::params() (temp_k, spot_mult) plus the pose. */
    float temp_k;
    float spot_mult;
    float exposure;
    float light_yaw;
    float light_pitch;
    /* GR_ENV_LATLONG: row-major RGB f32 texels, latlong_w * latlong_h * 3 floats,
     * row 0 at the +Y pole (v = 0).  Borrowed for the duration of the call. */
    const float *latlong_rgb;
    uint32_t latlong_w;
    uint32_t latlong_h;
} gr_environment;

/* Optional extension material data (not in the reference model): tabulated
 * absorption and a wavelength-dependent birefringence.  Pass NULL for reference
 * behaviour.  Tables are sampled at nm_first + i * nm_step and linearly
 * interpolated (clamped at the ends). */
typedef struct gr_material_ext {
    uint32_t n_absorption;      /* entries per table, 0 = use the Gaussian bands */
    float absorption_nm_first;
    float absorption_nm_step;
    const float *alpha_o_table; /* n_absorption values */
    const float *alpha_e_table; /* n_absorption values */
    uint32_t has_cauchy_e;      /* 1 = n_e from its own Cauchy fit below */
    float cauchy_e[3];          /* n_e(lambda) = a + b/l^2 + c/l^4, lambda in um */
} gr_material_ext;

/* Scene flags. */
#define GR_FLAG_KAHAN_FILM 0x1u /* compensated per-pixel sample sum (default: plain f32 in sample order) */
/* FP64 re-solve of ambiguous f32 decisions (an extension, off by default): a ray whose
 * f32 exit facet is within 1e-5 (relative) of another plane's, or of the other side's
 * extremum, is re-clipped in FP64, and a hero TIR decision with |sin^2(t) - 1| < 1e-5
 * is re-made in FP64.  Results then differ from the reference's f32 tracer on those
 * few rays (towards the FP64 result).  Single-scene calls only (gr_accumulate*,
 * gr_render_resident*, gr_trace_samples); gr_render_batch and gr_submit reject it. */
#define GR_FLAG_FP64_RESOLVE 0x2u

/* One render scene, = GpuSceneRef (renderer/gpu_backend.rs:85-99).  Every pointer is
 * borrowed for the duration of the call. */
typedef struct gr_scene {
    gr_camera camera;
    uint32_t width;
    uint32_t height;
    uint32_t max_bounces;
    uint32_t n_planes;
    const gr_plane *planes;    /* n_planes entries */
    const uint32_t *finishes;  /* NULL or n_planes entries: 0 = polished, 1 = frosted (diffuse
                                  reflect/transmit, apply_frosted_bounce, optics/raytracer/
                                  scattering.rs:522-602) */
    const gr_material *material;
    const gr_material_ext *material_ext; /* NULL = reference material model */
    gr_environment env;
    uint32_t flags;
    uint32_t reserved;
} gr_scene;

/* Context creation options (NULL = defaults). */
typedef struct gr_create_opts {
    int32_t device;               /* CUDA device ordinal, -1 = current/0 */
    uint64_t chunk_budget_bytes;  /* per-launch scratch budget, 0 = default (2 GiB) */
    uint64_t serve_budget_bytes;  /* device-memory budget for resident scenes/films, 0 = 60 GiB */
} gr_create_opts;

typedef struct gr_ctx gr_ctx;

/* ---- backend lifecycle ------------------------------------------------------ */

/* Replaces GpuBackend::acquire / GpuFrameRenderer::new (renderer/gpu_backend.rs:114-126,
 * renderer/gpu/frame.rs:574-594).  On failure *out is NULL and GR_NO_DEVICE/GR_ECUDA
 * is returned; the caller then behaves like GpuBackend::disabled(). */
gr_status gr_create(gr_ctx **out, const gr_create_opts *opts);

/* Releases every device resource owned by the context.  NULL is accepted. */
gr_status gr_destroy(gr_ctx *ctx);

/* Replaces GpuBackend::adapter_label (renderer/gpu_backend.rs:146-153): a
 * NUL-terminated device description owned by the context. */
const char *gr_device_label(gr_ctx *ctx);

/* Message for the most recent failing call on this thread ("" if none). */
const char *gr_last_error_string(void);

/* ABI version of the loaded library (GR_ABI_VERSION at build time). */
uint32_t gr_abi_version(void);

/* ---- the render path -------------------------------------------------------- */

/* Replaces GpuBackend::try_accumulate -> GpuFrameRenderer::accumulate
 * (renderer/gpu_backend.rs:160-193, renderer/gpu/frame.rs:632-647,664-814).
 * Traces samples [sample_offset, sample_offset + spp) of every pixel and ADDS each
 * pixel's sample sum (summed in sample order, then added once) into accum_xyz, a
 * host array of width*height*3 floats (Vec3 per pixel).  spp == 0 or an empty frame
 * is a no-op returning GR_OK.  A declined scene leaves accum_xyz untouched. */
gr_status gr_accumulate(gr_ctx *ctx, const gr_scene *scene, uint32_t sample_offset,
                        uint32_t spp, float *accum_xyz);

/* As gr_accumulate, but accum_xyz is a DEVICE pointer (width*height*3 floats) and the
 * work is enqueued on `stream` (a cudaStream_t, NULL = the context's stream).  The
 * call returns once the work is enqueued; scene data is uploaded first. */
gr_status gr_accumulate_device(gr_ctx *ctx, const gr_scene *scene, uint32_t sample_offset,
                               uint32_t spp, float *accum_xyz_device, void *stream);

/* Per-sample XYZ for samples [sample_offset, sample_offset + spp) of pixels
 * [first_pixel, first_pixel + n_pixels) into a host array of n_pixels*spp*3 floats,
 * ordered (pixel, sample) -- the reference kernel's per-tuple output layout
 * (renderer/shaders/spectral_transport.wgsl:672-691).  Used by parity tests. */
gr_status gr_trace_samples(gr_ctx *ctx, const gr_scene *scene, uint32_t first_pixel,
                           uint32_t n_pixels, uint32_t sample_offset, uint32_t spp,
                           float *xyz_out);

/* gr_accumulate plus a Stokes film (no counterpart in the reference, whose film is XYZ
 * only, renderer/gpu/frame.rs:799-814; the transport's per-channel StokesVector state,
 * optics/polarization.rs:4-66, is otherwise dropped when a path ends).  accum_xyz
 * (W*H*3) receives exactly what gr_accumulate adds; accum_stokes (W*H*4, host) receives
 * each pixel's sample-order sum of the luminance-weighted Stokes vector of the light
 * that escapes:  (I, Q, U, V) = sum_k ybar(lambda_k) * w * norm * env_k * S_k  over the
 * 8 hero channels, with the XYZ sum's spectral-MIS weight w, normaliser and intensity
 * clamp, so I equals that sum's Y before white balance.  Q, U, V are in the frame of
 * the last plane of incidence; every per-sample vector has sqrt(Q^2+U^2+V^2) <= I up to
 * rounding.  Plain kernel; not with GR_FLAG_FP64_RESOLVE. */
gr_status gr_accumulate_stokes(gr_ctx *ctx, const gr_scene *scene, uint32_t sample_offset, uint32_t spp,
                               float *accum_xyz, float *accum_stokes);

/* Device-side tone map: rgba[i] = ColorSpace::Srgb.encode(xyz[i] * scale, ACES)
 * (renderer/tonemap.rs:52-108, color/space.rs:290-334).  Host arrays. */
gr_status gr_tonemap(gr_ctx *ctx, const float *xyz, float scale, uint32_t n_px,
                     uint8_t *rgba);

/* ---- verification hooks --------------------------------------------------------- */

/* One sampler record, the device analogue of the reference's RngRecord
 * (renderer/gpu/rng_check.rs:54-109, shaders/rng_equivalence.wgsl:154): the per-sample
 * seed and stratified draws (optics/raytracer/sampling.rs:232-271) and, for bounces
 * 0..3, the Fresnel, Russian-roulette, birefringent-split and mode-coupling draws. */
typedef struct gr_rng_record {
    uint32_t seed;
    float jitter_x;
    float jitter_y;
    float hero_rand;
    float draws[4][4]; /* [bounce][fresnel, roulette, split, coupling] */
} gr_rng_record;

/* Device sampler records for n (pixel, sample) pairs (host arrays). */
gr_status gr_rng_records(gr_ctx *ctx, const uint32_t *pixels, const uint32_t *samples, uint32_t n,
                         gr_rng_record *out);

/* Event tallies of an instrumented launch over samples [sample_offset, +spp) of pixels
 * [first_pixel, +n_pixels) -- the inputs of the algorithmic FLOP model (extends
 * trace_spectral_ray_with_finish_instrumented, optics/raytracer/transport.rs:512-537).
 * counts[GR_EVENT_*] must hold GR_EVENT_COUNT entries. */
#define GR_EVENT_PATHS 0u
#define GR_EVENT_BOUNCES 1u        /* intersection tests (including the final miss) */
#define GR_EVENT_ESCAPES 2u
#define GR_EVENT_TIR 3u
#define GR_EVENT_REFLECT 4u
#define GR_EVENT_REFRACT 5u
#define GR_EVENT_ABSORB 6u         /* interior segments with Beer-Lambert absorption */
#define GR_EVENT_CHANNEL_TIR 7u    /* per-channel TIR phase evaluations */
#define GR_EVENT_CHANNEL_REFRACT 8u
#define GR_EVENT_ROULETTE 9u
#define GR_EVENT_ROTATIONS 10u     /* Stokes frame rotations */
#define GR_EVENT_ANISO_BOUNCES 11u
#define GR_EVENT_WALKOFF 12u
#define GR_EVENT_ROULETTE_KILLS 13u
#define GR_EVENT_COUNT 14u
gr_status gr_event_counts(gr_ctx *ctx, const gr_scene *scene, uint32_t first_pixel, uint32_t n_pixels,
                          uint32_t sample_offset, uint32_t spp, uint64_t *counts, uint32_t n_counts);

/* Measured dense FP32 FMA throughput of the device (TFLOP/s), the roofline
 * denominator of the transport kernels. */
gr_status gr_probe_fp32_peak(gr_ctx *ctx, double *tflops);

/* Per-tuple event sequence of the transport -- the device side of the reference's
 * instrumented trace (trace_spectral_ray_with_finish_instrumented,
 * optics/raytracer/transport.rs:512-537, whose log the facet-sequence check of
 * renderer/gpu/polyhedron_check.rs compares per hit).  For each tuple of samples
 * [sample_offset, +spp) of pixels [first_pixel, +n_pixels), in (pixel, sample) order:
 *   bounces[t]       the bounce index the path ended at (max_bounces at the cap);
 *   termination[t]   GR_TERM_*;
 *   facets[t*kmax+b] the facet hit at bounce b, t_hits[t*kmax+b] its distance, and
 *   events[t*kmax+b] the GR_SEQ_* event taken there, for b < min(kmax, recorded),
 *                    recorded = bounces + (termination == GR_TERM_ROULETTE); slots past
 *                    that hold -1 / 0 / 0xFF.
 * Host arrays.  The plain kernel with recording hooks runs the same functions in the
 * same order as every other transport kernel, so its sequences are theirs. */
#define GR_TERM_ESCAPED 0u
#define GR_TERM_ROULETTE 2u
#define GR_TERM_HIT_CAP 3u
#define GR_SEQ_TIR 0u
#define GR_SEQ_REFLECT 1u
#define GR_SEQ_REFRACT 2u
#define GR_SEQ_SCATTER 3u
#define GR_SEQ_NONE 0xFFu
gr_status gr_trace_events(gr_ctx *ctx, const gr_scene *scene, uint32_t first_pixel, uint32_t n_pixels,
                          uint32_t sample_offset, uint32_t spp, uint32_t kmax, uint32_t *bounces,
                          uint32_t *termination, int32_t *facets, float *t_hits, uint8_t *events);

/* Per-function case banks: the device functions the transport kernels inline, run one
 * case per thread over caller inputs -- the counterpart of the reference's Tier-2
 * per-function checks (renderer/gpu/transport_check/mod.rs:38-75, camera_check.rs,
 * environment_check.rs), which hold each function to a ULP budget.  `in` holds n rows
 * of n_in floats, `out` receives n rows of n_out floats (gr_case_bank_arity).  Banks
 * that read scene state take it from `scene` (camera and frame size, material,
 * environment); the others ignore it (NULL allowed).  Host arrays. */
#define GR_BANK_CAMERA_RAY 0u           /* x, y, jitter_x, jitter_y -> dir[3]; scene camera + frame */
#define GR_BANK_CMF 1u                  /* lambda -> xyz[3] (cie_1931_cmf_x8 lane) */
#define GR_BANK_BLACKBODY 2u            /* lambda -> blackbody_spectrum at scene env temp_k */
#define GR_BANK_DISPERSION 3u           /* lambda -> n (scene material dispersion) */
#define GR_BANK_ABSORPTION 4u           /* lambda -> alpha_o, alpha_e (bands or extension table) */
#define GR_BANK_PLEOCHROIC 5u           /* stokes[4], s_axis[3], k[3], a_o, a_e -> alpha (scene c-axis) */
#define GR_BANK_FRESNEL_REFLECTION 6u   /* r_s, r_p, stokes[4] -> stokes[4] */
#define GR_BANK_FRESNEL_TRANSMISSION 7u /* n1, n2, cos_i, cos_t, t_s, t_p, stokes[4] -> stokes[4] */
#define GR_BANK_FRAME_ROTATION 8u       /* psi, stokes[4] -> stokes[4] */
#define GR_BANK_TIR_RETARDATION 9u      /* delta, stokes[4] -> stokes[4] */
#define GR_BANK_SIGNED_PSI 10u          /* prev[3], cur[3], k[3] -> psi */
#define GR_BANK_TIR_PHASE_DELTA 11u     /* n1, cos_i, sin_i -> delta */
#define GR_BANK_EIGEN_UNIAXIAL 12u      /* k[3], c[3] -> ordinary[3], extraordinary[3] */
#define GR_BANK_WALK_OFF 13u            /* k[3], c[3], n_o, n_e -> extraordinary Poynting dir[3] */
#define GR_BANK_EXTRAORDINARY_INDEX 14u /* n_o, n_e, theta -> n_eff */
#define GR_BANK_THETA_C 15u             /* k[3], normal[3], n_o, n_e, entry -> theta (scene c-axis) */
#define GR_BANK_STUDIO 16u              /* dir[3], lambda -> radiance (scene studio environment) */
#define GR_BANK_RGB_SPECTRAL 17u        /* r, g, b, lambda -> rgb_to_spectral_radiance */
#define GR_BANK_EXP_POLY 18u            /* x -> simd::exp_f32x8 lane */
#define GR_BANK_HG_SAMPLE 19u           /* u1, u2, g, fwd[3] -> dir[3] */
#define GR_BANK_COSINE_HEMISPHERE 20u   /* u1, u2, n[3] -> dir[3] */
#define GR_BANK_E_FIELD 21u             /* stokes[4], s_axis[3], k[3] -> electric_field_direction[3] */
#define GR_BANK_VON_KRIES 22u           /* xyz[3] -> white-balanced xyz[3] (scene environment) */
#define GR_BANK_WAVELENGTHS 23u         /* hero_rand -> lambda[8] (wrapped_hero_wavelengths) */
#define GR_BANK_COUNT 24u
gr_status gr_case_bank_arity(uint32_t bank, uint32_t *n_in, uint32_t *n_out);
gr_status gr_case_bank(gr_ctx *ctx, uint32_t bank, const gr_scene *scene, const float *in, uint32_t n, float *out);

/* The compute capability the library's device code was built for, as the CUDA runtime
 * reports it for a kernel of this library on the context's device
 * (cudaFuncGetAttributes): binary_version 100 for the sm_100a cubin, ptx_version 0
 * when no PTX is embedded. */
gr_status gr_device_code_version(gr_ctx *ctx, uint32_t *binary_version, uint32_t *ptx_version);

/* The transport's convex clip (the paired shared-memory plane scan of every transport
 * kernel) for n rays, rays[6*i..] = origin[3], dir[3]: t[i] and facet[i] (-1 on a
 * miss) -- the device side of renderer/gpu/polyhedron_check.rs's case bank for
 * intersect_polyhedron (optics/raytracer/intersect.rs:93-132).  Host arrays. */
gr_status gr_intersect_rays(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const float *rays, uint32_t n,
                            float *t, int32_t *facet);

/* ---- optical metrics ------------------------------------------------------------ */

/* = GemOpticalMetrics (color/metrics.rs:33-39). */
typedef struct gr_metrics_out {
    float brilliance_pct;
    float fire_index;
    float scintillation_pct;
    float windowing_pct;
    float extinction_pct;
} gr_metrics_out;

/* One viewing pose (radians), the four scalar arguments of
 * evaluate_gem_optical_metrics. */
typedef struct gr_pose {
    float cam_yaw;
    float cam_pitch;
    float light_yaw;
    float light_pitch;
} gr_pose;

/* Form the fire / scintillation sums in f64 instead of the reference's f32 running
 * sums (counts are exact either way). */
#define GR_METRICS_FP64_SUMS 0x1u

/* evaluate_gem_optical_metrics (color/metrics.rs:1082-1237) for n_poses poses in one
 * device pass: one thread per (pose, 18x18 grid cell, aperture ray or temporal yaw
 * offset), then a per-pose reduction in the reference's cell order.  Classification
 * counts (brilliance, windowing, extinction, the cells' return fractions) are the
 * reference's exactly; fire can differ in its last bits through acosf.  n_planes == 0
 * gives the reference's placeholder values (85, 25, 75, 5, 5). */
gr_status gr_optical_metrics(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const gr_material *material,
                             const gr_pose *poses, uint32_t n_poses, uint32_t flags, gr_metrics_out *out);

/* evaluate_angular_profile_at_azimuth (color/metrics.rs:1262-1289): the 19 tilt
 * elevations 0, 5, ..., 90 degrees (pitch = deg * (pi / 180) in f32, as
 * f32::to_radians) as one batch; writes 19 values to each curve. */
gr_status gr_angular_profile(gr_ctx *ctx, const gr_plane *planes, uint32_t n_planes, const gr_material *material,
                             float cam_yaw, float light_yaw, float light_pitch, float *brilliance_19,
                             float *extinction_19, float *windowing_19);

/* ---- resident scenes (serving / benchmarks) ------------------------------------- */

/* Copies a scene to the device once (planes, map, tables, encoded constants) and
 * returns its id.  GR_EBUSY if it does not fit the context's serve budget.  Mirrors
 * the reference worker keeping a scene across sub-batches
 * (apps/gemray-worker/src/stream_emit/tracer.rs:64). */
gr_status gr_scene_upload(gr_ctx *ctx, const gr_scene *scene, uint64_t *scene_id);
gr_status gr_scene_release(gr_ctx *ctx, uint64_t scene_id);

/* gr_accumulate_device for a resident scene: no host data is read. */
gr_status gr_render_resident(gr_ctx *ctx, uint64_t scene_id, uint32_t sample_offset, uint32_t spp,
                             float *film_device, void *stream);

/* ---- batched launches ------------------------------------------------------------ */

/* One scene's sample range in a batched render: ADD samples [sample_offset,
 * sample_offset + spp) of every pixel of a resident scene into film_device
 * (W*H*3 f32 on the context's device). */
typedef struct gr_batch_item {
    uint64_t scene_id;
    float *film_device;
    uint32_t sample_offset;
    uint32_t spp;
} gr_batch_item;

/* Capture the batch's launch sequence as a CUDA graph and replay it whenever the same
 * batch shape (scenes, films, spp, frame sizes) recurs; sample offsets may change. */
#define GR_BATCH_GRAPH 0x1u

/* Renders all items (no counterpart in the reference, whose frame renderer takes one
 * scene per dispatch, renderer/gpu/frame.rs:632-814): items under 2 M path-samples --
 * scenes of any plane count, material and frame size -- are packed into shared
 * launches of at most the context's chunk budget of per-tuple scratch (GR_BATCH_GRAPH
 * applies to these); larger items, which fill the device on their own, render with
 * the single-scene kernels and their stone's tuned schedule, as gr_render_resident
 * does, before them.  Each film is bit-identical to gr_render_resident of its item
 * alone.  Work is queued on `stream` (NULL = the context stream) and the call returns
 * without waiting for it. */
gr_status gr_render_batch(gr_ctx *ctx, const gr_batch_item *items, uint32_t n_items, uint32_t flags, void *stream);

/* ---- serving: render requests over resident scenes ------------------------------ */

/* Request kinds. */
#define GR_REQ_RENDER 0u  /* ADD samples [sample_offset, sample_offset + spp) into a fresh film */
#define GR_REQ_METRICS 1u /* a brilliance/fire/scintillation pose sweep (gr_optical_metrics) */

/* One request, = RenderRequest{request_id, first_sample, samples}
 * (crates/gemray-net/src/messages/render.rs:65-70) for a resident scene, or a metric
 * sweep.  Pointers are copied at submit. */
typedef struct gr_request {
    uint32_t kind;
    uint32_t slice_spp;      /* render: > 0: at most this many samples per pixel per tick (a tick
                                carries ~8.4 M path-samples in one batched launch, filled from the
                                running sliced renders in arrival order); progress and cancellation
                                happen between slices.  0: rendered by the render lane in chunks
                                (see gr_submit).  The film does not depend on either */
    uint64_t scene_id;       /* render: resident scene */
    uint32_t sample_offset;  /* render: first absolute sample */
    uint32_t spp;            /* render: samples per pixel */
    uint32_t flags;          /* metrics: GR_METRICS_* */
    uint32_t n_planes;       /* metrics */
    const gr_plane *planes;  /* metrics */
    const gr_material *material; /* metrics */
    const gr_pose *poses;    /* metrics */
    uint32_t n_poses;        /* metrics */
    uint32_t reserved;
} gr_request;

/* Request states. */
#define GR_REQ_QUEUED 0u
#define GR_REQ_RUNNING 1u
#define GR_REQ_DONE 2u
#define GR_REQ_CANCELLED 3u
#define GR_REQ_FAILED 4u

typedef struct gr_request_status {
    uint32_t state;         /* GR_REQ_* */
    uint32_t samples_done;  /* render: samples per pixel folded into the film so far */
    gr_status error;        /* GR_REQ_FAILED: why (GR_EBUSY = can never fit the memory budget) */
    uint32_t reserved;
    double queued_ms;       /* submit -> admission */
    double latency_ms;      /* submit -> finished (0 while active) */
} gr_request_status;

/* Queues a request and returns at once (no counterpart in the reference's GPU path,
 * which renders one dispatch at a time; the worker's render loop is
 * apps/gemray-worker/src/render_core/mod.rs).  A worker thread admits requests in
 * arrival order while their film (W*H*3 f32) fits the context's serve budget next to
 * the resident scenes and unreleased films.  A render with slice_spp == 0 goes to the
 * render lane, which renders it in chunks of whole pixels (16 M path-samples) with the
 * single-scene kernels and the stone's tuned schedule, choosing after every chunk the
 * render that comes first by submission time plus remaining work: a small request
 * waits about one chunk behind a large one instead of all of it, and a large one that
 * has waited longer than a newer request's whole work goes first.  A sliced render
 * (slice_spp > 0) advances by one slice per tick in a shared batched launch beside the
 * lane.  Metric requests hold no film and run on another worker thread in
 * arrival order at the highest stream priority, beside the renders.  Slices continue
 * each pixel's running sum, so a film is bit-identical to one gr_render_resident call
 * over the same sample range on a zero film -- lane or ticks, for any slicing, alone
 * or in any mix. */
gr_status gr_submit(gr_ctx *ctx, const gr_request *request, uint64_t *request_id);
gr_status gr_poll(gr_ctx *ctx, uint64_t request_id, gr_request_status *status);
/* Blocks until the request has finished or timeout_ms passed (GR_ETIMEOUT). */
gr_status gr_wait(gr_ctx *ctx, uint64_t request_id, uint32_t timeout_ms, gr_request_status *status);
/* Stops a request between slices (a sliced render's film keeps the slices already
 * folded) or, in the lane, before it starts or between its chunks (the film is zero). */
gr_status gr_cancel(gr_ctx *ctx, uint64_t request_id);
/* Copies a finished (or cancelled) render's film, W*H*3 f32, to host memory. */
gr_status gr_request_film(gr_ctx *ctx, uint64_t request_id, float *xyz_host);
/* Copies a finished metrics request's n_poses results. */
gr_status gr_request_metrics(gr_ctx *ctx, uint64_t request_id, gr_metrics_out *out);
/* Frees a finished request and its film (GR_EBUSY while it is active). */
gr_status gr_request_release(gr_ctx *ctx, uint64_t request_id);

/* gr_render_resident that allocates no device memory.  No counterpart in the
 * reference (its frame renderer grows its buffers on demand, renderer/gpu/frame.rs:
 * 868-879); it exists for callers that must not allocate inside a render call.
 *
 * The per-tuple XYZ scratch is a fixed file-scope device array of
 * GR_STATIC_SCRATCH_BYTES (one per device per process) instead of the context's
 * growable buffer; the call makes no cudaMalloc / cudaFree and no library call that
 * allocates and always runs the PLAIN kernel.  The frame is
 * traced in chunks of floor(GR_STATIC_SCRATCH_TUPLES / spp) pixels, each folded into
 * the film before the next is traced (stream order), so results are identical to
 * gr_render_resident.  spp > GR_STATIC_SCRATCH_TUPLES (one pixel's samples do not fit)
 * is rejected with GR_EINVAL before any work.
 *
 * Nothing in the scratch needs to start at zero: each chunk's trace launch writes
 * every slot its fold then reads.  The film must hold the caller's running sum (the
 * call ADDS to it), exactly as for gr_render_resident.
 *
 * Set-up: the first call on each device looks up the array's address once
 * (cudaGetSymbolAddress, which may load the module); make that first call before any
 * stream capture begins.  A cudaDeviceReset in the process unloads the module and
 * leaves the cached address stale: after a reset, do not call this entry point again
 * in that process.  The call adds its launches to the counts gr_timing_read reports
 * (no timing events).  Races: the scratch is shared by every context on the
 * device, so calls whose device work may overlap (other contexts, or different
 * streams not ordered with each other) race on it; the caller must serialise them. */
#define GR_STATIC_SCRATCH_BYTES (16u << 20)
#define GR_STATIC_SCRATCH_TUPLES (GR_STATIC_SCRATCH_BYTES / 12u) /* 1,398,101 */
gr_status gr_render_resident_static(gr_ctx *ctx, uint64_t scene_id, uint32_t sample_offset, uint32_t spp,
                                    float *film_device, void *stream);

/* ---- frame-delta streaming (the worker's tracer / emitter split) ------------------ */

/* One render request streamed as FRAME deltas, replacing the worker's stream emitter
 * around the render path (apps/gemray-worker/src/stream_emit/: tracer.rs:64-117
 * run_tracer, emitter.rs:46-96 PendingDelta, sizing.rs:22-30 next_batch_size,
 * downsample.rs:17-53 downsample_preview; apps/gemray-worker/docs/architecture.md:
 * 33-129).  gr_stream_open starts a tracer thread that renders samples
 * [first_sample, first_sample + samples) of a resident scene in sub-batches, each
 * sized from the previous one's device time toward target_ms (x4 growth at most,
 * never 0), starting at first_batch samples; every sub-batch is traced into a zeroed
 * film (one per-pixel sum in sample order, the film a render_core::
 * trace_samples_with_gpu call returns) and then folded into the pending delta (copied
 * when the delta is empty, else added) and into the running total (added).  The
 * caller drains the delta on its own cadence with gr_stream_take: the payload is the
 * radiance wire format itself (W*H*3 little-endian f32 = W*H*12 bytes,
 * crates/gemray-net/src/radiance/mod.rs:26-67) and its contiguous sample range.
 * Drains never wait for a sub-batch in progress: the tracer folds into one of two
 * delta buffers while the other is copied out.  Cancellation (gr_stream_cancel) is
 * observed between sub-batches; the pending delta is then discarded.  fixed_batch != 0
 * replaces the adaptive sizing by sub-batches of exactly that many samples (the last
 * one shorter).  A stream keeps its scene resident: gr_scene_release returns
 * GR_EBUSY until the stream is closed.  Calls on one stream are thread-safe, except
 * that none may overlap its gr_stream_close. */
typedef struct gr_stream_opts {
    uint32_t target_ms;   /* sub-batch device-time target; 0 = 100 (sizing.rs:7) */
    uint32_t first_batch; /* first sub-batch in samples; 0 = 1 (tracer.rs:82) */
    uint32_t fixed_batch; /* != 0: every sub-batch has this many samples */
    uint32_t reserved;
} gr_stream_opts;

typedef enum gr_stream_state {
    GR_STREAM_RUNNING = 0,
    GR_STREAM_FINISHED = 1,  /* every sample traced and folded */
    GR_STREAM_CANCELLED = 2, /* stopped between sub-batches by gr_stream_cancel */
    GR_STREAM_FAILED = 3     /* a CUDA error stopped the tracer; see gr_stream_status */
} gr_stream_state;

gr_status gr_stream_open(gr_ctx *ctx, uint64_t scene_id, uint32_t first_sample, uint32_t samples,
                         const gr_stream_opts *opts /* NULL = defaults */, uint64_t *out_stream);
/* The pending delta (PendingDelta::take): writes W*H*3 floats to xyz_host and its
 * range; *samples = 0 (and nothing written) when nothing is pending or the stream was
 * cancelled. */
gr_status gr_stream_take(gr_ctx *ctx, uint64_t stream, uint32_t *first_sample, uint32_t *samples, float *xyz_host);
/* samples folded so far, the gr_stream_state, and the tracer's error (GR_OK unless
 * FAILED). */
gr_status gr_stream_status(gr_ctx *ctx, uint64_t stream, uint32_t *samples_done, uint32_t *state,
                           gr_status *tracer_error);
/* The running total (W*H*3 floats), as of the last folded sub-batch. */
gr_status gr_stream_total(gr_ctx *ctx, uint64_t stream, float *xyz_host);
/* downsample_preview of the running total to tw x th (box mean, tw/th 0 -> 1). */
gr_status gr_stream_preview(gr_ctx *ctx, uint64_t stream, uint32_t tw, uint32_t th, float *xyz_host);
gr_status gr_stream_cancel(gr_ctx *ctx, uint64_t stream);
/* Stops the tracer (as gr_stream_cancel), joins it and frees the stream. */
gr_status gr_stream_close(gr_ctx *ctx, uint64_t stream);
/* The sizing rule (sizing.rs:22-30): prev * target / elapsed, clamped to
 * [1, max(prev * 4, 1)] (u32 saturating), rounded; elapsed 0 -> max(prev * 4, 1). */
uint32_t gr_next_batch_size(uint32_t prev, double elapsed_ms, double target_ms);

/* ---- denoiser: guide pass and edge-avoiding A-Trous ------------------------------- */

/* = AtrousParams (crates/gemray/src/renderer/denoise/mod.rs:188-230); a NULL params
 * pointer means AtrousParams::default(): 5 passes, sigma_color 0.35, sigma_depth 0.1,
 * normal_power 64, taper_reference_spp 4, taper_identity_epsilon 0.02. */
typedef struct gr_atrous_params {
    uint32_t num_passes; /* clamped to [1, 8]; pass k dilates the 5x5 B3 kernel by 2^k */
    float sigma_color;   /* scaled by the taper 1 / sqrt(1 + spp / taper_reference_spp) */
    float sigma_depth;
    float normal_power;
    float taper_reference_spp;
    float taper_identity_epsilon; /* taper below this: the output is the input, bit for bit */
} gr_atrous_params;

/* The guide pass (apps/diagram-gui/src/bridge/guide_pass.rs, generate_guide_buffers):
 * for each pixel the primary ray through the pixel's corner (zero jitter) against the
 * scene's planes -- depth = hit t, normal = the hit plane's normal, facet_id = its
 * index, or (1e6, 0, -1) on a miss.  Reads only the scene's camera, width, height and
 * planes.  Host outputs (W*H, W*H*3, W*H), or device outputs ordered on `stream`. */
gr_status gr_guide_buffers(gr_ctx *ctx, const gr_scene *scene, float *depth, float *normal, int32_t *facet_id);
gr_status gr_guide_buffers_device(gr_ctx *ctx, const gr_scene *scene, float *depth, float *normal,
                                  int32_t *facet_id, void *stream);

/* AtrousDenoiser::denoise_into (denoise/mod.rs:560-684): `color` is the averaged XYZ
 * image (W*H*3), guides as produced by the guide pass, spp the sample count behind
 * the average; out (W*H*3) must not alias color.  Host or device buffers. */
gr_status gr_atrous_denoise(gr_ctx *ctx, const float *color, const float *depth, const float *normal,
                            const int32_t *facet_id, uint32_t width, uint32_t height, uint32_t spp,
                            const gr_atrous_params *params, float *out);
gr_status gr_atrous_denoise_device(gr_ctx *ctx, const float *color, const float *depth, const float *normal,
                                   const int32_t *facet_id, uint32_t width, uint32_t height, uint32_t spp,
                                   const gr_atrous_params *params, float *out, void *stream);

/* denoise_and_tonemap_frame (apps/diagram-gui/src/bridge/render_thread/denoise.rs):
 * the running-sum film scaled by 1 / sample_count, denoised with spp = sample_count,
 * tone-mapped at scale 1 to RGBA8 (W*H*4) -- all on the device. */
gr_status gr_denoise_tonemap_device(gr_ctx *ctx, const float *film, uint32_t sample_count, const float *depth,
                                    const float *normal, const int32_t *facet_id, uint32_t width, uint32_t height,
                                    const gr_atrous_params *params, void *rgba, void *stream);

/* ---- engine controls ---------------------------------------------------------- */

/* Transport kernel selection for single-scene renders.  PLAIN: one thread per
 * (pixel, sample) tuple, the reference kernel's launch shape.  WAVEFRONT and REGEN are
 * retired schedules (a global-queue wavefront engine, ~0.3x, and per-warp path
 * regeneration, 0.91x of STAGED on B200): both values are accepted and run AUTO's
 * choice.  STAGED: PLAIN's launch shape
 * with paths capped at 12 bounces; the ones still alive are parked and resumed, packed
 * densely, by a second kernel (capped at 20, then a third), so warps stop waiting on
 * a few long paths (+24-28% from 4 M tuples per launch up, e.g. the c2 frame).  AUTO
 * (default): STAGED for launches of at least GR_AUTO_STAGED_MIN_TUPLES tuples, PLAIN
 * below, where STAGED's extra launches and tails cost more than they save (measured
 * on B200: PLAIN 1.2x faster at 0.26 M tuples, STAGED 1.09x faster at 1.05 M).
 * Results are identical (same arithmetic per path). */
#define GR_KERNEL_PLAIN 0u
#define GR_KERNEL_WAVEFRONT 1u
#define GR_KERNEL_REGEN 2u
#define GR_KERNEL_STAGED 3u
#define GR_KERNEL_AUTO 4u
/* SORTED: clear isotropic stones (no birefringence, no absorption, no frosted facets or
 * scattering) only -- other scenes run AUTO's choice.  Each block keeps 128 paths in
 * shared memory and advances them bounce by bounce, any thread taking any path: dead
 * paths are finished and replaced by the launch's next tuples, and at every bounce the
 * reflecting and the refracting paths go to separate warps. */
#define GR_KERNEL_SORTED 5u
#define GR_AUTO_STAGED_MIN_TUPLES (1u << 19)
gr_status gr_set_kernel(gr_ctx *ctx, uint32_t kernel);

/* The staged schedule of a resident scene's renders: bounce caps of stages 1 and 2 and
 * the resident blocks per SM the kernels' register allocation targets (9, 10, 12 or 16:
 * 56, 48, 40 or 32 registers per thread).  Every schedule gives the same films; the
 * fastest depends on the stone (measured on B200: caps 12 / 20 on the c2 brilliant,
 * 8 / 16 on the c3 emerald, 3.8% faster there; 16 blocks per SM 6-8% faster than 9 on
 * both).  From the scene's second staged gr_render_resident call on, calls are timed with
 * device events as trials, in two rounds: caps 12 / 20 at each blocks-per-SM target, then
 * caps 8 / 16 and 16 / 28 at the fastest target; the schedule with the least time per
 * tuple is kept for the scene and entered in the context's tuning table.  Writes zeros
 * while the choice is still open (the built-in schedule, caps 12 / 20 at 16 blocks per
 * SM, runs meanwhile).  Batched launches (gr_render_batch, the request loop) run each
 * scene with its chosen first cap (their continuation stage is uncapped); gr_accumulate
 * and gr_accumulate_device choose the same way per stone (planes, finishes, material,
 * depth, flags and environment kind; not the view); a frame stream uses its scene's schedule as chosen when
 * the stream opened.  Scenes that need the frosted / scattering / biaxial kernels run
 * those at 9 blocks per SM whatever the schedule's target.  gr_scene_stage_caps reports
 * the caps alone. */
gr_status gr_scene_stage_caps(gr_ctx *ctx, uint64_t scene_id, uint32_t *cap_first, uint32_t *cap_second);
gr_status gr_scene_schedule(gr_ctx *ctx, uint64_t scene_id, uint32_t *cap_first, uint32_t *cap_second,
                            uint32_t *blocks_per_sm);
/* Pins a resident scene's schedule to one of the candidates (GR_EINVAL for any other
 * triple); (0, 0, 0) forgets the stone's choice and times the candidates afresh. */
gr_status gr_scene_set_schedule(gr_ctx *ctx, uint64_t scene_id, uint32_t cap_first, uint32_t cap_second,
                                uint32_t blocks_per_sm);

/* The context's tuning table: one schedule per stone (the scene key gr_accumulate uses),
 * measured on this device or loaded.  A stone met again -- a new upload, a new
 * gr_accumulate stone -- starts from its entry without trials.  gr_tuning_save writes it
 * as text (a first line naming GR_SCHEDULE_SET and the device label, then one
 * "key first second blocks ms_per_mtuple" line per stone), merged over the entries the
 * file already holds for the same device, through a renamed temporary file.
 * gr_tuning_load reads one (GR_EINVAL if it names another schedule set or device;
 * GR_ENOTFOUND if it cannot be read) and gives open scenes their entries.  With the
 * environment variable GR_TUNING_CACHE set to a path, gr_create loads that file and
 * gr_destroy saves to it: a per-device schedule cache across processes. */
#define GR_SCHEDULE_SET 2
gr_status gr_tuning_save(gr_ctx *ctx, const char *path);
gr_status gr_tuning_load(gr_ctx *ctx, const char *path, uint32_t *n_loaded);
gr_status gr_tuning_count(gr_ctx *ctx, uint32_t *n_entries);

/* Per-launch timing: while enabled, every trace and film-fold launch is bracketed by
 * CUDA events on its own stream.  gr_timing_read waits for them, returns the summed
 * kernel milliseconds and launch counts since the last read (or enable), and resets. */
gr_status gr_timing_enable(gr_ctx *ctx, uint32_t on);
gr_status gr_timing_read(gr_ctx *ctx, double *trace_ms, double *fold_ms, uint64_t *trace_launches,
                         uint64_t *fold_launches);

/* Waits for all work enqueued on the context's stream. */
gr_status gr_synchronize(gr_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t) for callers that enqueue around it. */
void *gr_stream(gr_ctx *ctx);

/* ---- scene builders (host only, no device work) --------------------------------- */

/* = Camera::new(yaw, pitch, distance, fov_deg) (optics/raytracer/camera.rs:62-93). */
gr_status gr_camera_new(float yaw, float pitch, float distance, float fov_deg, gr_camera *out);

/* = StandardGemCuts::standard_round_brilliant (geometry/cuts.rs:45-129): writes up to
 * cap planes and returns the full count (74). */
uint32_t gr_standard_round_brilliant(gr_plane *out, uint32_t cap);

/* = GpuGemMaterial::encode(&GemMaterial::by_name(name)) for the 13 built-in materials
 * (optics/materials.rs:136-1250, renderer/buffers.rs:313-385); exact-name match.
 * GR_ENOTFOUND for an unknown name. */
gr_status gr_builtin_material(const char *name, gr_material *out);

#ifdef __cplusplus
} /* extern "C" */
#endif

#ifdef __cplusplus
static_assert(sizeof(gr_plane) == 16, "gr_plane = GpuFacetPlane");
static_assert(sizeof(gr_band) == 12, "gr_band = GpuAbsorptionBand");
static_assert(sizeof(gr_dispersion) == 96, "gr_dispersion = DispersionParams");
static_assert(offsetof(gr_dispersion, param_a) == 16, "layout");
static_assert(offsetof(gr_dispersion, c_axis_and_birefringence) == 64, "layout");
static_assert(offsetof(gr_dispersion, is_anisotropic) == 80, "layout");
static_assert(sizeof(gr_material) == 432, "gr_material = GpuGemMaterial");
static_assert(offsetof(gr_material, crystal_system) == 96, "layout");
static_assert(offsetof(gr_material, o_ray_bands) == 116, "layout");
static_assert(offsetof(gr_material, e_ray_bands) == 212, "layout");
static_assert(offsetof(gr_material, scattering_sigma_s) == 308, "layout");
static_assert(offsetof(gr_material, beta_ray_bands) == 328, "layout");
static_assert(offsetof(gr_material, absorption_path_scale) == 424, "layout");
static_assert(sizeof(gr_camera) == 52, "gr_camera");
static_assert(sizeof(gr_metrics_out) == 20, "gr_metrics_out = GemOpticalMetrics");
static_assert(sizeof(gr_request) == 64, "gr_request");
static_assert(sizeof(gr_request_status) == 32, "gr_request_status");
#endif

#endif /* GEMRAY_CUDA_H */
