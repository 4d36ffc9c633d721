"""ctypes mirror of ``include/gemray_cuda.h``.

The structures here are byte-for-byte the C structs of the public header (which in
turn are byte-identical to the reference's ``GpuFacetPlane``, ``GpuAbsorptionBand``
and ``GpuGemMaterial``, crates/gemray/src/geometry/plane.rs:6-9 and
crates/gemray/src/renderer/buffers.rs:148-165,236-299).  ``load_library`` opens the
in-tree ``libgemray_cuda.so`` and declares every exported entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

GR_ABI_VERSION = 1
GR_MAX_BANDS = 8
GR_MAX_PLANES = 512
GR_MAX_BOUNCES = 4096

GR_OK = 0
GR_DECLINED_ENV = 1
GR_DECLINED_MATERIAL = 2
GR_NO_DEVICE = 3
GR_EINVAL = 4
GR_ENOMEM = 5
GR_ETIMEOUT = 6
GR_ECANCELLED = 7
GR_ECUDA = 8
GR_EBUSY = 9
GR_ENOTFOUND = 10

STATUS_NAMES = {
    0: "GR_OK", 1: "GR_DECLINED_ENV", 2: "GR_DECLINED_MATERIAL", 3: "GR_NO_DEVICE",
    4: "GR_EINVAL", 5: "GR_ENOMEM", 6: "GR_ETIMEOUT", 7: "GR_ECANCELLED", 8: "GR_ECUDA",
    9: "GR_EBUSY", 10: "GR_ENOTFOUND",
}

GR_DISP_SELLMEIER1 = 0
GR_DISP_SELLMEIER3 = 1
GR_DISP_CAUCHY = 2

GR_ENV_UNIFORM = 0
GR_ENV_STUDIO = 1
GR_ENV_LATLONG = 2

GR_FLAG_KAHAN_FILM = 0x1
GR_FLAG_FP64_RESOLVE = 0x2

EVENT_NAMES = ["paths", "bounces", "escapes", "tir", "reflect", "refract", "absorb", "channel_tir",
               "channel_refract", "roulette", "rotations", "aniso_bounces", "walkoff", "roulette_kills"]
GR_EVENT_COUNT = len(EVENT_NAMES)

GR_KERNEL_PLAIN = 0
GR_KERNEL_WAVEFRONT = 1
GR_KERNEL_REGEN = 2
GR_KERNEL_STAGED = 3
GR_KERNEL_AUTO = 4
GR_KERNEL_SORTED = 5
GR_AUTO_STAGED_MIN_TUPLES = 1 << 19
GR_STATIC_SCRATCH_BYTES = 16 << 20
GR_STATIC_SCRATCH_TUPLES = GR_STATIC_SCRATCH_BYTES // 12

# gr_trace_events: termination reasons and per-bounce events
GR_TERM_ESCAPED, GR_TERM_ROULETTE, GR_TERM_HIT_CAP = 0, 2, 3
GR_SEQ_TIR, GR_SEQ_REFLECT, GR_SEQ_REFRACT, GR_SEQ_SCATTER, GR_SEQ_NONE = 0, 1, 2, 3, 0xFF

# gr_case_bank: per-function case banks (layouts in include/gemray_cuda.h)
BANK_NAMES = ["camera_ray", "cmf", "blackbody", "dispersion", "absorption", "pleochroic", "fresnel_reflection",
              "fresnel_transmission", "frame_rotation", "tir_retardation", "signed_psi", "tir_phase_delta",
              "eigen_uniaxial", "walk_off", "extraordinary_index", "theta_c", "studio", "rgb_spectral", "exp_poly",
              "hg_sample", "cosine_hemisphere", "e_field", "von_kries", "wavelengths"]
GR_BANK = {n: i for i, n in enumerate(BANK_NAMES)}
GR_BANK_COUNT = len(BANK_NAMES)


class gr_plane(C.Structure):
    _fields_ = [("normal", C.c_float * 3), ("d", C.c_float)]


class gr_band(C.Structure):
    _fields_ = [("center_nm", C.c_float), ("width_nm", C.c_float), ("peak", C.c_float)]


class gr_dispersion(C.Structure):
    _fields_ = [
        ("model_type", C.c_uint32), ("pad0", C.c_uint32 * 3),
        ("param_a", C.c_float * 4), ("param_b", C.c_float * 4), ("param_c", C.c_float * 4),
        ("c_axis_and_birefringence", C.c_float * 4),
        ("is_anisotropic", C.c_uint32), ("biaxial_delta_beta_alpha", C.c_float),
        ("has_biaxial_delta", C.c_uint32), ("pad_tail", C.c_float),
    ]


class gr_material(C.Structure):
    _fields_ = [
        ("dispersion", gr_dispersion),
        ("crystal_system", C.c_uint32), ("optical_character", C.c_uint32),
        ("is_pleochroic", C.c_uint32), ("o_ray_band_count", C.c_uint32),
        ("e_ray_band_count", C.c_uint32),
        ("o_ray_bands", gr_band * GR_MAX_BANDS), ("e_ray_bands", gr_band * GR_MAX_BANDS),
        ("scattering_sigma_s", C.c_float), ("scattering_g", C.c_float),
        ("edge_rounding_radius", C.c_float), ("has_beta_ray", C.c_uint32),
        ("beta_ray_band_count", C.c_uint32), ("beta_ray_bands", gr_band * GR_MAX_BANDS),
        ("absorption_path_scale", C.c_float), ("pad_trailing", C.c_uint32),
    ]


class gr_camera(C.Structure):
    _fields_ = [
        ("origin", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
        ("up", C.c_float * 3), ("fov_tan", C.c_float),
    ]


class gr_metrics_out(C.Structure):
    _fields_ = [("brilliance_pct", C.c_float), ("fire_index", C.c_float), ("scintillation_pct", C.c_float),
                ("windowing_pct", C.c_float), ("extinction_pct", C.c_float)]


class gr_pose(C.Structure):
    _fields_ = [("cam_yaw", C.c_float), ("cam_pitch", C.c_float), ("light_yaw", C.c_float), ("light_pitch", C.c_float)]


GR_METRICS_FP64_SUMS = 0x1


class gr_batch_item(C.Structure):
    _fields_ = [("scene_id", C.c_uint64), ("film_device", C.c_void_p), ("sample_offset", C.c_uint32),
                ("spp", C.c_uint32)]


GR_BATCH_GRAPH = 0x1
GR_SCHEDULE_SET = 2
# staged schedules a stone chooses between: cap pairs x blocks per SM
SCHEDULE_CAP_PAIRS = ((12, 20), (8, 16), (16, 28))
SCHEDULE_BLOCKS = (9, 10, 12, 16)


GR_REQ_RENDER, GR_REQ_METRICS = 0, 1
GR_REQ_QUEUED, GR_REQ_RUNNING, GR_REQ_DONE, GR_REQ_CANCELLED, GR_REQ_FAILED = 0, 1, 2, 3, 4
REQUEST_STATES = {0: "queued", 1: "running", 2: "done", 3: "cancelled", 4: "failed"}


class gr_request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("slice_spp", C.c_uint32), ("scene_id", C.c_uint64),
                ("sample_offset", C.c_uint32), ("spp", C.c_uint32), ("flags", C.c_uint32), ("n_planes", C.c_uint32),
                ("planes", C.c_void_p), ("material", C.c_void_p), ("poses", C.c_void_p), ("n_poses", C.c_uint32),
                ("reserved", C.c_uint32)]


class gr_request_status(C.Structure):
    _fields_ = [("state", C.c_uint32), ("samples_done", C.c_uint32), ("error", C.c_int), ("reserved", C.c_uint32),
                ("queued_ms", C.c_double), ("latency_ms", C.c_double)]


class gr_stream_opts(C.Structure):
    _fields_ = [("target_ms", C.c_uint32), ("first_batch", C.c_uint32), ("fixed_batch", C.c_uint32),
                ("reserved", C.c_uint32)]


GR_STREAM_RUNNING, GR_STREAM_FINISHED, GR_STREAM_CANCELLED, GR_STREAM_FAILED = 0, 1, 2, 3


class gr_atrous_params(C.Structure):
    _fields_ = [("num_passes", C.c_uint32), ("sigma_color", C.c_float), ("sigma_depth", C.c_float),
                ("normal_power", C.c_float), ("taper_reference_spp", C.c_float),
                ("taper_identity_epsilon", C.c_float)]


class gr_environment(C.Structure):
    _fields_ = [
        ("mode", C.c_uint32), ("uniform_rgb", C.c_float * 3),
        ("temp_k", C.c_float), ("spot_mult", C.c_float), ("exposure", C.c_float),
        ("light_yaw", C.c_float), ("light_pitch", C.c_float),
        ("latlong_rgb", C.POINTER(C.c_float)), ("latlong_w", C.c_uint32), ("latlong_h", C.c_uint32),
    ]


class gr_material_ext(C.Structure):
    _fields_ = [
        ("n_absorption", C.c_uint32), ("absorption_nm_first", C.c_float),
        ("absorption_nm_step", C.c_float),
        ("alpha_o_table", C.POINTER(C.c_float)), ("alpha_e_table", C.POINTER(C.c_float)),
        ("has_cauchy_e", C.c_uint32), ("cauchy_e", C.c_float * 3),
    ]


class gr_scene(C.Structure):
    _fields_ = [
        ("camera", gr_camera),
        ("width", C.c_uint32), ("height", C.c_uint32), ("max_bounces", C.c_uint32),
        ("n_planes", C.c_uint32),
        ("planes", C.POINTER(gr_plane)), ("finishes", C.POINTER(C.c_uint32)),
        ("material", C.POINTER(gr_material)), ("material_ext", C.POINTER(gr_material_ext)),
        ("env", gr_environment), ("flags", C.c_uint32), ("reserved", C.c_uint32),
    ]


class gr_rng_record(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("jitter_x", C.c_float), ("jitter_y", C.c_float),
                ("hero_rand", C.c_float), ("draws", (C.c_float * 4) * 4)]


class gr_create_opts(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("chunk_budget_bytes", C.c_uint64),
        ("serve_budget_bytes", C.c_uint64),
    ]


assert C.sizeof(gr_plane) == 16
assert C.sizeof(gr_band) == 12
assert C.sizeof(gr_dispersion) == 96
assert C.sizeof(gr_material) == 432
assert gr_material.o_ray_bands.offset == 116
assert gr_material.absorption_path_scale.offset == 424
assert C.sizeof(gr_camera) == 52

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_NAME = "libgemray_cuda.so"


def library_path() -> Path:
    return PACKAGE_DIR / LIB_NAME


# (name, restype, argtypes) of every entry point declared in include/gemray_cuda.h.
_ctx_p = C.c_void_p
EXPORTS = [
    ("gr_create", C.c_int, [C.POINTER(_ctx_p), C.POINTER(gr_create_opts)]),
    ("gr_destroy", C.c_int, [_ctx_p]),
    ("gr_device_label", C.c_char_p, [_ctx_p]),
    ("gr_last_error_string", C.c_char_p, []),
    ("gr_abi_version", C.c_uint32, []),
    ("gr_accumulate", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
    ("gr_accumulate_device", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("gr_trace_samples", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.POINTER(C.c_float)]),
    ("gr_accumulate_stokes", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.POINTER(C.c_float),
                                       C.POINTER(C.c_float)]),
    ("gr_tonemap", C.c_int, [_ctx_p, C.POINTER(C.c_float), C.c_float, C.c_uint32, C.POINTER(C.c_uint8)]),
    ("gr_rng_records", C.c_int, [_ctx_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint32,
                                 C.POINTER(gr_rng_record)]),
    ("gr_event_counts", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.POINTER(C.c_uint64), C.c_uint32]),
    ("gr_probe_fp32_peak", C.c_int, [_ctx_p, C.POINTER(C.c_double)]),
    ("gr_trace_events", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_float), C.POINTER(C.c_uint8)]),
    ("gr_case_bank_arity", C.c_int, [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("gr_case_bank", C.c_int, [_ctx_p, C.c_uint32, C.POINTER(gr_scene), C.POINTER(C.c_float), C.c_uint32,
                               C.POINTER(C.c_float)]),
    ("gr_device_code_version", C.c_int, [_ctx_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("gr_intersect_rays", C.c_int, [_ctx_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.c_uint32,
                                    C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    ("gr_optical_metrics", C.c_int, [_ctx_p, C.c_void_p, C.c_uint32, C.POINTER(gr_material), C.POINTER(gr_pose),
                                     C.c_uint32, C.c_uint32, C.POINTER(gr_metrics_out)]),
    ("gr_angular_profile", C.c_int, [_ctx_p, C.c_void_p, C.c_uint32, C.POINTER(gr_material), C.c_float, C.c_float,
                                     C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    ("gr_scene_upload", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.POINTER(C.c_uint64)]),
    ("gr_scene_release", C.c_int, [_ctx_p, C.c_uint64]),
    ("gr_render_resident", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("gr_render_resident_static", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("gr_render_batch", C.c_int, [_ctx_p, C.POINTER(gr_batch_item), C.c_uint32, C.c_uint32, C.c_void_p]),
    ("gr_submit", C.c_int, [_ctx_p, C.POINTER(gr_request), C.POINTER(C.c_uint64)]),
    ("gr_poll", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(gr_request_status)]),
    ("gr_wait", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.POINTER(gr_request_status)]),
    ("gr_cancel", C.c_int, [_ctx_p, C.c_uint64]),
    ("gr_request_film", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_float)]),
    ("gr_request_metrics", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(gr_metrics_out)]),
    ("gr_request_release", C.c_int, [_ctx_p, C.c_uint64]),
    ("gr_stream_open", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(gr_stream_opts),
                                 C.POINTER(C.c_uint64)]),
    ("gr_stream_take", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_float)]),
    ("gr_stream_status", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_int)]),
    ("gr_stream_total", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_float)]),
    ("gr_stream_preview", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
    ("gr_stream_cancel", C.c_int, [_ctx_p, C.c_uint64]),
    ("gr_stream_close", C.c_int, [_ctx_p, C.c_uint64]),
    ("gr_next_batch_size", C.c_uint32, [C.c_uint32, C.c_double, C.c_double]),
    ("gr_guide_buffers", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.POINTER(C.c_int32)]),
    ("gr_guide_buffers_device", C.c_int, [_ctx_p, C.POINTER(gr_scene), C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    ("gr_atrous_denoise", C.c_int, [_ctx_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_int32), C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.POINTER(gr_atrous_params), C.POINTER(C.c_float)]),
    ("gr_atrous_denoise_device", C.c_int, [_ctx_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.POINTER(gr_atrous_params), C.c_void_p,
                                           C.c_void_p]),
    ("gr_denoise_tonemap_device", C.c_int, [_ctx_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_uint32, C.c_uint32, C.POINTER(gr_atrous_params), C.c_void_p,
                                            C.c_void_p]),
    ("gr_timing_enable", C.c_int, [_ctx_p, C.c_uint32]),
    ("gr_timing_read", C.c_int, [_ctx_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64)]),
    ("gr_set_kernel", C.c_int, [_ctx_p, C.c_uint32]),
    ("gr_scene_stage_caps", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("gr_scene_schedule", C.c_int, [_ctx_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]),
    ("gr_scene_set_schedule", C.c_int, [_ctx_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]),
    ("gr_tuning_save", C.c_int, [_ctx_p, C.c_char_p]),
    ("gr_tuning_load", C.c_int, [_ctx_p, C.c_char_p, C.POINTER(C.c_uint32)]),
    ("gr_tuning_count", C.c_int, [_ctx_p, C.POINTER(C.c_uint32)]),
    ("gr_synchronize", C.c_int, [_ctx_p]),
    ("gr_stream", C.c_void_p, [_ctx_p]),
    ("gr_camera_new", C.c_int, [C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(gr_camera)]),
    ("gr_builtin_material", C.c_int, [C.c_char_p, C.POINTER(gr_material)]),
    ("gr_standard_round_brilliant", C.c_uint32, [C.POINTER(gr_plane), C.c_uint32]),
]

_lib = None


class LibraryMissing(RuntimeError):
    """The CUDA engine's shared library is not built (run __graft_entry__.build())."""


def load_library(path: os.PathLike | None = None):
    """Open libgemray_cuda.so (in-tree) and declare its entry points.

    Raises LibraryMissing if the library has not been built: the engine has no
    CPU fallback.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else library_path()
    if not p.exists():
        raise LibraryMissing(f"{p} not found; build it with __graft_entry__.build()")
    lib = C.CDLL(str(p))
    for name, res, args in EXPORTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
