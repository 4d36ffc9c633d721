"""Loader for the oracle library (oracle/libgr_oracle.so) used by the test suite.

The oracle is test infrastructure: a CPU restatement of the reference tracer that the
CUDA engine is checked against.  Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

from gemray_studio_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "libgr_oracle.so"
ORACLE_LIB_AVX2 = ORACLE_DIR / "libgr_oracle_avx2.so"


def _host_has_avx2() -> bool:
    try:
        flags = Path("/proc/cpuinfo").read_text()
    except OSError:
        return False
    return " avx2 " in flags and " fma " in flags and " bmi2 " in flags

_lib = None


def build_oracle() -> Path:
    sources = [ORACLE_DIR / n for n in ("gro_capi.cpp", "gr_oracle.hpp", "gro_scene.hpp", "Makefile")]
    newest = max(p.stat().st_mtime for p in sources)
    if any(not p.exists() or p.stat().st_mtime < newest for p in (ORACLE_LIB, ORACLE_LIB_AVX2)):
        subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
    return ORACLE_LIB


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not ORACLE_LIB.exists():
        build_oracle()
    path = ORACLE_LIB_AVX2 if ORACLE_LIB_AVX2.exists() and _host_has_avx2() else ORACLE_LIB
    L = C.CDLL(str(path))
    F = C.c_float
    U = C.c_uint32
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_uint32)
    sc = C.POINTER(abi.gr_scene)
    L.gro_hash_u32.restype = U
    L.gro_hash_u32.argtypes = [U]
    L.gro_rng_draw.restype = F
    L.gro_rng_draw.argtypes = [U, U, U]
    L.gro_radical_inverse.restype = F
    L.gro_radical_inverse.argtypes = [U, U]
    L.gro_sample_draws.restype = None
    L.gro_sample_draws.argtypes = [up, up, C.c_uint64, up, fp, fp, fp]
    L.gro_camera_new.restype = None
    L.gro_camera_new.argtypes = [F, F, F, F, C.POINTER(abi.gr_camera)]
    L.gro_standard_round_brilliant.restype = U
    L.gro_standard_round_brilliant.argtypes = [C.POINTER(abi.gr_plane), U]
    L.gro_builtin_material.restype = C.c_int
    L.gro_builtin_material.argtypes = [C.c_char_p, C.POINTER(abi.gr_material)]
    L.gro_white_balance.restype = None
    L.gro_white_balance.argtypes = [F, fp]
    L.gro_trace_samples_f64.restype = C.c_int
    L.gro_trace_samples_f64.argtypes = [C.POINTER(abi.gr_scene), U, U, U, U, fp, C.c_int]
    L.gro_furnace_target.restype = None
    L.gro_furnace_target.argtypes = [F, fp]
    L.gro_studio_env.restype = F
    L.gro_studio_env.argtypes = [fp, F, F, F, F, F, F]
    L.gro_studio_env_spec.restype = F
    L.gro_studio_env_spec.argtypes = [fp, F, F, F, F, F]
    L.gro_exp_poly.restype = F
    L.gro_exp_poly.argtypes = [F]
    L.gro_trace_ray.restype = C.c_int
    L.gro_trace_ray.argtypes = [sc, fp, fp, U, F, U, C.c_int, C.POINTER(C.c_double), up, up]
    L.gro_probe_grid.restype = C.c_int
    L.gro_probe_grid.argtypes = [sc, U, U, U, U, fp]
    L.gro_cosine_hemisphere.restype = None
    L.gro_cosine_hemisphere.argtypes = [F, F, fp, fp]
    L.gro_sample_hg.restype = None
    L.gro_sample_hg.argtypes = [F, F, F, fp, fp]
    L.gro_biaxial_wave_indices.restype = None
    L.gro_biaxial_wave_indices.argtypes = [F, F, F, fp, fp, fp]
    L.gro_biaxial_eigen.restype = None
    L.gro_biaxial_eigen.argtypes = [F, F, F, fp, fp, fp, fp]
    L.gro_biaxial_poynting.restype = None
    L.gro_biaxial_poynting.argtypes = [F, F, F, fp, fp, C.c_int, fp]
    L.gro_material_indicatrix.restype = C.c_int
    L.gro_material_indicatrix.argtypes = [C.POINTER(abi.gr_material), F, fp, fp]
    L.gro_downsample_preview.restype = None
    L.gro_downsample_preview.argtypes = [fp, U, U, U, U, fp]
    L.gro_guide_buffers.restype = None
    L.gro_guide_buffers.argtypes = [sc, fp, fp, C.POINTER(C.c_int32)]
    L.gro_taper_strength.restype = F
    L.gro_taper_strength.argtypes = [U, F]
    L.gro_cos_pow.restype = F
    L.gro_cos_pow.argtypes = [F, F]
    L.gro_atrous_denoise.restype = None
    L.gro_atrous_denoise.argtypes = [fp, fp, fp, C.POINTER(C.c_int32), U, U, U, U, F, F, F, F, F, fp]
    L.gro_shading_normal.restype = None
    L.gro_shading_normal.argtypes = [C.POINTER(abi.gr_plane), U, fp, C.c_int, fp, F, fp]
    L.gro_accumulate.restype = C.c_int
    L.gro_accumulate.argtypes = [sc, U, U, fp, C.c_int]
    L.gro_accumulate_f64.restype = C.c_int
    L.gro_accumulate_f64.argtypes = [sc, U, U, C.POINTER(C.c_double), C.c_int]
    L.gro_trace_samples.restype = C.c_int
    L.gro_trace_samples.argtypes = [sc, U, U, U, U, fp, up, up, up, C.c_int]
    L.gro_accumulate_rows.restype = C.c_int
    L.gro_accumulate_rows.argtypes = [sc, up, U, U, U, fp, C.c_int]
    L.gro_metrics.restype = None
    L.gro_metrics.argtypes = [C.POINTER(abi.gr_plane), U, C.POINTER(abi.gr_material), F, F, F, F, fp]
    L.gro_tonemap.restype = None
    L.gro_tonemap.argtypes = [fp, F, U, C.POINTER(C.c_uint8)]
    L.gro_material_channel.restype = C.c_int
    L.gro_material_channel.argtypes = [C.POINTER(abi.gr_material), C.POINTER(abi.gr_material_ext), F, C.c_int,
                                       C.POINTER(C.c_double)]
    L.gro_trace_events.restype = C.c_int
    L.gro_trace_events.argtypes = [sc, U, U, U, U, U, up, up, C.POINTER(C.c_int32), fp, C.POINTER(C.c_uint8), C.c_int]
    L.gro_case_bank.restype = C.c_int
    L.gro_case_bank.argtypes = [U, C.c_int, sc, fp, U, C.POINTER(C.c_double)]
    L.gro_case_bank_arity.restype = C.c_int
    L.gro_case_bank_arity.argtypes = [U, up, up]
    L.gro_intersect_rays.restype = C.c_int
    L.gro_intersect_rays.argtypes = [C.c_void_p, U, fp, U, C.c_int, fp, C.POINTER(C.c_int32)]
    L.gro_trace_samples_stokes.restype = C.c_int
    L.gro_trace_samples_stokes.argtypes = [sc, U, U, U, U, fp, fp, C.c_int]
    L.gro_accumulate_stokes.restype = C.c_int
    L.gro_accumulate_stokes.argtypes = [sc, U, U, fp, fp, C.c_int]
    L.gro_rng_records.restype = None
    L.gro_rng_records.argtypes = [up, up, U, up]
    _lib = L
    return L
