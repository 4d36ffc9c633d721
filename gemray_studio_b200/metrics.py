"""Optical metrics on the device: the reference's color/metrics.rs entry points over
the C ABI (``gr_optical_metrics`` / ``gr_angular_profile``).

Names, argument order and units (radians) follow crates/gemray/src/color/metrics.rs;
the extra first argument is the engine context (a ``GpuFrameRenderer``).  Poses are
evaluated as one device batch, so a tilt sweep or a pose grid costs one launch pair.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from .backend import GpuFrameRenderer, _raise_for

# color/metrics.rs:42-45
PROFILE_ANGLES_DEG = tuple(float(5 * i) for i in range(19))


@dataclass(frozen=True)
class GemOpticalMetrics:
    """= GemOpticalMetrics (color/metrics.rs:33-39)."""

    brilliance_pct: float
    fire_index: float
    scintillation_pct: float
    windowing_pct: float
    extinction_pct: float


def _planes_arg(planes):
    p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
    return p, p.ctypes.data_as(C.c_void_p), p.shape[0]


def evaluate_poses(r: GpuFrameRenderer, planes, material: abi.gr_material, poses, fp64_sums: bool = False) -> np.ndarray:
    """Metrics for each row (cam_yaw, cam_pitch, light_yaw, light_pitch) of `poses`;
    returns an (N, 5) float32 array in GemOpticalMetrics field order."""
    poses = np.ascontiguousarray(poses, np.float32).reshape(-1, 4)
    n = poses.shape[0]
    out = (abi.gr_metrics_out * max(n, 1))()
    keep, pp, npl = _planes_arg(planes)
    pz = poses.ctypes.data_as(C.POINTER(abi.gr_pose))
    st = r.lib.gr_optical_metrics(r.ctx, pp, npl, C.byref(material), pz, n,
                                  abi.GR_METRICS_FP64_SUMS if fp64_sums else 0, out)
    _raise_for(r.lib, st)
    return np.ctypeslib.as_array(out).view(np.float32).reshape(-1, 5)[:n].copy()


def evaluate_gem_optical_metrics(r: GpuFrameRenderer, planes, material: abi.gr_material, cam_yaw: float,
                                 cam_pitch: float, light_yaw: float, light_pitch: float) -> GemOpticalMetrics:
    """= evaluate_gem_optical_metrics (color/metrics.rs:1082-1237)."""
    row = evaluate_poses(r, planes, material, [[cam_yaw, cam_pitch, light_yaw, light_pitch]])[0]
    return GemOpticalMetrics(*(float(x) for x in row))


def evaluate_angular_profile_at_azimuth(r: GpuFrameRenderer, planes, material: abi.gr_material, cam_yaw: float,
                                        light_yaw: float, light_pitch: float):
    """= evaluate_angular_profile_at_azimuth (color/metrics.rs:1262-1289): the
    (brilliance, extinction, windowing) curves over PROFILE_ANGLES_DEG."""
    b, e, w = (np.zeros(19, np.float32) for _ in range(3))
    keep, pp, npl = _planes_arg(planes)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    st = r.lib.gr_angular_profile(r.ctx, pp, npl, C.byref(material), cam_yaw, light_yaw, light_pitch, fp(b), fp(e), fp(w))
    _raise_for(r.lib, st)
    return b, e, w


def evaluate_angular_profile(r: GpuFrameRenderer, planes, material: abi.gr_material, light_yaw: float,
                             light_pitch: float):
    """= evaluate_angular_profile (color/metrics.rs:1299-1306): azimuth 0."""
    return evaluate_angular_profile_at_azimuth(r, planes, material, 0.0, light_yaw, light_pitch)
